// Vector, reduction, regulariser and layout kernels.
//
// The elementwise kernels restate Core/src/blas.hpp (init_data, clamp_min,
// invert_x, invert_min_x, sum_axpy, scal_xby) and the regularisers restate
// Core/src/tikhonov.cpp and Core/src/total_v.cpp; operations whose rounding
// the reference fixes are written with explicitly rounded intrinsics so the
// results agree bit for bit.  The CGLS step scalars are the one intentional
// change: their inner products are FP64 sums (deterministic two-stage
// reductions), where the reference sums in float.
#include "common.cuh"
#include "kernels.h"

namespace ccpi {
namespace {

constexpr int kThreads = 256;
constexpr int kGrid = 148 * 8; // 8 CTAs per SM on the 148-SM B200

__global__ void fill_kernel(float *p, i64 n, float v) {
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x)
    p[i] = v;
}

// blas.hpp:100-116 invert_min_x(x, 0): x > 0 ? 1/x : 0.  The reference
// divides in double and rounds to float, which equals the float quotient.
__global__ void invert_pos_kernel(float *p, i64 n) {
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x) {
    const float x = p[i];
    p[i] = (x > 0.0f) ? __fdiv_rn(1.0f, x) : 0.0f;
  }
}

// blas.hpp:86-98 invert_x: x != 0 ? 1/x : x.
__global__ void invert_nonzero_kernel(float *p, i64 n) {
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x) {
    const float x = p[i];
    if (x != 0.0f)
      p[i] = __fdiv_rn(1.0f, x);
  }
}

__global__ void clamp0_kernel(float *p, i64 n) {
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x) {
    const float x = p[i];
    p[i] = (x < 0.0f) ? 0.0f : x;
  }
}

__global__ void sumsq_kernel(const float *__restrict__ x, i64 n, double *partials) {
  __shared__ double red[kThreads / 32];
  double t = 0.0;
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x) {
    const double v = x[i];
    t += v * v;
  }
  t = cta_sum<kThreads / 32>(t, red);
  if (threadIdx.x == 0)
    partials[blockIdx.x] = t;
}

__device__ double block_sum_fixed(const double *p, int n, double *red) {
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    t += p[i];
  return cta_sum<kThreads / 32>(t, red);
}

// s[0] = |r|^2 of the current search direction's normal equations,
// s[1] = alpha, s[2] = beta, s[3] = iteration counter.
__global__ void cgls_scalars_kernel(int op, const double *p1, int n1, const double *p2, int n2,
                                    double *s, double *norms) {
  __shared__ double red[kThreads / 32];
  const double a = block_sum_fixed(p1, n1, red);
  const double b = (op == S_ALPHA2) ? block_sum_fixed(p2, n2, red) : 0.0;
  if (threadIdx.x != 0)
    return;
  switch (op) {
  case S_INIT:
    s[0] = a;
    s[1] = 0.0;
    s[2] = 0.0;
    s[3] = 0.0;
    break;
  case S_ALPHA:
  case S_ALPHA2: {
    const double den = a + b;
    s[1] = (den > 0.0) ? s[0] / den : 0.0;
    break;
  }
  case S_BETA: {
    s[2] = (s[0] > 0.0) ? a / s[0] : 0.0;
    s[0] = a;
    if (norms)
      norms[int(s[3])] = sqrt(a);
    s[3] += 1.0;
    break;
  }
  }
}

// Step scalars of a solve whose volume is cut into slabs over several
// ranks.  sum[0] is the one double the ranks all-reduce between stages:
// SH_LOCAL writes this rank's FP64 sum of the partials (p1, then p2), the
// other ops read the all-reduced total.  s[] as in cgls_scalars_kernel.
__global__ void shard_scalars_kernel(int op, const double *p1, int n1, const double *p2, int n2,
                                     double *sum, double *s, double *norms) {
  __shared__ double red[kThreads / 32];
  if (op == SH_LOCAL) {
    const double a = block_sum_fixed(p1, n1, red);
    const double b = p2 ? block_sum_fixed(p2, n2, red) : 0.0;
    if (threadIdx.x == 0)
      sum[0] = a + b;
    return;
  }
  if (threadIdx.x != 0)
    return;
  const double t = sum[0];
  switch (op) {
  case SH_INIT:
    s[0] = t;
    s[1] = 0.0;
    s[2] = 0.0;
    s[3] = 0.0;
    break;
  case SH_ALPHA:
    s[1] = (t > 0.0) ? s[0] / t : 0.0;
    break;
  case SH_BETA:
    s[2] = (s[0] > 0.0) ? t / s[0] : 0.0;
    s[0] = t;
    if (norms)
      norms[int(s[3])] = sqrt(t);
    s[3] += 1.0;
    break;
  }
}

// The first and last z planes of a slab, [x][y] each: what the neighbouring
// slabs take as their halo planes.
__global__ void pack_edges_kernel(const float *__restrict__ a, int nxy, int nz, float *lo,
                                  float *hi) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nxy; c += gridDim.x * blockDim.x) {
    lo[c] = a[i64(c) * nz];
    hi[c] = a[i64(c) * nz + nz - 1];
  }
}

// blas.hpp:307-322 sum_axpy: y += a x, a rounded to float, unfused.
__global__ void axpy_scalar_kernel(float *y, const float *__restrict__ x, i64 n, const double *s,
                                   int idx, float sign) {
  const float a = float(s[idx]) * sign;
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x)
    y[i] = __fadd_rn(y[i], __fmul_rn(a, x[i]));
}

// x += alpha d (cgls.cpp:120), then d = s + beta d (blas.hpp:362-376).
__global__ void cgls_xd_kernel(float *x, float *d, const float *__restrict__ sv, i64 n,
                               const double *s) {
  const float a = float(s[1]), b = float(s[2]);
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x) {
    const float dv = d[i];
    x[i] = __fadd_rn(x[i], __fmul_rn(a, dv));
    d[i] = __fadd_rn(__fmul_rn(b, dv), sv[i]);
  }
}

__global__ void cgls_d_kernel(float *d, const float *__restrict__ sv, i64 n, const double *s) {
  const float b = float(s[2]);
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x)
    d[i] = __fadd_rn(__fmul_rn(b, d[i]), sv[i]);
}

__global__ void add_scaled_kernel(float *out, const float *in, const float *__restrict__ d,
                                  i64 n, const double *s) {
  const float a = float(s[1]);
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n; i += i64(gridDim.x) * blockDim.x)
    out[i] = __fadd_rn(in[i], __fmul_rn(a, d[i]));
}

// ---------------------------------------------------------- regularisers
// A volume [x][y][z], optionally one slab of a volume cut along z: lo / hi
// then hold the neighbouring slabs' adjacent planes (nx * ny, [x][y]),
// which stand in for the planes k = -1 and k = nz; without them the z
// neighbours mirror at the ends as in the reference.
struct Vol {
  const float *a;
  int nx, ny, nz;
  const float *lo = nullptr, *hi = nullptr;
  __device__ float at(int i, int j, int k) const {
    if (k < 0)
      return lo[i64(i) * ny + j];
    if (k >= nz)
      return hi[i64(i) * ny + j];
    return a[(i64(i) * ny + j) * nz + k];
  }
  // z neighbours: across a cut into the halo plane (a halo plane's own
  // outer neighbour, which no result uses, reads the halo plane again)
  __device__ int zdn(int k) const {
    if (lo)
      return k - 1 < -1 ? -1 : k - 1;
    return (nz == 1) ? k : ((k - 1 < 0) ? k + 1 : k - 1);
  }
  __device__ int zup(int k) const {
    if (hi)
      return k + 1 > nz ? nz : k + 1;
    return (nz == 1) ? k : ((k + 1 >= nz) ? k - 1 : k + 1);
  }
};

// Mirrored neighbours (tikhonov.cpp:10-22, total_v.cpp:31-52).  An axis of
// length 1 has no neighbour; the reference then reads index -1 or 1 out of
// bounds, here the voxel itself is used.
__device__ __forceinline__ int mirror_up(int i, int n) {
  return n == 1 ? i : ((i + 1 >= n) ? i - 1 : i + 1);
}
__device__ __forceinline__ int mirror_dn(int i, int n) {
  return n == 1 ? i : ((i - 1 < 0) ? i + 1 : i - 1);
}

// tikhonov.cpp:29-30: 0.25 * (sum of four xy neighbours) - centre.
__device__ float tikhonov_at(const Vol &v, int i, int j, int k) {
  const float s4 = __fadd_rn(__fadd_rn(__fadd_rn(v.at(mirror_up(i, v.nx), j, k),
                                                 v.at(mirror_dn(i, v.nx), j, k)),
                                       v.at(i, mirror_up(j, v.ny), k)),
                             v.at(i, mirror_dn(j, v.ny), k));
  return float(0.25 * double(s4) - double(v.at(i, j, k)));
}

__device__ __forceinline__ int sgn(float x) { return (x > 0.0f) - (x < 0.0f); }

// minmod term of total_v.cpp:62-67 (evaluated in double, stored as float)
__device__ __forceinline__ float minmod(float p, float m) {
  const float mn = (fabsf(m) < fabsf(p)) ? fabsf(m) : fabsf(p);
  return float(0.5 * double(sgn(p) + sgn(m)) * double(mn));
}

// One of the normalised forward differences D1, D2, D3 at (i, j, k)
// (D_func, total_v.cpp:77-146; D1_func is the same D1).
__device__ float tv_d(const Vol &v, int i, int j, int k, int which) {
  const float c = v.at(i, j, k);
  const float x1 = __fsub_rn(v.at(mirror_up(i, v.nx), j, k), c);
  const float y1 = __fsub_rn(v.at(i, mirror_up(j, v.ny), k), c);
  const float y0 = __fsub_rn(c, v.at(i, mirror_dn(j, v.ny), k));
  const float x0 = __fsub_rn(c, v.at(mirror_dn(i, v.nx), j, k));
  const float z1 = __fsub_rn(v.at(i, j, v.zup(k)), c);
  const float z0 = __fsub_rn(c, v.at(i, j, v.zdn(k)));
  float d2x = minmod(y1, y0);
  float d2y = minmod(x1, x0);
  float d3x = minmod(z1, z0);
  d2x = __fmul_rn(d2x, d2x);
  d2y = __fmul_rn(d2y, d2y);
  d3x = __fmul_rn(d3x, d3x);
  const float eps = FLT_EPSILON;
  if (which == 0) {
    const float t = __fsqrt_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(x1, x1), d2x), d3x), eps));
    return __fdiv_rn(x1, t);
  } else if (which == 1) {
    const float t = __fsqrt_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(y1, y1), d2y), d3x), eps));
    return __fdiv_rn(y1, t);
  }
  const float t = __fsqrt_rn(__fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(z1, z1), d2y), d2x), eps));
  return __fdiv_rn(z1, t);
}

// TV_main (total_v.cpp:149-195): backward-difference divergence.
__device__ float tv_at(const Vol &v, int i, int j, int k) {
  const float dv1 = __fsub_rn(tv_d(v, i, j, k, 0), tv_d(v, mirror_dn(i, v.nx), j, k, 0));
  const float dv2 = __fsub_rn(tv_d(v, i, j, k, 1), tv_d(v, i, mirror_dn(j, v.ny), k, 1));
  const float dv3 = __fsub_rn(tv_d(v, i, j, k, 2), tv_d(v, i, j, v.zdn(k), 2));
  return __fadd_rn(__fadd_rn(dv1, dv2), dv3);
}

template <int ALG> __device__ __forceinline__ float reg_at(const Vol &v, int i, int j, int k) {
  return ALG == 3 ? tikhonov_at(v, i, j, k) : tv_at(v, i, j, k);
}

template <int ALG>
__global__ void reg_accumulate_kernel(Vol v, float *acc, float lambda, double *partials) {
  __shared__ double red[kThreads / 32];
  const i64 n = i64(v.nx) * v.ny * v.nz;
  double t = 0.0;
  for (i64 idx = blockIdx.x * i64(blockDim.x) + threadIdx.x; idx < n;
       idx += i64(gridDim.x) * blockDim.x) {
    const int k = int(idx % v.nz);
    const i64 ij = idx / v.nz;
    const int j = int(ij % v.ny), i = int(ij / v.ny);
    const float o = __fadd_rn(acc[idx], __fmul_rn(lambda, reg_at<ALG>(v, i, j, k)));
    acc[idx] = o;
    t += double(o) * double(o);
  }
  t = cta_sum<kThreads / 32>(t, red);
  if (threadIdx.x == 0)
    partials[blockIdx.x] = t;
}

template <int ALG>
__global__ void reg_step_kernel(Vol v, float *out, float lambda) {
  const i64 n = i64(v.nx) * v.ny * v.nz;
  for (i64 idx = blockIdx.x * i64(blockDim.x) + threadIdx.x; idx < n;
       idx += i64(gridDim.x) * blockDim.x) {
    const int k = int(idx % v.nz);
    const i64 ij = idx / v.nz;
    const int j = int(ij % v.ny), i = int(ij / v.ny);
    out[idx] = __fadd_rn(v.a[idx], __fmul_rn(lambda, reg_at<ALG>(v, i, j, k)));
  }
}

template <int ALG> __global__ void reg_apply_kernel(Vol v, float *out) {
  const i64 n = i64(v.nx) * v.ny * v.nz;
  for (i64 idx = blockIdx.x * i64(blockDim.x) + threadIdx.x; idx < n;
       idx += i64(gridDim.x) * blockDim.x) {
    const int k = int(idx % v.nz);
    const i64 ij = idx / v.nz;
    const int j = int(ij % v.ny), i = int(ij / v.ny);
    out[idx] = reg_at<ALG>(v, i, j, k);
  }
}

// ------------------------------------------------------------- layouts
__global__ void pack_parallel_kernel(const float *__restrict__ in, float *__restrict__ out, int na,
                                     int nv, int nh, int nv_pad, int voff) {
  const i64 n = i64(na) * nh * nv_pad;
  for (i64 idx = blockIdx.x * i64(blockDim.x) + threadIdx.x; idx < n;
       idx += i64(gridDim.x) * blockDim.x) {
    const int v = int(idx % nv_pad);
    const i64 ah = idx / nv_pad;
    const int h = int(ah % nh), a = int(ah / nh);
    const int vs = v - voff;
    out[idx] = (vs >= 0 && vs < nv) ? in[(i64(a) * nv + vs) * nh + h] : 0.0f;
  }
}

__global__ void pack_cone_kernel(const float *__restrict__ in, float *__restrict__ out, int na,
                                 int nh, int nv, int nv_pad, int voff) {
  const i64 n = i64(na) * nh * nv_pad;
  for (i64 idx = blockIdx.x * i64(blockDim.x) + threadIdx.x; idx < n;
       idx += i64(gridDim.x) * blockDim.x) {
    const int v = int(idx % nv_pad);
    const i64 ah = idx / nv_pad;
    const int vs = v - voff;
    out[idx] = (vs >= 0 && vs < nv) ? in[ah * nv + vs] : 0.0f;
  }
}

__global__ void unpack_parallel_kernel(const float *__restrict__ in, float *__restrict__ out,
                                       int na, int nh, int nv) {
  const i64 n = i64(na) * nh * nv;
  for (i64 idx = blockIdx.x * i64(blockDim.x) + threadIdx.x; idx < n;
       idx += i64(gridDim.x) * blockDim.x) {
    const int h = int(idx % nh);
    const i64 av = idx / nh;
    const int v = int(av % nv), a = int(av / nv);
    out[idx] = in[(i64(a) * nh + h) * nv + v];
  }
}

int grid_for(i64 n) {
  const i64 g = (n + kThreads - 1) / kThreads;
  return int(g < kGrid ? (g < 1 ? 1 : g) : kGrid);
}

} // namespace

void k_fill(float *p, i64 n, float v, cudaStream_t st) {
  fill_kernel<<<grid_for(n), kThreads, 0, st>>>(p, n, v);
}
void k_invert_pos(float *p, i64 n, cudaStream_t st) {
  invert_pos_kernel<<<grid_for(n), kThreads, 0, st>>>(p, n);
}
void k_invert_nonzero(float *p, i64 n, cudaStream_t st) {
  invert_nonzero_kernel<<<grid_for(n), kThreads, 0, st>>>(p, n);
}
void k_clamp0(float *p, i64 n, cudaStream_t st) {
  clamp0_kernel<<<grid_for(n), kThreads, 0, st>>>(p, n);
}
int sumsq_blocks() { return kGrid; }
void k_sumsq_partials(const float *x, i64 n, double *partials, int nblocks, cudaStream_t st) {
  sumsq_kernel<<<nblocks, kThreads, 0, st>>>(x, n, partials);
}
void k_cgls_scalars(int op, const double *p1, int n1, const double *p2, int n2, double *s,
                    double *norms, cudaStream_t st) {
  cgls_scalars_kernel<<<1, kThreads, 0, st>>>(op, p1, n1, p2, n2, s, norms);
}
void k_axpy_scalar(float *y, const float *x, i64 n, const double *s, int idx, float sign,
                   cudaStream_t st) {
  axpy_scalar_kernel<<<grid_for(n), kThreads, 0, st>>>(y, x, n, s, idx, sign);
}
void k_cgls_xd(float *x, float *d, const float *sv, i64 n, const double *s, cudaStream_t st) {
  cgls_xd_kernel<<<grid_for(n), kThreads, 0, st>>>(x, d, sv, n, s);
}
void k_cgls_d(float *d, const float *sv, i64 n, const double *s, cudaStream_t st) {
  cgls_d_kernel<<<grid_for(n), kThreads, 0, st>>>(d, sv, n, s);
}
void k_add_scaled(float *out, const float *in, const float *d, i64 n, const double *s,
                  cudaStream_t st) {
  add_scaled_kernel<<<grid_for(n), kThreads, 0, st>>>(out, in, d, n, s);
}
void k_shard_scalars(int op, const double *p1, int n1, const double *p2, int n2, double *sum,
                     double *s, double *norms, cudaStream_t st) {
  shard_scalars_kernel<<<1, kThreads, 0, st>>>(op, p1, n1, p2, n2, sum, s, norms);
}
void k_pack_edges(const float *a, int nx, int ny, int nz, float *lo, float *hi, cudaStream_t st) {
  const int nxy = nx * ny;
  pack_edges_kernel<<<grid_for(nxy), kThreads, 0, st>>>(a, nxy, nz, lo, hi);
}
void k_reg_accumulate(int alg, const float *a, float *acc, int nx, int ny, int nz, float lambda,
                      double *partials, int nblocks, cudaStream_t st, const float *lo,
                      const float *hi) {
  Vol v{a, nx, ny, nz, lo, hi};
  if (alg == 3)
    reg_accumulate_kernel<3><<<nblocks, kThreads, 0, st>>>(v, acc, lambda, partials);
  else
    reg_accumulate_kernel<4><<<nblocks, kThreads, 0, st>>>(v, acc, lambda, partials);
}
void k_reg_step(int alg, const float *a, float *out, int nx, int ny, int nz, float lambda,
                cudaStream_t st, const float *lo, const float *hi) {
  Vol v{a, nx, ny, nz, lo, hi};
  const i64 n = i64(nx) * ny * nz;
  if (alg == 3)
    reg_step_kernel<3><<<grid_for(n), kThreads, 0, st>>>(v, out, lambda);
  else
    reg_step_kernel<4><<<grid_for(n), kThreads, 0, st>>>(v, out, lambda);
}
void k_reg_apply(int alg, const float *a, float *out, int nx, int ny, int nz, cudaStream_t st) {
  Vol v{a, nx, ny, nz};
  const i64 n = i64(nx) * ny * nz;
  if (alg == 3)
    reg_apply_kernel<3><<<grid_for(n), kThreads, 0, st>>>(v, out);
  else
    reg_apply_kernel<4><<<grid_for(n), kThreads, 0, st>>>(v, out);
}
void k_pack_parallel(const float *in, float *out, int na, int nv, int nh, int nv_pad, int voff,
                     cudaStream_t st) {
  pack_parallel_kernel<<<grid_for(i64(na) * nh * nv_pad), kThreads, 0, st>>>(in, out, na, nv, nh,
                                                                             nv_pad, voff);
}
void k_pack_cone(const float *in, float *out, int na, int nh, int nv, int nv_pad, int voff,
                 cudaStream_t st) {
  pack_cone_kernel<<<grid_for(i64(na) * nh * nv_pad), kThreads, 0, st>>>(in, out, na, nh, nv,
                                                                         nv_pad, voff);
}
void k_unpack_parallel(const float *in, float *out, int na, int nh, int nv, cudaStream_t st) {
  unpack_parallel_kernel<<<grid_for(i64(na) * nh * nv), kThreads, 0, st>>>(in, out, na, nh, nv);
}

} // namespace ccpi
