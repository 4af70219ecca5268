// Cone-beam projectors for sm_100a.
//
// Forward (cone_beam::f2D, Core/src/c2D.cpp:469-625): ray-driven.  One warp
// owns one ray (angle a, detector column h).  The warp walks the ray's xy
// Siddon path once in voxel-normalised coordinates (c2D.cpp:193-467, FP64
// geometry, alphas rounded to float exactly as the reference stores them)
// and stages the (alpha, column) list in its own slice of shared memory.
// The lanes then own detector rows v and replay the list: each xy segment is
// split across at most two z slices with the reference's float arithmetic
// and its three row regimes (all-inside, lower edge, upper edge;
// c2D.cpp:17-191), and the row is finally scaled by the source-pixel
// distance.  Per row the additions happen in the reference's order with
// unfused float operations, so the result matches the reference bit for bit.
//
// Backward (cone_beam::b2D, c2D.cpp:948-1119): voxel-column gather, the
// reference's design.  One CTA owns one xy column; it finds, angle chunk by
// angle chunk, every (angle, detector column) ray that crosses the column
// with the reference's entry/exit alphas (c2D.cpp:788-946).  cb_bp_gather
// then has each thread form its own voxels' sums over the rays' detector
// rows (c2D.cpp:640-751) in the reference's order, bit for bit; columns
// taller than 1024 voxels use cb_bp_kernel, whose warps spread rows into a
// shared-memory accumulator with float atomics (unspecified order, equal to
// the reference to float rounding).
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace ccpi {
namespace {

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }
// std::min(a, b) as the reference evaluates it: (b < a) ? b : a.  Every
// call passes b = a ray's exit alpha, which is never NaN and never -0, and
// for such b the NaN-propagating hardware minimum returns the same value for
// every a (NaN a gives NaN, +-0 a with b > 0 gives a), in one instruction
// instead of a compare and a select.
#ifndef CB_FMIN_NAN
#define CB_FMIN_NAN 1
#endif
__device__ __forceinline__ float fmin_ref(float a, float b) {
#if CB_FMIN_NAN
  float r;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
#else
  return (b < a) ? b : a;
#endif
}

// xy walk of ray p1 -> p2 over the whole volume; writes alphas[0..n-1] and
// cells[0..n-2] (x*ny + y, or -1) with lane 0; returns n (0 if missed).
__device__ int cb_walk(const Geom &g, double p1x, double p1y, double p2x, double p2y,
                       float *alphas, int *cells, int cap) {
  const double eps = double(kEps);
  const int nx = g.nx, ny = g.ny;
  const bool w = (threadIdx.x & 31) == 0;
  const double q1x = (p1x - g.origin[0]) / g.size[0];
  const double q1y = (p1y - g.origin[1]) / g.size[1];
  const double q2x = (p2x - g.origin[0]) / g.size[0];
  const double q2y = (p2y - g.origin[1]) / g.size[1];
  const double ddx = q2x - q1x, ddy = q2y - q1y;
  const double idx = 1.0 / ddx, idy = 1.0 / ddy;
  int n = 0;
  if (fabs(ddx) < eps) {
    if (fabs(ddy) < eps)
      return 0;
    const int i = int(floor(q1x));
    if (i < 0 || i >= nx)
      return 0;
    if (ddy < 0.0) {
      if (w)
        alphas[0] = float((double(ny) - q1y) * idy);
      for (int j = ny - 1; j >= 0; j--) {
        if (w) {
          alphas[ny - j] = float((double(j) - q1y) * idy);
          cells[ny - 1 - j] = i * ny + j;
        }
      }
    } else {
      if (w)
        alphas[0] = float((0.0 - q1y) * idy);
      for (int j = 0; j < ny; j++) {
        if (w) {
          alphas[j + 1] = float((double(j + 1) - q1y) * idy);
          cells[j] = i * ny + j;
        }
      }
    }
    return ny + 1;
  }
  if (fabs(ddy) < eps) {
    const int j = int(floor(q1y));
    if (j < 0 || j >= ny)
      return 0;
    if (ddx < 0.0) {
      if (w)
        alphas[0] = float((double(nx) - q1x) * idx);
      for (int i = nx - 1; i >= 0; i--) {
        if (w) {
          alphas[nx - i] = float((double(i) - q1x) * idx);
          cells[nx - 1 - i] = i * ny + j;
        }
      }
    } else {
      if (w)
        alphas[0] = float((0.0 - q1x) * idx);
      for (int i = 0; i < nx; i++) {
        if (w) {
          alphas[i + 1] = float((double(i + 1) - q1x) * idx);
          cells[i] = i * ny + j;
        }
      }
    }
    return nx + 1;
  }
  const double ax0 = (0.0 - q1x) * idx, ay0 = (0.0 - q1y) * idy;
  const double axn = (double(nx) - q1x) * idx, ayn = (double(ny) - q1y) * idy;
  const double amin = dmax(dmax(dmin(ax0, axn), dmin(ay0, ayn)), 0.0);
  const double amax = dmin(dmin(dmax(ax0, axn), dmax(ay0, ayn)), 1.0);
  if (!(amin < amax - eps))
    return 0;
  const int sx = ddx > 0.0 ? 1 : -1, sy = ddy > 0.0 ? 1 : -1;
  int x = 0, y = 0;
  const bool x_face_first = !(sx > 0 && sy < 0);
  const double axe = sx > 0 ? ax0 : axn, aye = sy > 0 ? ay0 : ayn;
  auto cx = [&]() { return int(floor(q1x + amin * ddx)); };
  auto cy = [&]() { return int(floor(q1y + amin * ddy)); };
  if (x_face_first) {
    if (amin == axe) {
      x = sx > 0 ? 0 : nx - 1;
      y = (sx < 0 && sy < 0 && amin == ayn) ? ny - 1 : cy();
    } else if (amin == aye) {
      x = cx();
      y = sy > 0 ? 0 : ny - 1;
    }
  } else {
    if (amin == aye) {
      x = cx();
      y = ny - 1;
    } else if (amin == axe) {
      x = 0;
      y = cy();
    }
  }
  if (w)
    alphas[0] = float(amin);
  n = 1;
  while ((sx > 0 ? x < nx : x >= 0) && (sy > 0 ? y < ny : y >= 0) && n < cap) {
    const double nxa = (double(sx > 0 ? x + 1 : x) - q1x) * idx;
    const double nya = (double(sy > 0 ? y + 1 : y) - q1y) * idy;
    const int cell = (x >= 0 && x < nx && y >= 0 && y < ny) ? x * ny + y : -1;
    double an;
    if (nxa < nya - eps) {
      an = nxa;
      x += sx;
    } else if (nya < nxa - eps) {
      an = nya;
      y += sy;
    } else {
      an = dmax(nxa, nya);
      x += sx;
      y += sy;
    }
    if (w) {
      cells[n - 1] = cell;
      alphas[n] = float(an);
    }
    n++;
  }
  return n;
}

template <int EPI>
__device__ __forceinline__ float cb_fp_epi(float acc, i64 idx, const Epi &e, double &ssq) {
  if (EPI == EPI_NORM) {
    ssq += double(acc) * double(acc);
    return acc;
  } else if (EPI == EPI_SIRT) {
    return __fmul_rn(__fadd_rn(-acc, e.b[idx]), e.w[idx]);
  } else if (EPI == EPI_MLEM) {
    const float q = (acc != 0.0f) ? __fdiv_rn(e.b[idx], acc) : 0.0f;
    return (q < 0.0f) ? 0.0f : q;
  }
  return acc;
}

constexpr int kFpWarps = 4;
#ifndef CB_FP_PACKED
#define CB_FP_PACKED 1
#endif

// Floats of the slice-plane table copy at the start of the forward
// projector's shared memory (nz + 1 entries, rounded up to 4).
__host__ __device__ inline int cb_vz_floats(int nz) { return (nz + 1 + 3) & ~3; }

// Row regimes of a walked ray (c2D.cpp:45-99), evaluated warp-parallel:
// cells [1, ncom) have every row's slice and its neighbour inside the
// column; rows [min_v_all, max_v_all] stay inside it for every cell.
__device__ __forceinline__ void cb_row_regimes(const Geom &g, const float *alphas, int n,
                                               int lane, int &ncom, int &min_v_all,
                                               int &max_v_all) {
  const int nzm1 = g.nz - 1, mid = g.mid;
  const float pzbz = g.pzbz, inv_dz = g.inv_dz;
  ncom = 0;
  min_v_all = mid;
  max_v_all = mid - 1;
  if (n < 2)
    return;
  int min_xy_all = n, max_xy_all = n;
  const float dz0 = g.dz[0], dzl = g.dz[g.nv - 1];
  bool got_lo = false, got_hi = false;
  for (int m0 = 1; m0 < n && !(got_lo && got_hi); m0 += 32) {
    const int m = m0 + lane;
    int klo = 1, khi = nzm1 - 1;
    if (m < n) {
      const float av = __fmul_rn(alphas[m - 1], inv_dz);
      klo = int(floorf(__fadd_rn(pzbz, __fmul_rn(av, dz0))));
      khi = int(floorf(__fadd_rn(pzbz, __fmul_rn(av, dzl))));
    }
    if (!got_lo) {
      const unsigned b = __ballot_sync(0xffffffffu, m < n && klo <= 0);
      if (b) {
        const int src = __ffs(b) - 1;
        const int k = __shfl_sync(0xffffffffu, klo, src);
        min_xy_all = (k == 0) ? m0 + src : 0;
        got_lo = true;
      }
    }
    if (!got_hi) {
      const unsigned b = __ballot_sync(0xffffffffu, m < n && khi >= nzm1);
      if (b) {
        const int src = __ffs(b) - 1;
        const int k = __shfl_sync(0xffffffffu, khi, src);
        max_xy_all = (k == nzm1) ? m0 + src : 0;
        got_hi = true;
      }
    }
  }
  ncom = min(min_xy_all, max_xy_all);
  const float avl = __fmul_rn(alphas[n - 2], inv_dz);
  for (int v0 = 0; v0 < mid; v0 += 32) {
    const int v = v0 + lane;
    const bool ok = v < mid && int(floorf(__fadd_rn(pzbz, __fmul_rn(avl, g.dz[v])))) > 0;
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (b) {
      min_v_all = v0 + __ffs(b) - 1;
      break;
    }
  }
  for (int v1 = g.nv - 1; v1 >= mid; v1 -= 32) {
    const int v = v1 - lane;
    const bool ok = v >= mid && int(floorf(__fadd_rn(pzbz, __fmul_rn(avl, g.dz[v])))) < nzm1;
    const unsigned b = __ballot_sync(0xffffffffu, ok);
    if (b) {
      max_v_all = v1 - (__ffs(b) - 1);
      break;
    }
  }
}

// RPL = detector rows per lane per pass (a pass covers 32 * RPL rows);
// FULL: nv is a multiple of 32 * RPL (no idle rows).  BATCH: nb volumes
// (one after another) share each ray's walk and row regimes (EPI_STORE
// only).  Without it the item loop runs once and compiles away: a run-time
// loop costs the single-volume form 10 % at 512^3.
template <int EPI, int RPL, bool FULL, bool BATCH>
__global__ void __launch_bounds__(kFpWarps * 32)
    cb_fp_kernel(Geom g, const float *__restrict__ vol0, float *__restrict__ pix0, Epi e,
                 const int2 *__restrict__ hrange, int cap, int nb) {
  extern __shared__ unsigned char smem_raw[];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *svz = reinterpret_cast<float *>(smem_raw);
  float *alphas = svz + cb_vz_floats(g.nz) + size_t(wib) * 2 * cap;
  int *cells = reinterpret_cast<int *>(alphas + cap);
  for (int i = threadIdx.x; i <= g.nz; i += blockDim.x)
    svz[i] = g.vz[i];
  __syncthreads();
  const int nrays = g.na * g.nh;
  const int nzm1 = g.nz - 1, mid = g.mid;
  const float pzbz = g.pzbz, pzbz1 = g.pzbz1, inv_dz = g.inv_dz;
  double ssq = 0.0;
  for (int ray = blockIdx.x * kFpWarps + wib; ray < nrays; ray += gridDim.x * kFpWarps) {
    const int a = ray / g.nh, h = ray - a * g.nh;
    const int2 hr = hrange[a];
    int n = 0;
    if (h >= hr.x && h <= hr.y) {
      const double c = g.cosA[a], s = g.sinA[a];
      const double p2x = c * g.detx - s * g.hpix[h];
      const double p2y = s * g.detx + c * g.hpix[h];
      n = cb_walk(g, g.p1x[a], g.p1y[a], p2x, p2y, alphas, cells, cap);
    }
    __syncwarp();
    int ncom, min_v_all, max_v_all;
    cb_row_regimes(g, alphas, n, lane, ncom, min_v_all, max_v_all);
    // Rows, RPL per lane per pass.  Cells [1, mfast) have every row inside
    // the slab (c2D.cpp:99-145); the rest take the edge rules (:146-190).
    const int mfast = min(ncom, n);
    for (int b = 0; b < (BATCH ? nb : 1); b++) {
    // batch item b: its volume and its sinogram
    const float *__restrict__ vol = vol0 + i64(b) * g.nx * g.ny * g.nz;
    float *__restrict__ pix = pix0 + i64(b) * g.na * g.nh * g.nv;
    for (int vb = 0; vb < g.nv; vb += 32 * RPL) {
      float acc[RPL], dzv[RPL], izv[RPL];
      bool vok[RPL], below[RPL];
#pragma unroll
      for (int q = 0; q < RPL; q++) {
        const int v = vb + q * 32 + lane;
        acc[q] = 0.0f;
        vok[q] = v < g.nv;
        below[q] = v < mid;
        dzv[q] = vok[q] ? g.dz[v] : 0.0f;
        izv[q] = vok[q] ? g.iz[v] : 0.0f;
      }
      // In [1, mfast) the regime search has shown that the lowest row's
      // slice index is >= 1 and the highest row's < nz - 1 (c2D.cpp:45-99),
      // so every row's k and its neighbour k -/+ 1 are inside the column.
      int dk[RPL];
      const float *vzq[RPL];
#pragma unroll
      for (int q = 0; q < RPL; q++) {
        dk[q] = below[q] ? -1 : 1;
        vzq[q] = svz + (below[q] ? 0 : 1);
      }
#if CB_FP_PACKED
      if (FULL) {
        // rows q and q + 1 as packed pairs: per row the same unfused float
        // operations as below, two rows per multiply and subtract
        // instruction; the products only feed scalar adds
        float2 acc2[RPL / 2], dz2[RPL / 2], iz2[RPL / 2];
#pragma unroll
        for (int q = 0; q < RPL; q += 2) {
          acc2[q / 2] = make_float2(0.0f, 0.0f);
          dz2[q / 2] = make_float2(dzv[q], dzv[q + 1]);
          iz2[q / 2] = make_float2(izv[q], izv[q + 1]);
        }
        for (int m = 1; m < mfast; m++) {
          const float a0 = alphas[m - 1], a1 = alphas[m];
          const int cell = cells[m - 1];
          if (cell < 0)
            continue;
          const float *col = vol + i64(cell) * g.nz;
          const float av = __fmul_rn(a0, inv_dz);
          const float2 av2 = make_float2(av, av), a02 = make_float2(a0, a0),
                       a12 = make_float2(a1, a1);
#pragma unroll
          for (int q = 0; q < RPL; q += 2) {
            const float2 kz = mul2_rn(av2, dz2[q / 2]);
            const int k0 = int(__fadd_rn(pzbz, kz.x)), k1 = int(__fadd_rn(pzbz, kz.y));
            const float2 pl = mul2_rn(make_float2(vzq[q][k0], vzq[q + 1][k1]), iz2[q / 2]);
            const float2 mz = make_float2(fmin_ref(pl.x, a1), fmin_ref(pl.y, a1));
            const float2 lo = sub2_rn(mz, a02), hi = sub2_rn(a12, mz);
            const float2 pk = mul2_rn(make_float2(__ldg(col + k0), __ldg(col + k1)), lo);
            const float2 pn =
                mul2_rn(make_float2(__ldg(col + k0 + dk[q]), __ldg(col + k1 + dk[q + 1])), hi);
            acc2[q / 2] = add2_rn(acc2[q / 2],
                                  make_float2(__fadd_rn(pk.x, pn.x), __fadd_rn(pk.y, pn.y)));
          }
        }
#pragma unroll
        for (int q = 0; q < RPL; q += 2) {
          acc[q] = acc2[q / 2].x;
          acc[q + 1] = acc2[q / 2].y;
        }
      } else
#endif
      for (int m = 1; m < mfast; m++) {
        const float a0 = alphas[m - 1], a1 = alphas[m];
        const int cell = cells[m - 1];
        if (cell < 0)
          continue;
        const float *col = vol + i64(cell) * g.nz;
        const float av = __fmul_rn(a0, inv_dz);
#pragma unroll
        for (int q = 0; q < RPL; q++) {
          if (!FULL && !vok[q])
            continue;
          const int k = int(__fadd_rn(pzbz, __fmul_rn(av, dzv[q])));
          const float *ck = col + k;
          const float mz = fmin_ref(__fmul_rn(vzq[q][k], izv[q]), a1);
          acc[q] = __fadd_rn(acc[q], __fadd_rn(__fmul_rn(__ldg(ck), __fsub_rn(mz, a0)),
                                               __fmul_rn(__ldg(ck + dk[q]), __fsub_rn(a1, mz))));
        }
      }
      for (int m = max(mfast, 1); m < n; m++) {
        const float a0 = alphas[m - 1], a1 = alphas[m];
        const int cell = cells[m - 1];
        if (cell < 0)
          continue;
        const float *col = vol + i64(cell) * g.nz;
        const float av = __fmul_rn(a0, inv_dz);
#pragma unroll
        for (int q = 0; q < RPL; q++) {
          const int v = vb + q * 32 + lane;
          if (!vok[q])
            continue;
          if (v >= min_v_all && v <= max_v_all) {
            const int k = int(__fadd_rn(pzbz, __fmul_rn(av, dzv[q])));
            const int kn = below[q] ? k - 1 : k + 1;
            if (unsigned(k) > unsigned(nzm1) || unsigned(kn) > unsigned(nzm1))
              continue;
            const float mz = fmin_ref(__fmul_rn(svz[below[q] ? k : k + 1], izv[q]), a1);
            acc[q] = __fadd_rn(acc[q], __fadd_rn(__fmul_rn(__ldg(col + k), __fsub_rn(mz, a0)),
                                                 __fmul_rn(__ldg(col + kn), __fsub_rn(a1, mz))));
          } else if (ncom >= 1) {
            if (v < min_v_all) {
              const int k = int(__fadd_rn(pzbz1, __fmul_rn(av, dzv[q]))) - 1;
              if (k > 0 && k <= nzm1) {
                const float mz = fmin_ref(__fmul_rn(svz[k], izv[q]), a1);
                acc[q] = __fadd_rn(acc[q],
                                   __fadd_rn(__fmul_rn(__ldg(col + k), __fsub_rn(mz, a0)),
                                             __fmul_rn(__ldg(col + k - 1), __fsub_rn(a1, mz))));
              } else if (k == 0) {
                const float mz = fmin_ref(__fmul_rn(svz[0], izv[q]), a1);
                acc[q] = __fadd_rn(acc[q], __fmul_rn(__ldg(col), __fsub_rn(mz, a0)));
              }
            } else {
              const int k = int(__fadd_rn(pzbz, __fmul_rn(av, dzv[q])));
              if (k < nzm1 && k >= 0) {
                const float mz = fmin_ref(__fmul_rn(svz[k + 1], izv[q]), a1);
                acc[q] = __fadd_rn(acc[q],
                                   __fadd_rn(__fmul_rn(__ldg(col + k), __fsub_rn(mz, a0)),
                                             __fmul_rn(__ldg(col + k + 1), __fsub_rn(a1, mz))));
              } else if (k == nzm1) {
                const float mz = fmin_ref(__fmul_rn(svz[g.nz], izv[q]), a1);
                acc[q] = __fadd_rn(acc[q], __fmul_rn(__ldg(col + nzm1), __fsub_rn(mz, a0)));
              }
            }
          }
        }
      }
      const i64 rbase = i64(ray) * g.nv;
#pragma unroll
      for (int q = 0; q < RPL; q++) {
        const int v = vb + q * 32 + lane;
        if (v < g.nv) {
          const float dcv = g.dconv[i64(h) * g.nv + v];
          const float out = cb_fp_epi<EPI>(__fmul_rn(acc[q], dcv), rbase + v, e, ssq);
          // the SIRT / MLEM residual is the back projector's input: with
          // e.pre it is stored times d_conv (the reference's dpixels)
          pix[rbase + v] = ((EPI == EPI_SIRT || EPI == EPI_MLEM) && e.pre) ? __fmul_rn(out, dcv) : out;
        }
      }
    }
    } // batch items
    __syncwarp();
  }
  if (EPI == EPI_NORM) {
    __shared__ double red[kFpWarps];
    const double t = cta_sum<kFpWarps>(ssq, red);
    if (threadIdx.x == 0)
      e.partials[blockIdx.x] = t;
  }
}

// ---- backward, ray-driven scatter (the transpose of cb_fp_kernel)
//
// One warp per ray (angle a, detector column h), as in the forward
// projector, with the same walk.  The reference's back projector is not the
// exact transpose of its forward projector: it drops rays parallel to an
// axis and picks each row's slice rule from a band kept per voxel column
// (c2D.cpp:657-750), where the forward projector keeps one per ray.  So
// per (cell, row) this kernel takes the back projector's rule, from the
// plan's column band table: slice k, neighbour and weights (mz - a0,
// a1 - mz), and the row's value p = pix * d_conv times each weight goes to
// the two voxels.  Each lane holds RPL consecutive rows of a pass
// (v = vb + lane * RPL + j).  The slice index is monotone in the row, so a
// slice's rows mostly sit in one lane: the lane sums a run of rows with the
// same slice and side in registers, in row order, and adds the run's two
// sums (to the slice and to its neighbour) with float atomics when the
// slice changes and at the end of the pass.  The order of the additions
// into a voxel is not fixed: the result equals the reference's b2D to float
// rounding, not bit for bit (cb_bp_gather is that form).  `vol` must be
// zero on entry; PRE: `pix` is already scaled by d_conv.
//
// (A form with lanes on rows 32 apart and a warp segmented reduction per
// target was measured slower on every geometry: 1250 against 1012 ms at
// 512^3, 69 against 58 ms at 256^3.)
template <int RPL, bool PRE>
__global__ void __launch_bounds__(kFpWarps * 32, 8)
    cb_bp_scatter(Geom g, const float *__restrict__ pix, float *__restrict__ vol,
               const int2 *__restrict__ hrange, int cap) {
  extern __shared__ unsigned char smem_raw[];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float *svz = reinterpret_cast<float *>(smem_raw);
  float *alphas = svz + cb_vz_floats(g.nz) + size_t(wib) * 2 * cap;
  int *cells = reinterpret_cast<int *>(alphas + cap);
  for (int i = threadIdx.x; i <= g.nz; i += blockDim.x)
    svz[i] = g.vz[i];
  __syncthreads();
  const int nrays = g.na * g.nh;
  const int nz = g.nz, nzm1 = g.nz - 1, mid = g.mid;
  const float pzbz = g.pzbz, pzbz1 = g.pzbz1, inv_dz = g.inv_dz;
  for (int ray = blockIdx.x * kFpWarps + wib; ray < nrays; ray += gridDim.x * kFpWarps) {
    const int a = ray / g.nh, h = ray - a * g.nh;
    const int2 hr = hrange[a];
    int n = 0;
    if (h >= hr.x && h <= hr.y) {
      const double c = g.cosA[a], s = g.sinA[a];
      // the back projector takes no ray parallel to an axis
      // (c2D.cpp:909-912), with its own differences
      const double bdx = (g.cdx[a] - s * g.hpix[h]) - g.p1x[a];
      const double bdy = (g.sdx[a] + c * g.hpix[h]) - g.p1y[a];
      if (fabs(bdx) >= double(kEps) && fabs(bdy) >= double(kEps)) {
        const double p2x = c * g.detx - s * g.hpix[h];
        const double p2y = s * g.detx + c * g.hpix[h];
        n = cb_walk(g, g.p1x[a], g.p1y[a], p2x, p2y, alphas, cells, cap);
      }
    }
    __syncwarp();
    const i64 rbase = i64(ray) * g.nv;
    for (int vb = 0; n >= 2 && vb < g.nv; vb += 32 * RPL) {
      float p[RPL], dzv[RPL], izv[RPL];
      bool vok[RPL], below[RPL];
      // per row, fixed by its side of the source: the neighbour's step, the
      // slice plane the weights use (k or k + 1) and the lowest slice whose
      // neighbour stays inside the column
      int dk[RPL], off[RPL], klo[RPL];
#pragma unroll
      for (int j = 0; j < RPL; j++) {
        const int v = vb + lane * RPL + j;
        vok[j] = v < g.nv;
        below[j] = v < mid;
        dk[j] = below[j] ? -1 : 1;
        off[j] = below[j] ? 0 : 1;
        klo[j] = below[j] ? 1 : 0;
        dzv[j] = vok[j] ? g.dz[v] : 0.0f;
        izv[j] = vok[j] ? g.iz[v] : 0.0f;
        const float y = vok[j] ? __ldg(pix + rbase + v) : 0.0f;
        p[j] = (PRE || !vok[j]) ? y : __fmul_rn(y, g.dconv[i64(h) * g.nv + v]);
      }
      // the crossed column's band, loaded one cell ahead
      int2 band_next = cells[0] >= 0 ? g.colband[cells[0]] : make_int2(0, 0);
      for (int m = 1; m < n; m++) {
        const int cell = cells[m - 1];
        const int2 band = band_next;
        if (m + 1 < n && cells[m] >= 0)
          band_next = g.colband[cells[m]];
        if (cell < 0)
          continue;
        const float a0 = alphas[m - 1], a1 = alphas[m];
        const float av = __fmul_rn(a0, inv_dz);
        float *col = vol + i64(cell) * nz;
        int ck = -1, ckn = -1, ckey = -1; // the lane's current run
        float r1 = 0.0f, r2 = 0.0f;
        // one row's run logic: a run of rows with the same slice and side
        // sums its two products in registers; when the slice changes the
        // run's two sums go to its slice and neighbour
        auto run = [&](int k, int kn, bool up, float s1, float s2) {
          const int key = k >= 0 ? 2 * k + (up ? 1 : 0) : -1;
          if (key != ckey) {
            if (ck >= 0) {
              atomicAdd(col + ck, r1);
              if (ckn >= 0)
                atomicAdd(col + ckn, r2);
            }
            ck = k;
            ckn = kn;
            ckey = key;
            r1 = 0.0f;
            r2 = 0.0f;
          }
          if (k >= 0) {
            r1 = __fadd_rn(r1, s1);
            r2 = __fadd_rn(r2, s2);
          }
        };
        if (vb + 32 * RPL <= band.y && vb >= band.x && vb + 32 * RPL <= g.nv) {
          // every row of the pass valid and inside the column's band (the
          // test is the same for the whole warp): the band rule alone, rows
          // j and j + 1 as packed pairs with the same unfused operations
          // per row (a packed product only feeds scalar adds)
#pragma unroll
          for (int j = 0; j + 1 < RPL; j += 2) {
            const float2 kz = mul2_rn(make_float2(av, av), make_float2(dzv[j], dzv[j + 1]));
            const int k0 = int(__fadd_rn(pzbz, kz.x)), k1 = int(__fadd_rn(pzbz, kz.y));
            // k and its neighbour k -/+ 1 inside [0, nz - 1]: one range test
            // (a one-slice column holds no neighbour)
            const bool ok0 = nzm1 > 0 && unsigned(k0 - klo[j]) <= unsigned(nzm1 - 1);
            const bool ok1 = nzm1 > 0 && unsigned(k1 - klo[j + 1]) <= unsigned(nzm1 - 1);
            const float z0 = ok0 ? svz[k0 + off[j]] : 0.0f;
            const float z1 = ok1 ? svz[k1 + off[j + 1]] : 0.0f;
            const float2 pl = mul2_rn(make_float2(z0, z1), make_float2(izv[j], izv[j + 1]));
            const float2 mz = make_float2(fmin_ref(pl.x, a1), fmin_ref(pl.y, a1));
            const float2 w1 = sub2_rn(mz, make_float2(a0, a0));
            const float2 w2 = sub2_rn(make_float2(a1, a1), mz);
            const float2 pp = make_float2(p[j], p[j + 1]);
            const float2 s1 = mul2_rn(pp, w1), s2 = mul2_rn(pp, w2);
            // the pair's runs, with no run state: one pair of atomics when
            // both rows share slice and side (their sums added in row
            // order), else one pair per row
            const bool same = ok0 && ok1 && k0 == k1 && dk[j] == dk[j + 1];
            if (ok0) {
              float *c0 = col + k0;
              atomicAdd(c0, same ? __fadd_rn(s1.x, s1.y) : s1.x);
              atomicAdd(c0 + dk[j], same ? __fadd_rn(s2.x, s2.y) : s2.x);
            }
            if (ok1 && !same) {
              float *c1 = col + k1;
              atomicAdd(c1, s1.y);
              atomicAdd(c1 + dk[j + 1], s2.y);
            }
          }
          if (RPL % 2) {
            constexpr int j = RPL - 1; // the odd row, alone
            const int k0 = int(__fadd_rn(pzbz, __fmul_rn(av, dzv[j])));
            const bool ok0 = nzm1 > 0 && unsigned(k0 - klo[j]) <= unsigned(nzm1 - 1);
            const float z0 = ok0 ? svz[k0 + off[j]] : 0.0f;
            const float mz = fmin_ref(__fmul_rn(z0, izv[j]), a1);
            if (ok0) {
              atomicAdd(col + k0, __fmul_rn(p[j], __fsub_rn(mz, a0)));
              atomicAdd(col + k0 + dk[j], __fmul_rn(p[j], __fsub_rn(a1, mz)));
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < RPL; j++) {
            const int v = vb + lane * RPL + j;
            // the back projector's rule for this row (c2D.cpp:680-750): a
            // band row feeds its slice k and the neighbour on the source's
            // side (k - 1 below the source, k + 1 above), a row below the
            // band k and k - 1, a row above it k and k + 1
            int k = -1, kn = -1;
            bool up = false;
            float w1 = 0.0f, w2 = 0.0f;
            if (vok[j]) {
              if (v >= band.x && v < band.y) {
                const int kk = int(__fadd_rn(pzbz, __fmul_rn(av, dzv[j])));
                const int kkn = below[j] ? kk - 1 : kk + 1;
                if (unsigned(kk) <= unsigned(nzm1) && unsigned(kkn) <= unsigned(nzm1)) {
                  const float mz = fmin_ref(__fmul_rn(svz[below[j] ? kk : kk + 1], izv[j]), a1);
                  k = kk;
                  kn = kkn;
                  up = !below[j];
                  w1 = __fsub_rn(mz, a0);
                  w2 = __fsub_rn(a1, mz);
                }
              } else if (v < band.x) {
                const int kk = int(__fadd_rn(pzbz1, __fmul_rn(av, dzv[j]))) - 1;
                if (kk > 0 && kk <= nzm1) {
                  const float mz = fmin_ref(__fmul_rn(svz[kk], izv[j]), a1);
                  k = kk;
                  kn = kk - 1;
                  w1 = __fsub_rn(mz, a0);
                  w2 = __fsub_rn(a1, mz);
                } else if (kk == 0) {
                  k = 0;
                  w1 = __fsub_rn(fmin_ref(__fmul_rn(svz[0], izv[j]), a1), a0);
                }
              } else {
                const int kk = int(__fadd_rn(pzbz, __fmul_rn(av, dzv[j])));
                up = true;
                if (kk < nzm1 && kk >= 0) {
                  const float mz = fmin_ref(__fmul_rn(svz[kk + 1], izv[j]), a1);
                  k = kk;
                  kn = kk + 1;
                  w1 = __fsub_rn(mz, a0);
                  w2 = __fsub_rn(a1, mz);
                } else if (kk == nzm1) {
                  k = nzm1;
                  w1 = __fsub_rn(fmin_ref(__fmul_rn(svz[nz], izv[j]), a1), a0);
                }
              }
            }
            run(k, kn, up, __fmul_rn(p[j], w1), __fmul_rn(p[j], w2));
          }
        }
        if (ck >= 0) {
          atomicAdd(col + ck, r1);
          if (ckn >= 0)
            atomicAdd(col + ckn, r2);
        }
      }
    }
    __syncwarp();
  }
}

// ---- backward
constexpr int kBpThreads = 256;
constexpr int kBpAngleChunk = 64;
constexpr int kBpMaxRaysPerAngle = 24;

// Rays (angle a, columns h) crossing voxel column [x0,xn) x [y0,yn), with
// their entry/exit alphas (bproject_ah, c2D.cpp:831-936).  Calls f(h, a0, a1).
template <class F>
__device__ void cb_column_rays(const Geom &g, int a, double x0, double xn, double y0,
                               double yn, F &&f) {
  const double eps = double(kEps);
  const double c = g.cosA[a], s = g.sinA[a];
  const double p1x = g.p1x[a], p1y = g.p1y[a];
  const double dx0 = x0 - p1x, dy0 = y0 - p1y, dxn = xn - p1x, dyn = yn - p1y;
  const double cx0 = c * x0 - g.src[0], cxn = c * xn - g.src[0];
  const double sy0 = s * y0, syn = s * yn;
  double y00, y01, y10, y11;
  if (fabs(s) > fabs(c)) {
    const double il = g.cl / s;
    y00 = (c - dx0 / (sy0 + cx0)) * il;
    y01 = (c - dx0 / (syn + cx0)) * il;
    y10 = (c - dxn / (sy0 + cxn)) * il;
    y11 = (c - dxn / (syn + cxn)) * il;
  } else {
    const double il = g.cl / c;
    y00 = (-s + dy0 / (cx0 + sy0)) * il;
    y01 = (-s + dyn / (cx0 + syn)) * il;
    y10 = (-s + dy0 / (cxn + sy0)) * il;
    y11 = (-s + dyn / (cxn + syn)) * il;
  }
  const int h00 = int(floor(y00 * g.cipix + g.chpix0));
  const int h01 = int(floor(y01 * g.cipix + g.chpix0));
  const int h10 = int(floor(y10 * g.cipix + g.chpix0));
  const int h11 = int(floor(y11 * g.cipix + g.chpix0));
  const int hmin = max(min(min(h00, h01), min(h10, h11)), 0);
  const int hmax = min(max(max(h00, h01), max(h10, h11)), g.nh - 1);
  for (int h = hmin; h <= hmax; h++) {
    const double p2x = g.cdx[a] - s * g.hpix[h];
    const double p2y = g.sdx[a] + c * g.hpix[h];
    const double ddx = p2x - p1x, ddy = p2y - p1y;
    if (fabs(ddx) < eps || fabs(ddy) < eps)
      continue; // rejected by the reference ("Ooops", c2D.cpp:909-912)
    const double idx = 1.0 / ddx, idy = 1.0 / ddy;
    const double ax0 = dx0 * idx, ay0 = dy0 * idy, axn = dxn * idx, ayn = dyn * idy;
    const double amin = dmax(dmax(dmin(ax0, axn), dmin(ay0, ayn)), 0.0);
    const double amax = dmin(dmin(dmax(ax0, axn), dmax(ay0, ayn)), 1.0);
    if (amin < amax - eps)
      f(h, float(amin), float(amax));
  }
}

// Band rows [lo, hi) of a ray entering a column at a0: rows whose slice and
// its neighbour stay inside the column (c2D.cpp:664-668).
__device__ __forceinline__ int cb_band_lo(const Geom &g, float a0) {
  return int(ceilf(__fadd_rn(g.pzdeps, __fdiv_rn(g.z1, a0))));
}
__device__ __forceinline__ int cb_band_hi(const Geom &g, float a0) {
  return int(floorf(__fadd_rn(g.pzdv, __fdiv_rn(g.znm, a0))));
}

// The back projector's band of every voxel column (c2D.cpp:657-676): the
// rows inside the band of every ray that crosses the column.  One warp per
// column, lanes over the angles; geometry only, built once per plan.
constexpr int kBandWarps = 8;
__global__ void __launch_bounds__(kBandWarps * 32) cb_column_band_kernel(Geom g, int2 *band) {
  const int col = blockIdx.x * kBandWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (col >= g.nx * g.ny)
    return; // the whole warp
  const int i = col / g.ny, j = col - i * g.ny;
  const double x0 = g.origin[0] + double(i) * g.size[0];
  const double xn = g.origin[0] + double(i + 1) * g.size[0];
  const double y0 = g.origin[1] + double(j) * g.size[1];
  const double yn = g.origin[1] + double(j + 1) * g.size[1];
  int lo = 0, hi = g.nv;
  for (int a = lane; a < g.na; a += 32)
    cb_column_rays(g, a, x0, xn, y0, yn, [&](int, float a0, float) {
      lo = max(lo, cb_band_lo(g, a0));
      hi = min(hi, cb_band_hi(g, a0));
    });
  lo = __reduce_max_sync(0xffffffffu, lo);
  hi = __reduce_min_sync(0xffffffffu, hi);
  if (lane == 0)
    band[col] = make_int2(lo, hi);
}

template <int EPI>
__global__ void __launch_bounds__(kBpThreads)
    cb_bp_kernel(Geom g, const float *__restrict__ pix, float *__restrict__ vol, Epi e,
                 int *err) {
  extern __shared__ unsigned char smem_raw[];
  float *acc = reinterpret_cast<float *>(smem_raw);
  const int cap = kBpAngleChunk * kBpMaxRaysPerAngle;
  int *seg_ah = reinterpret_cast<int *>(acc + g.nz);
  float *seg_a0 = reinterpret_cast<float *>(seg_ah + cap);
  float *seg_a1 = seg_a0 + cap;
  __shared__ int s_count, s_minv, s_maxv, s_ovf;
  const int col = blockIdx.x;
  const int i = col / g.ny, j = col - (col / g.ny) * g.ny;
  const double x0 = g.origin[0] + double(i) * g.size[0];
  const double xn = g.origin[0] + double(i + 1) * g.size[0];
  const double y0 = g.origin[1] + double(j) * g.size[1];
  const double yn = g.origin[1] + double(j + 1) * g.size[1];
  for (int z = threadIdx.x; z < g.nz; z += blockDim.x)
    acc[z] = 0.0f;
  if (threadIdx.x == 0) {
    // rows [min_v, max_v) stay inside the column for every ray
    // (c2D.cpp:657-676), from the plan's table
    const int2 b = g.colband[col];
    s_minv = b.x;
    s_maxv = b.y;
    s_ovf = 0;
  }
  __syncthreads();
  const int min_v = s_minv, max_v = s_maxv;
  const int nzm1 = g.nz - 1, mid = g.mid;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  for (int ac = 0; ac < g.na; ac += kBpAngleChunk) {
    if (threadIdx.x == 0)
      s_count = 0;
    __syncthreads();
    for (int a = ac + threadIdx.x; a < min(g.na, ac + kBpAngleChunk); a += blockDim.x) {
      cb_column_rays(g, a, x0, xn, y0, yn, [&](int h, float a0, float a1) {
        const int slot = atomicAdd(&s_count, 1);
        if (slot < cap) {
          seg_ah[slot] = a * g.nh + h;
          seg_a0[slot] = a0;
          seg_a1[slot] = a1;
        } else {
          s_ovf = 1;
        }
      });
    }
    __syncthreads();
    const int nseg = min(s_count, cap);
    for (int sgi = wib; sgi < nseg; sgi += kBpThreads / 32) {
      const int ah = seg_ah[sgi];
      const int h = ah % g.nh;
      const float a0 = seg_a0[sgi], a1 = seg_a1[sgi];
      const float av = __fmul_rn(a0, g.inv_dz);
      const float *prow = pix + i64(ah) * g.nv;
      const float *drow = g.dconv + i64(h) * g.nv;
      for (int v = lane; v < g.nv; v += 32) {
        const float p = __fmul_rn(__ldg(prow + v), __ldg(drow + v));
        const float dzv = g.dz[v], izv = g.iz[v];
        if (v >= min_v && v < max_v) {
          const int k = int(__fadd_rn(g.pzbz, __fmul_rn(av, dzv)));
          if (v < mid) {
            if (k < 1 || k > nzm1)
              continue;
            const float mz = fmin_ref(__fmul_rn(g.vz[k], izv), a1);
            atomicAdd(acc + k, __fmul_rn(p, __fsub_rn(mz, a0)));
            atomicAdd(acc + k - 1, __fmul_rn(p, __fsub_rn(a1, mz)));
          } else {
            if (k < 0 || k >= nzm1)
              continue;
            const float mz = fmin_ref(__fmul_rn(g.vz[k + 1], izv), a1);
            atomicAdd(acc + k, __fmul_rn(p, __fsub_rn(mz, a0)));
            atomicAdd(acc + k + 1, __fmul_rn(p, __fsub_rn(a1, mz)));
          }
        } else if (v < min_v) {
          const int k = int(__fadd_rn(g.pzbz1, __fmul_rn(av, dzv))) - 1;
          if (k > 0 && k <= nzm1) {
            const float mz = fmin_ref(__fmul_rn(g.vz[k], izv), a1);
            atomicAdd(acc + k, __fmul_rn(p, __fsub_rn(mz, a0)));
            atomicAdd(acc + k - 1, __fmul_rn(p, __fsub_rn(a1, mz)));
          } else if (k == 0) {
            const float mz = fmin_ref(__fmul_rn(g.vz[0], izv), a1);
            atomicAdd(acc, __fmul_rn(p, __fsub_rn(mz, a0)));
          }
        } else {
          const int k = int(__fadd_rn(g.pzbz, __fmul_rn(av, dzv)));
          if (k < nzm1 && k >= 0) {
            const float mz = fmin_ref(__fmul_rn(g.vz[k + 1], izv), a1);
            atomicAdd(acc + k, __fmul_rn(p, __fsub_rn(mz, a0)));
            atomicAdd(acc + k + 1, __fmul_rn(p, __fsub_rn(a1, mz)));
          } else if (k == nzm1) {
            const float mz = fmin_ref(__fmul_rn(g.vz[k + 1], izv), a1);
            atomicAdd(acc + k, __fmul_rn(p, __fsub_rn(mz, a0)));
          }
        }
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_ovf)
    atomicExch(err, 2);
  double ssq = 0.0;
  const i64 base = i64(col) * g.nz;
  for (int z = threadIdx.x; z < g.nz; z += blockDim.x) {
    const float v = acc[z];
    float o = v;
    if (EPI == EPI_NORM) {
      ssq += double(v) * double(v);
    } else if (EPI == EPI_SIRT) {
      const float t = __fadd_rn(e.x[base + z], __fmul_rn(1.0f, __fmul_rn(v, e.w[base + z])));
      o = (t < 0.0f) ? 0.0f : t;
    } else if (EPI == EPI_MLEM) {
      const float t = __fmul_rn(e.x[base + z], __fmul_rn(e.w[base + z], v));
      o = (t < 0.0f) ? 0.0f : t;
    }
    vol[base + z] = o;
  }
  if (EPI == EPI_NORM) {
    __shared__ double red[kBpThreads / 32];
    const double t = cta_sum<kBpThreads / 32>(ssq, red);
    if (threadIdx.x == 0)
      e.partials[blockIdx.x] = t;
  }
}

// ---- backward, deterministic gather in the reference's summation order
//
// cone_beam::calc_ah_z (c2D.cpp:640-751) adds, for every voxel of a column,
// first the band rows of every ray (list order: angle, then detector
// column; rows ascending, each row feeding its slice k and the neighbour
// k -/+ 1), then the edge rows of every ray (below the band descending,
// above it ascending).  Here one CTA owns one column and each thread owns
// NZT of its voxels.  Rays are staged per angle chunk.  For a stage of
// kGaStage rays each thread loads its band rows (RMAX per ray, all loads in
// flight together), forms every row's two contributions exactly as the
// reference does (p (mz - a0) for the row's slice k, p (a1 - mz) for its
// neighbour) and records, for every slice K, the first band row whose index
// reaches K (k is monotone in the row).  Each voxel thread then adds, per
// ray, exactly the contributions that go to its voxel, in the reference's
// order, so every voxel's sum is formed in the same order with the same
// unfused float operations as the reference.
constexpr int kGaThreads = 256;
constexpr int kGaChunk = 64;
constexpr int kGaRays = kBpMaxRaysPerAngle; // slots per angle
#ifndef CB_GA_STAGE
#define CB_GA_STAGE 3 // rays per stage when the kernel multiplies by d_conv itself
#endif
#ifndef CB_GA_STAGE_PRE
#define CB_GA_STAGE_PRE 4 // rays per stage on a sinogram already scaled by d_conv
#endif
#ifndef CB_GA_FAST
#define CB_GA_FAST 1
#endif
#ifndef CB_GA_PACKED
#define CB_GA_PACKED 1
#endif
#ifndef CB_GA_TILE
#define CB_GA_TILE 16 // CTAs walk the columns in 16 x 16 tiles (0: row-major order)
#endif
constexpr int kGaStageMax = 8;

__host__ __device__ inline int round4(int n) { return (n + 3) & ~3; }

// Shared-memory layout of cb_bp_gather (offsets in 4-byte words) for
// `st` rays per stage.
struct GaLayout {
  int vz, dz, iz, seg_h, seg_a0, seg_a1, cnt, off, map, fr, prow, drow, total;
  __host__ __device__ GaLayout(int nz, int nv, int st) {
    vz = 0;
    dz = vz + cb_vz_floats(nz);
    iz = dz + round4(nv);
    seg_h = iz + round4(nv);
    seg_a0 = seg_h + kGaChunk * kGaRays;
    seg_a1 = seg_a0 + kGaChunk * kGaRays;
    cnt = seg_a1 + kGaChunk * kGaRays;
    off = cnt + round4(kGaChunk + 1);
    map = off + round4(kGaChunk + 1);
    fr = map + kGaChunk * kGaRays;
    prow = fr + st * round4(nz + 2);
    drow = prow + st * round4(nv);
    total = drow + st * round4(nv);
  }
};

// Voxel column of CTA b: CTAs run through the xy plane in T x T tiles, so
// the columns in flight at any time form a compact patch whose rays (and
// the sinogram rows they read) overlap and stay in L2.  Any order gives the
// same sums: each CTA owns its column.
__device__ __forceinline__ int cb_ga_column(int b, int nx, int ny) {
#if CB_GA_TILE > 0
  constexpr int T = CB_GA_TILE;
  if (nx % T != 0 || ny % T != 0)
    return b;
  const int tile = b / (T * T), in = b - tile * (T * T);
  const int tpr = ny / T; // tiles along y
  const int ti = tile / tpr, tj = tile - ti * tpr;
  return (ti * T + in / T) * ny + tj * T + in % T;
#else
  return b;
#endif
}

// Stage the rays of angles [ac, ac + nac) in list order: slots per angle,
// then a prefix over angles and a flat map.  Returns the ray count.  Each
// slot holds the ray's detector column h and its entry and exit alphas.
__device__ int cb_ga_stage_rays(const Geom &g, int ac, int nac, double x0, double xn, double y0,
                                double yn, int *seg_h, float *seg_a0, float *seg_a1, int *cnt,
                                int *off, int *map, int *ovf) {
  const int tid = threadIdx.x;
  if (tid < nac) {
    int c = 0;
    cb_column_rays(g, ac + tid, x0, xn, y0, yn, [&](int h, float a0, float a1) {
      if (c < kGaRays) {
        const int idx = tid * kGaRays + c;
        seg_h[idx] = h;
        seg_a0[idx] = a0;
        seg_a1[idx] = a1;
      }
      c++;
    });
    if (c > kGaRays) {
      *ovf = 1;
      c = kGaRays;
    }
    cnt[tid] = c;
  }
  __syncthreads();
  if (tid == 0) {
    int acc = 0;
    for (int t = 0; t < nac; t++) {
      off[t] = acc;
      acc += cnt[t];
    }
    off[nac] = acc;
  }
  __syncthreads();
  if (tid < nac)
    for (int c = 0; c < cnt[tid]; c++)
      map[off[tid] + c] = tid * kGaRays + c;
  __syncthreads();
  return off[nac];
}

// First-row table: row v of slice k follows row v - 1 of slice kp, so v is
// the first band row of the slices kp + 1 .. k (entries 0 .. nz + 1 kept).
__device__ __forceinline__ void cb_ga_mark(int *f, int kp, int k, int v, int nz) {
#if CB_GA_FAST
  if (k == kp + 1 && k >= 0 && k <= nz + 1) {
    f[k] = v; // the usual step: one slice per row change
    return;
  }
#endif
  for (int K = max(kp + 1, 0); K <= min(k, nz + 1); K++)
    f[K] = v;
}

// Register bound: 4 CTAs per SM for one voxel per thread; taller columns
// need more shared memory per CTA, which allows 3 (or 2) anyway.
// PRE: the sinogram is already scaled by d_conv (the reference's dpixels,
// c2D.cpp:1096-1117, formed by the producer of the back projector's input),
// so a staged row is one load and no multiply.  ST rays per stage.
// BATCH: nbatch sinograms (EPI_STORE only); without it the item loop runs
// once and compiles away.
template <int EPI, int NZT, int RMAX, bool PRE, int ST, bool BATCH>
__global__ void __launch_bounds__(kGaThreads, NZT == 1 ? 4 : (NZT == 2 ? 3 : 2))
    cb_bp_gather(Geom g, const float *__restrict__ pix0, float *__restrict__ vol0, Epi e,
                 int *err, int nbatch) {
  static_assert(ST <= kGaStageMax, "stage too large");
  extern __shared__ unsigned char smem_raw[];
  int *W = reinterpret_cast<int *>(smem_raw);
  const int nz = g.nz, nv = g.nv, nzm1 = nz - 1, mid = g.mid;
  const GaLayout L(nz, nv, ST);
  float *svz = reinterpret_cast<float *>(W + L.vz);
  float *sdz = reinterpret_cast<float *>(W + L.dz);
  float *siz = reinterpret_cast<float *>(W + L.iz);
  int *seg_h = W + L.seg_h;
  float *seg_a0 = reinterpret_cast<float *>(W + L.seg_a0);
  float *seg_a1 = reinterpret_cast<float *>(W + L.seg_a1);
  int *cnt = W + L.cnt, *off = W + L.off, *map = W + L.map, *fr = W + L.fr;
  float *prow = reinterpret_cast<float *>(W + L.prow); // staged pixel rows
  float *drow = reinterpret_cast<float *>(W + L.drow); // their d_conv rows
  const int frs = round4(nz + 2), prs = round4(nv);
  __shared__ int s_minv, s_maxv, s_ovf;
  __shared__ int s_kf[ST], s_kl[ST]; // slices of a staged ray's first/last band row
  // the column's square; kept in shared memory so that its FP64 corners
  // hold no registers through the row and voxel phases
  __shared__ double s_box[4];
  const int tid = threadIdx.x;
  const int col = cb_ga_column(blockIdx.x, g.nx, g.ny);
  const int i = col / g.ny, j = col - (col / g.ny) * g.ny;
  for (int t = tid; t <= nz; t += blockDim.x)
    svz[t] = g.vz[t];
  for (int t = tid; t < nv; t += blockDim.x) {
    sdz[t] = g.dz[t];
    siz[t] = g.iz[t];
  }
  if (tid == 0) {
    // band limits over every ray of the column (c2D.cpp:657-676), from
    // the plan's table
    const int2 b = g.colband[col];
    s_minv = b.x;
    s_maxv = b.y;
    s_ovf = 0;
    s_box[0] = g.origin[0] + double(i) * g.size[0];
    s_box[1] = g.origin[0] + double(i + 1) * g.size[0];
    s_box[2] = g.origin[1] + double(j) * g.size[1];
    s_box[3] = g.origin[1] + double(j + 1) * g.size[1];
  }
  __syncthreads();
  const int min_v = s_minv, max_v = s_maxv;
  const int nb = max_v - min_v;
  const int lo_end = min(mid, max_v);         // lower band rows [min_v, lo_end)
  const int up_begin = max(mid, min_v);       // upper band rows [up_begin, max_v)
  const float pzbz = g.pzbz, pzbz1 = g.pzbz1, inv_dz = g.inv_dz;
  // this thread's band rows v = min_v + tid + r * 256 are the same for every
  // ray: their z tables stay in registers (sd: delta_z of v, sp: of v - 1,
  // si: inv_delz of v)
  float rsd[RMAX], rsp[RMAX], rsi[RMAX];
#pragma unroll
  for (int r = 0; r < RMAX; r++) {
    const int v = min_v + tid + r * kGaThreads;
    const bool in = v < max_v;
    rsd[r] = in ? sdz[v] : 0.0f;
    rsp[r] = (in && v > min_v) ? sdz[v - 1] : 0.0f;
    rsi[r] = in ? siz[v] : 0.0f;
  }
  const float sd_first = nb > 0 ? sdz[min_v] : 0.0f, sd_last = nb > 0 ? sdz[max_v - 1] : 0.0f;
  double ssq = 0.0;
  // nbatch sinograms (one after another) share the column's band limits
  for (int bi = 0; bi < (BATCH ? nbatch : 1); bi++) {
  const float *__restrict__ pix = pix0 + i64(bi) * g.na * g.nh * nv;
  float *__restrict__ vol = vol0 + i64(bi) * g.nx * g.ny * nz;
  float acc[NZT];
#pragma unroll
  for (int q = 0; q < NZT; q++)
    acc[q] = 0.0f;

  // ---- band rows of every ray (c2D.cpp:680-713)
  for (int ac = 0; nb > 0 && ac < g.na; ac += kGaChunk) {
    const int nac = min(kGaChunk, g.na - ac);
    const int nseg = cb_ga_stage_rays(g, ac, nac, s_box[0], s_box[1], s_box[2], s_box[3], seg_h,
                                      seg_a0, seg_a1, cnt, off, map, &s_ovf);
    for (int s0 = 0; s0 < nseg; s0 += ST) {
      const int ns = min(ST, nseg - s0);
      // 1) this thread's band rows v = min_v + tid + r * 256 of every staged
      //    ray: pixel values (times d_conv unless pre-scaled), all loads
      //    issued together
      float pv[ST][RMAX], dv[PRE ? 1 : ST][RMAX];
#pragma unroll
      for (int s = 0; s < ST; s++) {
        const int m = map[s0 + (s < ns ? s : 0)];
        const int h = seg_h[m];
        const float *prw = pix + (i64(ac + m / kGaRays) * g.nh + h) * nv;
#pragma unroll
        for (int r = 0; r < RMAX; r++) {
          const int v = min_v + tid + r * kGaThreads;
          const bool ok = s < ns && v < max_v;
          pv[s][r] = ok ? __ldg(prw + v) : 0.0f;
        }
        if (!PRE) {
          const float *drw = g.dconv + i64(h) * nv;
#pragma unroll
          for (int r = 0; r < RMAX; r++) {
            const int v = min_v + tid + r * kGaThreads;
            dv[PRE ? 0 : s][r] = (s < ns && v < max_v) ? __ldg(drw + v) : 0.0f;
          }
        }
      }
      // 2) per ray: the first band row of every slice index (the whole
      //    table: below the first row's slice min_v, above the last row's
      //    max_v) and each row's two contributions as the reference forms
      //    them (c2D.cpp:694-711): c1 = p (mz - a0) goes to slice k, c2 =
      //    p (a1 - mz) to k - 1 below the source row, to k + 1 from it on
#pragma unroll
      for (int s = 0; s < ST; s++) {
        if (s >= ns)
          break;
        const int m = map[s0 + s];
        const float a0 = seg_a0[m], a1 = seg_a1[m];
        const float av = __fmul_rn(a0, inv_dz);
        int *f = fr + s * frs;
        const int kf = int(__fadd_rn(pzbz, __fmul_rn(av, sd_first)));
        const int kl = int(__fadd_rn(pzbz, __fmul_rn(av, sd_last)));
#if CB_GA_FAST
        // only voxels kf - 1 .. kl + 1 receive rows of this ray, and they
        // read entries kf - 2 .. kl + 3: the band rows' transitions write
        // (kf, kl], six threads write the ends
        if (tid < 6) {
          const int K = tid < 3 ? kf - tid : kl + tid - 2;
          if (K >= 0 && K <= nz + 1)
            f[K] = tid < 3 ? min_v : max_v;
        }
        if (tid == 0) {
          s_kf[s] = kf;
          s_kl[s] = kl;
        }
#else
        for (int K = tid; K <= nz + 1; K += kGaThreads) {
          if (K <= kf)
            f[K] = min_v;
          else if (K > kl)
            f[K] = max_v;
        }
#endif
        float *c1 = prow + s * prs, *c2 = drow + s * prs;
#if CB_GA_PACKED
        const float2 av2 = make_float2(av, av), a02 = make_float2(a0, a0),
                     a12 = make_float2(a1, a1);
#endif
#pragma unroll
        for (int r = 0; r < RMAX; r++) {
#if CB_GA_PACKED
          if (r + 1 < RMAX && (r & 1) == 0) {
            // rows r and r + 1 as packed pairs: the same unfused float
            // operations per row, two rows per multiply and subtract
            const int v0 = min_v + tid + r * kGaThreads, v1 = v0 + kGaThreads;
            const float2 kk = mul2_rn(av2, make_float2(rsd[r], rsd[r + 1]));
            const float2 kq = mul2_rn(av2, make_float2(rsp[r], rsp[r + 1]));
            const int k0 = int(__fadd_rn(pzbz, kk.x)), k1 = int(__fadd_rn(pzbz, kk.y));
            if (v0 < max_v && v0 > min_v)
              cb_ga_mark(f, int(__fadd_rn(pzbz, kq.x)), k0, v0, nz);
            if (v1 < max_v)
              cb_ga_mark(f, int(__fadd_rn(pzbz, kq.y)), k1, v1, nz);
            const int kz0 = min(max(v0 < mid ? k0 : k0 + 1, 0), nz);
            const int kz1 = min(max(v1 < mid ? k1 : k1 + 1, 0), nz);
            const float2 pl =
                mul2_rn(make_float2(svz[kz0], svz[kz1]), make_float2(rsi[r], rsi[r + 1]));
            const float2 mz = make_float2(fmin_ref(pl.x, a1), fmin_ref(pl.y, a1));
            const float2 p = PRE ? make_float2(pv[s][r], pv[s][r + 1])
                                 : mul2_rn(make_float2(pv[s][r], pv[s][r + 1]),
                                           make_float2(dv[PRE ? 0 : s][r], dv[PRE ? 0 : s][r + 1]));
            const float2 w1 = mul2_rn(p, sub2_rn(mz, a02)), w2 = mul2_rn(p, sub2_rn(a12, mz));
            if (v0 < max_v) {
              c1[v0] = w1.x;
              c2[v0] = w2.x;
            }
            if (v1 < max_v) {
              c1[v1] = w1.y;
              c2[v1] = w2.y;
            }
            continue;
          }
          if (r & 1)
            continue; // done with its pair
#endif
          const int v = min_v + tid + r * kGaThreads;
          if (v < max_v) {
            const int k = int(__fadd_rn(pzbz, __fmul_rn(av, rsd[r])));
            if (v > min_v)
              cb_ga_mark(f, int(__fadd_rn(pzbz, __fmul_rn(av, rsp[r]))), k, v, nz);
            const int kz = min(max(v < mid ? k : k + 1, 0), nz);
            const float mz = fmin_ref(__fmul_rn(svz[kz], rsi[r]), a1);
            const float p = PRE ? pv[s][r] : __fmul_rn(pv[s][r], dv[PRE ? 0 : s][r]);
            c1[v] = __fmul_rn(p, __fsub_rn(mz, a0));
            c2[v] = __fmul_rn(p, __fsub_rn(a1, mz));
          }
        }
      }
      __syncthreads();
      // 3) each voxel adds its rows' contributions in the reference's order
      for (int s = 0; s < ns; s++) {
        const int *f = fr + s * frs;
        const float *c1 = prow + s * prs, *c2 = drow + s * prs;
#if CB_GA_FAST
        const int klo = s_kf[s] - 1, khi = s_kl[s] + 1;
#endif
#pragma unroll
        for (int q = 0; q < NZT; q++) {
          const int K = tid + q * kGaThreads;
          if (K >= nz)
            continue;
#if CB_GA_FAST
          if (K < klo || K > khi)
            continue; // no row of this ray feeds voxel K
#endif
          const int fm = K >= 1 ? f[K - 1] : min_v, f0 = f[K], f1 = f[K + 1];
          float t = acc[q];
          // below the source row: rows of slice K give c1, then rows of
          // slice K + 1 give c2 (their neighbour k - 1 == K)
          for (int v = f0, ve = min(f[K + 2], lo_end); v < ve; v++)
            t = __fadd_rn(t, (v < f1 ? c1 : c2)[v]);
          // from the source row on: rows of slice K - 1 give c2 (their
          // neighbour k + 1 == K), then rows of slice K give c1
          for (int v = max(fm, up_begin), ve = min(f1, max_v); v < ve; v++)
            t = __fadd_rn(t, (v < f0 ? c2 : c1)[v]);
          acc[q] = t;
        }
      }
      __syncthreads();
    }
  }

  // ---- edge rows of every ray (c2D.cpp:715-750)
  if (min_v > 0 || max_v < nv) {
    for (int ac = 0; ac < g.na; ac += kGaChunk) {
      const int nac = min(kGaChunk, g.na - ac);
      const int nseg = cb_ga_stage_rays(g, ac, nac, s_box[0], s_box[1], s_box[2], s_box[3],
                                        seg_h, seg_a0, seg_a1, cnt, off, map, &s_ovf);
      for (int s = 0; s < nseg; s++) {
        const int m = map[s];
        const int h = seg_h[m];
        const float a0 = seg_a0[m], a1 = seg_a1[m];
        const float av = __fmul_rn(a0, inv_dz);
        const float *prw = pix + (i64(ac + m / kGaRays) * g.nh + h) * nv;
        const float *drw = g.dconv + i64(h) * nv;
#pragma unroll
        for (int q = 0; q < NZT; q++) {
          const int K = tid + q * kGaThreads;
          if (K >= nz)
            continue;
          for (int v = min(min_v, nv) - 1; v >= 0; v--) {
            const int k = int(__fadd_rn(pzbz1, __fmul_rn(av, sdz[v]))) - 1;
            if (k < K)
              break; // k only falls as v falls (and k < 0 ends the reference's loop)
            if (k > K + 1)
              continue;
            const float p = PRE ? __ldg(prw + v) : __fmul_rn(__ldg(prw + v), __ldg(drw + v));
            if (k > 0) {
              const float mz = fmin_ref(__fmul_rn(svz[k], siz[v]), a1);
              acc[q] = __fadd_rn(acc[q], __fmul_rn(p, k == K ? __fsub_rn(mz, a0)
                                                             : __fsub_rn(a1, mz)));
            } else if (K == 0) {
              const float mz = fmin_ref(__fmul_rn(svz[0], siz[v]), a1);
              acc[q] = __fadd_rn(acc[q], __fmul_rn(p, __fsub_rn(mz, a0)));
            }
          }
          for (int v = max(max_v, 0); v < nv; v++) {
            const int k = int(__fadd_rn(pzbz, __fmul_rn(av, sdz[v])));
            if (k > K || k > nzm1)
              break; // k only rises with v (and k > nz - 1 ends the reference's loop)
            if (k < K - 1)
              continue;
            const float p = PRE ? __ldg(prw + v) : __fmul_rn(__ldg(prw + v), __ldg(drw + v));
            const float mz = fmin_ref(__fmul_rn(svz[k + 1], siz[v]), a1);
            if (k == K)
              acc[q] = __fadd_rn(acc[q], __fmul_rn(p, __fsub_rn(mz, a0)));
            else if (k < nzm1)
              acc[q] = __fadd_rn(acc[q], __fmul_rn(p, __fsub_rn(a1, mz)));
          }
        }
      }
      __syncthreads();
    }
  }
  const i64 base = i64(col) * nz;
#pragma unroll
  for (int q = 0; q < NZT; q++) {
    const int K = tid + q * kGaThreads;
    if (K >= nz)
      continue;
    const float v = acc[q];
    float o = v;
    if (EPI == EPI_NORM) {
      ssq += double(v) * double(v);
    } else if (EPI == EPI_SIRT) {
      const float t = __fadd_rn(e.x[base + K], __fmul_rn(1.0f, __fmul_rn(v, e.w[base + K])));
      o = (t < 0.0f) ? 0.0f : t;
    } else if (EPI == EPI_MLEM) {
      const float t = __fmul_rn(e.x[base + K], __fmul_rn(e.w[base + K], v));
      o = (t < 0.0f) ? 0.0f : t;
    }
    vol[base + K] = o;
  }
  } // batch items
  if (tid == 0 && s_ovf)
    atomicExch(err, 2);
  if (EPI == EPI_NORM) {
    __shared__ double red[kGaThreads / 32];
    const double t = cta_sum<kGaThreads / 32>(ssq, red);
    if (threadIdx.x == 0)
      e.partials[blockIdx.x] = t;
  }
}

} // namespace

size_t cb_fp_smem(const Geom &g) {
  return (size_t(cb_vz_floats(g.nz)) + size_t(kFpWarps) * 2 * size_t(g.nx + g.ny + 2)) *
         sizeof(float);
}

// Consecutive rows per lane of the scatter for nv rows: fewest idle rows,
// then 2, 3, 1 (measured at 512^3, 256^3 and on 24-row detectors).
int cb_scatter_rpl(int nv) {
  int best = 2;
  long long best_waste = -1;
  for (int r : {2, 3, 1}) {
    const long long per = 32ll * r;
    const long long waste = ((nv + per - 1) / per) * per - nv;
    if (best_waste < 0 || waste < best_waste) {
      best = r;
      best_waste = waste;
    }
  }
  return best;
}

int cb_backward_scatter(const Geom &g, const float *pix, float *vol, int pre,
                        const int2 *hrange, int grid, cudaStream_t st) {
  if (cudaMemsetAsync(vol, 0, size_t(g.nx) * g.ny * g.nz * sizeof(float), st) != cudaSuccess)
    return 2;
  const size_t smem = cb_fp_smem(g);
  const int cap = g.nx + g.ny + 2;
#define CB_SC_GO(R)                                                                        \
  (pre ? cb_bp_scatter<R, true><<<grid, kFpWarps * 32, smem, st>>>(g, pix, vol, hrange, cap)  \
       : cb_bp_scatter<R, false><<<grid, kFpWarps * 32, smem, st>>>(g, pix, vol, hrange, cap))
  switch (cb_scatter_rpl(g.nv)) {
  case 1:
    CB_SC_GO(1);
    break;
  case 3:
    CB_SC_GO(3);
    break;
  default:
    CB_SC_GO(2);
  }
#undef CB_SC_GO
  return 0;
}

int cb_column_bands(const Geom &g, int2 *band, cudaStream_t st) {
  const int ncol = g.nx * g.ny;
  cb_column_band_kernel<<<(ncol + kBandWarps - 1) / kBandWarps, kBandWarps * 32, 0, st>>>(g, band);
  return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

namespace {
// Rows per lane for nv rows: fewest idle lanes, then fewest passes.
int cb_fp_rpl(int nv) {
#ifdef CB_FP_FORCE_RPL
  return CB_FP_FORCE_RPL;
#endif
  int best = 4;
  long long best_waste = -1;
  for (int r : {4, 8, 12}) {
    const long long per = 32ll * r;
    const long long waste = ((nv + per - 1) / per) * per - nv;
    if (best_waste < 0 || waste < best_waste || (waste == best_waste && r > best)) {
      best = r;
      best_waste = waste;
    }
  }
  return best;
}

template <int EPI>
void launch_cb_fp(const Geom &g, const float *vol, float *pix, const Epi &e, const int2 *hrange,
                  int grid, cudaStream_t st, int nb) {
  const size_t smem = cb_fp_smem(g);
  const int cap = g.nx + g.ny + 2;
  const int r = (g.tune_rpl == 4 || g.tune_rpl == 8 || g.tune_rpl == 12) ? g.tune_rpl
                                                                          : cb_fp_rpl(g.nv);
  const bool full = g.nv % (32 * r) == 0;
#define CB_FP_GO(R, F, B)                                                                  \
  cb_fp_kernel<EPI, R, F, B><<<grid, kFpWarps * 32, smem, st>>>(g, vol, pix, e, hrange, cap, nb)
  if constexpr (EPI == EPI_STORE) {
    if (nb > 1) {
      if (r == 12)
        full ? CB_FP_GO(12, true, true) : CB_FP_GO(12, false, true);
      else if (r == 8)
        full ? CB_FP_GO(8, true, true) : CB_FP_GO(8, false, true);
      else
        full ? CB_FP_GO(4, true, true) : CB_FP_GO(4, false, true);
      return;
    }
  }
  if (r == 12)
    full ? CB_FP_GO(12, true, false) : CB_FP_GO(12, false, false);
  else if (r == 8)
    full ? CB_FP_GO(8, true, false) : CB_FP_GO(8, false, false);
  else
    full ? CB_FP_GO(4, true, false) : CB_FP_GO(4, false, false);
#undef CB_FP_GO
}
} // namespace

namespace {
size_t cb_bp_atomic_smem(const Geom &g) {
  return size_t(g.nz) * sizeof(float) +
         size_t(kBpAngleChunk) * kBpMaxRaysPerAngle * (sizeof(int) + 2 * sizeof(float));
}
// the larger of the two stage sizes' layouts
size_t cb_bp_gather_smem(const Geom &g) {
  return size_t(GaLayout(g.nz, g.nv, std::max(CB_GA_STAGE, CB_GA_STAGE_PRE)).total) * 4;
}
// voxels per thread of the deterministic gather, 0 if it does not apply
int cb_bp_gather_nzt(const Geom &g) {
  if (cb_bp_gather_smem(g) > 200 * 1024 || g.nv > 4 * kGaThreads)
    return 0;
  return g.nz <= kGaThreads ? 1 : g.nz <= 2 * kGaThreads ? 2 : g.nz <= 4 * kGaThreads ? 4 : 0;
}
// band rows per thread of the deterministic gather (nv <= 1024)
int cb_bp_gather_rmax(const Geom &g) { return (g.nv + kGaThreads - 1) / kGaThreads; }
} // namespace

size_t cb_bp_smem(const Geom &g) {
  return cb_bp_gather_nzt(g) ? cb_bp_gather_smem(g) : cb_bp_atomic_smem(g);
}

int cb_prepare(const Geom &g) {
  const int fp = int(cb_fp_smem(g)), bp = int(cb_bp_atomic_smem(g));
  const int ga = int(cb_bp_gather_smem(g));
  cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
#define CB_FP_ALL(R, F)                                                                    \
  (const void *)cb_fp_kernel<EPI_STORE, R, F, false>,                                       \
      (const void *)cb_fp_kernel<EPI_NORM, R, F, false>,                                    \
      (const void *)cb_fp_kernel<EPI_SIRT, R, F, false>,                                    \
      (const void *)cb_fp_kernel<EPI_MLEM, R, F, false>,                                    \
      (const void *)cb_fp_kernel<EPI_STORE, R, F, true>
  const void *fps[] = {CB_FP_ALL(4, false), CB_FP_ALL(8, false), CB_FP_ALL(12, false),
                       CB_FP_ALL(4, true),  CB_FP_ALL(8, true),  CB_FP_ALL(12, true),
                       (const void *)cb_bp_scatter<1, false>,
                       (const void *)cb_bp_scatter<1, true>,
                       (const void *)cb_bp_scatter<2, false>,
                       (const void *)cb_bp_scatter<2, true>,
                       (const void *)cb_bp_scatter<3, false>,
                       (const void *)cb_bp_scatter<3, true>};
#undef CB_FP_ALL
  const void *bps[] = {(const void *)cb_bp_kernel<EPI_STORE>, (const void *)cb_bp_kernel<EPI_NORM>,
                       (const void *)cb_bp_kernel<EPI_SIRT>, (const void *)cb_bp_kernel<EPI_MLEM>};
  for (const void *f : fps)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, fp) != cudaSuccess)
      e1 = cudaErrorInvalidValue;
  for (const void *f : bps)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bp) != cudaSuccess)
      e2 = cudaErrorInvalidValue;
  if (cb_bp_gather_nzt(g)) {
#define CB_GA_EPI(Z, R)                                                                    \
  (const void *)cb_bp_gather<EPI_STORE, Z, R, false, CB_GA_STAGE, false>,                   \
      (const void *)cb_bp_gather<EPI_NORM, Z, R, false, CB_GA_STAGE, false>,                \
      (const void *)cb_bp_gather<EPI_SIRT, Z, R, false, CB_GA_STAGE, false>,                \
      (const void *)cb_bp_gather<EPI_MLEM, Z, R, false, CB_GA_STAGE, false>,                \
      (const void *)cb_bp_gather<EPI_STORE, Z, R, true, CB_GA_STAGE_PRE, false>,            \
      (const void *)cb_bp_gather<EPI_NORM, Z, R, true, CB_GA_STAGE_PRE, false>,             \
      (const void *)cb_bp_gather<EPI_SIRT, Z, R, true, CB_GA_STAGE_PRE, false>,             \
      (const void *)cb_bp_gather<EPI_MLEM, Z, R, true, CB_GA_STAGE_PRE, false>,             \
      (const void *)cb_bp_gather<EPI_STORE, Z, R, false, CB_GA_STAGE, true>,                \
      (const void *)cb_bp_gather<EPI_STORE, Z, R, true, CB_GA_STAGE_PRE, true>
#define CB_GA_ALL(Z) CB_GA_EPI(Z, 1), CB_GA_EPI(Z, 2), CB_GA_EPI(Z, 3), CB_GA_EPI(Z, 4)
    const void *gas[] = {CB_GA_ALL(1), CB_GA_ALL(2), CB_GA_ALL(4)};
#undef CB_GA_EPI
#undef CB_GA_ALL
    for (const void *f : gas)
      if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, ga) != cudaSuccess)
        e2 = cudaErrorInvalidValue;
  }
  return (e1 == cudaSuccess && e2 == cudaSuccess) ? 0 : 1;
}

int cb_forward(const Geom &g, const float *vol, float *pix, int mode, const Epi &e,
               const int2 *hrange, int grid, cudaStream_t st, int nb) {
  switch (mode) {
  case EPI_STORE:
    launch_cb_fp<EPI_STORE>(g, vol, pix, e, hrange, grid, st, nb);
    break;
  case EPI_NORM:
    launch_cb_fp<EPI_NORM>(g, vol, pix, e, hrange, grid, st, nb);
    break;
  case EPI_SIRT:
    launch_cb_fp<EPI_SIRT>(g, vol, pix, e, hrange, grid, st, nb);
    break;
  case EPI_MLEM:
    launch_cb_fp<EPI_MLEM>(g, vol, pix, e, hrange, grid, st, nb);
    break;
  default:
    return 1;
  }
  return 0;
}

namespace {
// out[a][h][v] = in[a][h][v] * d_conv[h][v]: the reference's dpixels
// (c2D.cpp:1096-1117), the same float products the back projector would
// form row by row.
__global__ void cb_prescale_kernel(const float *__restrict__ in, float *__restrict__ out,
                                   const float *__restrict__ dconv, i64 per_angle, i64 n) {
  for (i64 i = blockIdx.x * i64(blockDim.x) + threadIdx.x; i < n;
       i += i64(gridDim.x) * blockDim.x)
    out[i] = __fmul_rn(in[i], dconv[i % per_angle]);
}

template <int EPI, bool PRE, int ST>
void launch_cb_ga(const Geom &g, int nzt, int rmax, const float *pix, float *vol, const Epi &e,
                  int *err, cudaStream_t st, int nbatch) {
  const int ncol = g.nx * g.ny;
  const size_t gsm = cb_bp_gather_smem(g);
#define CB_GA_ONE(Z, R, B)                                                                 \
  cb_bp_gather<EPI, Z, R, PRE, ST, B><<<ncol, kGaThreads, gsm, st>>>(g, pix, vol, e, err, nbatch)
#define CB_GA_GO(Z, B)                                                                     \
  (rmax == 1   ? CB_GA_ONE(Z, 1, B)                                                         \
   : rmax == 2 ? CB_GA_ONE(Z, 2, B)                                                         \
   : rmax == 3 ? CB_GA_ONE(Z, 3, B)                                                         \
               : CB_GA_ONE(Z, 4, B))
  if constexpr (EPI == EPI_STORE) {
    if (nbatch > 1) {
      if (nzt == 1)
        CB_GA_GO(1, true);
      else if (nzt == 2)
        CB_GA_GO(2, true);
      else
        CB_GA_GO(4, true);
      return;
    }
  }
  if (nzt == 1)
    CB_GA_GO(1, false);
  else if (nzt == 2)
    CB_GA_GO(2, false);
  else
    CB_GA_GO(4, false);
#undef CB_GA_GO
#undef CB_GA_ONE
}

template <int EPI>
void launch_cb_bp(const Geom &g, const float *pix, float *vol, const Epi &e, int *err,
                  cudaStream_t st, int nbatch) {
  const int ncol = g.nx * g.ny;
  const int nzt = cb_bp_gather_nzt(g), rmax = cb_bp_gather_rmax(g);
  if (nzt && e.pre) {
    launch_cb_ga<EPI, true, CB_GA_STAGE_PRE>(g, nzt, rmax, pix, vol, e, err, st, nbatch);
    return;
  }
  switch (nzt) {
  case 1:
  case 2:
  case 4:
    launch_cb_ga<EPI, false, CB_GA_STAGE>(g, nzt, rmax, pix, vol, e, err, st, nbatch);
    break;
  default:
    // columns taller than the gather handles: one launch per batch item
    for (int b = 0; b < nbatch; b++)
      cb_bp_kernel<EPI><<<ncol, kBpThreads, cb_bp_atomic_smem(g), st>>>(
          g, pix + i64(b) * g.na * g.nh * g.nv, vol + i64(b) * g.nx * g.ny * g.nz, e, err);
  }
}
} // namespace

bool cb_bp_takes_prescaled(const Geom &g) { return cb_bp_gather_nzt(g) != 0; }

void cb_prescale(const Geom &g, const float *in, float *out, cudaStream_t st) {
  const i64 per = i64(g.nh) * g.nv, n = i64(g.na) * per;
  const i64 blocks = std::min<i64>((n + 255) / 256, i64(sm_count()) * 8);
  cb_prescale_kernel<<<int(std::max<i64>(blocks, 1)), 256, 0, st>>>(in, out, g.dconv, per, n);
}

int cb_backward(const Geom &g, const float *pix, float *vol, int mode, const Epi &e,
                int *err, cudaStream_t st, int nbatch) {
  switch (mode) {
  case EPI_STORE:
    launch_cb_bp<EPI_STORE>(g, pix, vol, e, err, st, nbatch);
    break;
  case EPI_NORM:
    launch_cb_bp<EPI_NORM>(g, pix, vol, e, err, st, nbatch);
    break;
  case EPI_SIRT:
    launch_cb_bp<EPI_SIRT>(g, pix, vol, e, err, st, nbatch);
    break;
  case EPI_MLEM:
    launch_cb_bp<EPI_MLEM>(g, pix, vol, e, err, st, nbatch);
    break;
  default:
    return 1;
  }
  return 0;
}

} // namespace ccpi
