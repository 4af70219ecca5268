// Shared device-side definitions for the B200 projectors and solvers.
//
// Data layout in HBM is the reference's (Core/src/base_types.hpp:45-63,
// instruments.cpp:29-33): sinogram [angle][h][v] with detector rows v
// fastest, volume [x][y][z] with z fastest.  The v/z axis is the lane axis
// of every projector kernel, so warps read and write contiguous rows.
//
// Arithmetic that decides which voxels a ray visits, or that the reference
// rounds in a particular order, is written with explicitly rounded
// intrinsics (__dadd_rn, __fmul_rn, ...) and the projector translation units
// are compiled with --fmad=false: the reference's x86-64 build never fuses a
// multiply-add, and fusing would change both tie decisions and results.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace ccpi {

typedef long long i64;

// Tie tolerance of both walks (p2D.cpp:20, c2D.cpp:15).
constexpr float kEps = FLT_EPSILON;

// Geometry of one problem as the kernels see it.  Plain data plus device
// pointers to per-angle / per-pixel tables built on the host (cos/sin are
// evaluated by the host C library, as the reference does, so angle tables
// are identical bit for bit).
struct Geom {
  int kind; // 0 parallel beam, 1 cone beam
  int na, nh, nv, nx, ny, nz;
  double origin[3], size[3];
  const double *cosA, *sinA; // na
  const double *hpix, *vpix; // nh, nv
  // ---- parallel beam (p2D.cpp)
  double det_x;           // 2 * max |origin|
  float d_conv;           // 3 * det_x, the ray's alpha span
  double ihp, hp0;        // 1/pixel step, h_pixels[0]/step
  const double *yoff, *ioff, *blen; // back-projector trapezoid tables (na)
  int map_type;           // 1, 2, 4 rows per slice, 0 general
  const int *map;         // nv: row -> slice
  const int *vlo, *vhi;   // nz: rows [vlo, vhi) mapping to each slice
  // ---- cone beam (c2D.cpp)
  double src[3], detx;
  double cl, cipix, chpix0; // det_x - src_x, 1/h step, (src_y - h0)/step
  const double *p1x, *p1y, *cdx, *sdx; // na
  const float *dconv;     // nh * nv source-pixel distance
  const float *dz, *iz;   // nv: v_pix - src_z and its reciprocal
  const float *vz;        // nz + 1: slice planes relative to src_z
  float inv_dz, pzbz, pzbz1, pzdv, z1, znm, pzdeps;
  int mid;                // first row above the source
  // nx * ny: per voxel column the back projector's band rows [x, y) that
  // stay inside the column for every ray crossing it (c2D.cpp:657-676)
  const int2 *colband;
  // ---- launch shapes chosen by ccpi_plan_autotune (0: the built-in choice)
  int tune_vw;            // parallel back projector: slices per lane (4, 8, 16)
  int tune_rpl;           // cone forward projector: rows per lane (4, 8, 12)
  int tune_scatter;       // cone back projector: 1 ray-driven scatter, 0 voxel gather
};

// Epilogue operands shared by the fused projector epilogues.
struct Epi {
  const float *b;    // measured sinogram (SIRT/MLEM) or unused
  const float *w;    // per-element weight: R (SIRT fp), C (SIRT bp), N (MLEM bp)
  float *x;          // volume updated in place by the back-projector epilogues
  double *partials;  // one FP64 partial sum of squares per CTA (NORM modes)
  int pre;           // cone beam: the back projector's input is already scaled by
                     // d_conv, and the forward projector's SIRT / MLEM output is
                     // stored scaled (the reference's dpixels, c2D.cpp:1096-1117)
};

enum EpiMode {
  EPI_STORE = 0, // out = A x
  EPI_NORM = 1,  // out = A x, and per-CTA sum of squares in FP64
  EPI_SIRT = 2,  // fp: r = (b - Ax) R       bp: x = max(x + C A^T r, 0)
  EPI_MLEM = 3,  // fp: q = max(b / Ax, 0)   bp: x = max(x (N A^T q), 0)
  EPI_ONES = 4,  // the input is all ones: out = A 1 or A^T 1 (no input read;
                 // 1 * l == l exactly, so the sums are those of a ones input)
};

__device__ __forceinline__ int warp_lane() { return threadIdx.x & 31; }

#ifndef CCPI_AXPY_PACKED
#define CCPI_AXPY_PACKED 1
#endif

// Blackwell packed FP32 pairs (PTX mul/sub/add.rn.f32x2, sm_100): one
// instruction rounds both lanes to nearest, each on its own, exactly as two
// scalar __fmul_rn / __fsub_rn / __fadd_rn would (subnormals kept, no .ftz).
// One rule keeps them equal to the unfused scalar arithmetic: a packed add
// or sub never takes a packed product as an operand, because ptxas
// contracts mul.f32x2 -> add.f32x2 into a fused multiply-add even with
// explicit rounding.  Products feed scalar adds instead.
__device__ __forceinline__ float2 mul2_rn(float2 a, float2 b) {
  float2 r;
  asm("{ .reg .b64 x, y, z;\n\t"
      "mov.b64 x, {%2, %3};\n\t"
      "mov.b64 y, {%4, %5};\n\t"
      "mul.rn.f32x2 z, x, y;\n\t"
      "mov.b64 {%0, %1}, z;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 sub2_rn(float2 a, float2 b) {
  float2 r;
  asm("{ .reg .b64 x, y, z;\n\t"
      "mov.b64 x, {%2, %3};\n\t"
      "mov.b64 y, {%4, %5};\n\t"
      "sub.rn.f32x2 z, x, y;\n\t"
      "mov.b64 {%0, %1}, z;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
  float2 r;
  asm("{ .reg .b64 x, y, z;\n\t"
      "mov.b64 x, {%2, %3};\n\t"
      "mov.b64 y, {%4, %5};\n\t"
      "add.rn.f32x2 z, x, y;\n\t"
      "mov.b64 {%0, %1}, z;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}

// (ax, ay) += (xx, xy) * w: the products as one packed multiply, the sums
// as scalar adds (see above: no packed add of a packed product).
__device__ __forceinline__ void axpy2_packed(float &ax, float &ay, float xx, float xy, float w) {
  const float2 p = mul2_rn(make_float2(xx, xy), make_float2(w, w));
  ax = __fadd_rn(ax, p.x);
  ay = __fadd_rn(ay, p.y);
}

// (ax, ay) += (p0, p1) as one packed add (p0, p1 not packed products).
__device__ __forceinline__ void add2_packed(float &ax, float &ay, float p0, float p1) {
  const float2 r = add2_rn(make_float2(ax, ay), make_float2(p0, p1));
  ax = r.x;
  ay = r.y;
}

// acc += x * w with scalar products and packed sums (the back projector's
// form; the forward projector's axpy4 packs the products instead).
__device__ __forceinline__ void axpy4_pa(float4 &acc, const float4 x, float w) {
#if CCPI_AXPY_PACKED
  add2_packed(acc.x, acc.y, __fmul_rn(x.x, w), __fmul_rn(x.y, w));
  add2_packed(acc.z, acc.w, __fmul_rn(x.z, w), __fmul_rn(x.w, w));
#else
  acc.x = __fadd_rn(acc.x, __fmul_rn(x.x, w));
  acc.y = __fadd_rn(acc.y, __fmul_rn(x.y, w));
  acc.z = __fadd_rn(acc.z, __fmul_rn(x.z, w));
  acc.w = __fadd_rn(acc.w, __fmul_rn(x.w, w));
#endif
}

// acc += x * w, element-wise, unfused (two roundings per element, as the
// reference's x86-64 build computes it).
__device__ __forceinline__ void axpy4(float4 &acc, const float4 x, float w) {
#if CCPI_AXPY_PACKED
  axpy2_packed(acc.x, acc.y, x.x, x.y, w);
  axpy2_packed(acc.z, acc.w, x.z, x.w, w);
#else
  acc.x = __fadd_rn(acc.x, __fmul_rn(x.x, w));
  acc.y = __fadd_rn(acc.y, __fmul_rn(x.y, w));
  acc.z = __fadd_rn(acc.z, __fmul_rn(x.z, w));
  acc.w = __fadd_rn(acc.w, __fmul_rn(x.w, w));
#endif
}

// acc += 1 * l for a ones input: the product is l exactly, so only the sums.
__device__ __forceinline__ void add_len4(float4 &acc, float l) {
  acc.x = __fadd_rn(acc.x, l);
  acc.y = __fadd_rn(acc.y, l);
  acc.z = __fadd_rn(acc.z, l);
  acc.w = __fadd_rn(acc.w, l);
}

// Deterministic CTA reduction of a double (fixed shuffle/smem order).
template <int NWARPS>
__device__ __forceinline__ double cta_sum(double v, double *scratch) {
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    scratch[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NWARPS; i++)
      t += scratch[i];
  }
  __syncthreads();
  return t;
}

} // namespace ccpi
