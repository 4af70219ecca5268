// Parallel-beam Siddon projectors for sm_100a.
//
// Forward (parallel_beam::f2D, Core/src/p2D.cpp:468-611): ray-driven.  One
// warp owns one ray (angle a, detector column h) and its lanes own detector
// rows v, so every voxel-column read and every sinogram write is a
// contiguous, coalesced row (float4 per lane when the layout allows).  The
// xy walk is warp-uniform and is evaluated exactly as the reference does:
// the volume is cut into 32x32 xy blocks, blocks are visited in the
// reference's (x-block, y-block) order, each block applies the reference's
// detector-column range rule and is walked from its own entry point with
// block-local alpha tables, ties within FLT_EPSILON advance both axes, and
// lengths are rounded to float.  Per row the sum is accumulated in the same
// order with unfused float multiply and add, so the result equals the
// reference bit for bit.
//
// Backward (parallel_beam::b2D, p2D.cpp:950-1087 with bproject_ah
// :775-948): a voxel-driven gather, the reference's own design.  A CTA owns
// a tile of xy voxel columns; it first evaluates, per (column, angle), the
// detector columns whose rays cross the voxel square and their exact
// trapezoid chord weights (FP64 geometry, float weights), staged in shared
// memory; then each thread owns (column, z) pairs and accumulates the
// sinogram rows in angle-then-column order, as the reference does.  No
// atomics.
//
// Both kernels take fused epilogues (EpiMode): the SIRT and MLEM updates and
// the FP64 sum of squares CGLS needs are applied to each output element
// before it is stored, so no extra pass over HBM is spent on them.
#include "common.cuh"
#include "kernels.h"

namespace ccpi {
namespace {

constexpr int kBlock = 32; // the reference's xy block edge (p2D.cpp:498-499)

// std::max / std::min semantics (first argument on ties).
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

// Detector columns that can see the xy box [vx,wx) x [vy,wy) (p2D.cpp:527-595;
// the per-voxel form at :808-915 is the same rule).
__device__ void pb_hrange(const Geom &g, double vx, double wx, double vy, double wy,
                          double c, double s, int &hmin, int &hmax) {
  const double eps = double(kEps);
  hmin = 0;
  hmax = g.nh - 1;
  if (fabs(c) < eps) {
    if (s < 0.0) {
      hmin = int(floor(vx * g.ihp - g.hp0));
      hmax = int(floor((wx - eps) * g.ihp - g.hp0));
    } else {
      hmin = int(ceil((-wx + eps) * g.ihp - g.hp0));
      hmax = int(ceil((-vx) * g.ihp - g.hp0));
    }
    hmin = max(hmin, 0);
    hmax = min(hmax, g.nh - 1);
  } else if (fabs(s) < eps) {
    if (c < 0.0) {
      hmin = int(ceil((-wy + eps) * g.ihp - g.hp0));
      hmax = int(ceil((-vy) * g.ihp - g.hp0));
    } else {
      hmin = int(floor(vy * g.ihp - g.hp0));
      hmax = int(floor((wy - eps) * g.ihp - g.hp0));
    }
    hmin = max(hmin, 0);
    hmax = min(hmax, g.nh - 1);
  } else {
    double ymin, ymax;
    if (c > 0.0) {
      if (s > 0.0) {
        ymin = vy * c - wx * s;
        ymax = wy * c - vx * s;
      } else {
        ymin = vy * c - vx * s;
        ymax = wy * c - wx * s;
      }
    } else {
      if (s > 0.0) {
        ymin = wy * c - wx * s;
        ymax = vy * c - vx * s;
      } else {
        ymin = wy * c - vx * s;
        ymax = vy * c - wx * s;
      }
    }
    hmin = (ymin < g.hpix[0]) ? 0 : int(floor(ymin * g.ihp - g.hp0));
    hmax = min(int(floor(ymax * g.ihp - g.hp0)), g.nh - 1);
  }
}

// Walk one non-axis-parallel ray through one block from the block's own
// entry point (p2D.cpp:284-458), calling emit(column, length) per cell.
// column = gx * ny + gy, or -1 outside the volume (the reference forms the
// same flattened offset (x * ny + y) * nz and reads it).  The next x and y boundary
// alphas are kept between steps and only the one crossed is re-evaluated,
// with the reference's formula (b + i d - p2) / cos.
template <class F>
__device__ __forceinline__ void pb_walk_block(const Geom &g, double p2x, double p2y,
                                              double c, double s, int bx0, int by0,
                                              int nxb, int nyb, double vx, double vy,
                                              F &emit) {
  const double eps = double(kEps);
  const double dx = g.size[0], dy = g.size[1];
  const double xn = vx + double(nxb) * dx, yn = vy + double(nyb) * dy;
  const double ic = 1.0 / c, is = 1.0 / s;
  const double ax0 = (vx - p2x) * ic, ay0 = (vy - p2y) * is;
  const double axn = (xn - p2x) * ic, ayn = (yn - p2y) * is;
  const double amin = dmax(dmax(dmin(ax0, axn), dmin(ay0, ayn)), double(-g.d_conv));
  const double amax = dmin(dmin(dmax(ax0, axn), dmax(ay0, ayn)), 0.0);
  if (!(amin < amax - eps))
    return;
  const int sx = c > 0.0 ? 1 : -1, sy = s > 0.0 ? 1 : -1;
  int x = 0, y = 0;
  const bool x_face_first = !(sx > 0 && sy < 0); // octant (+,-) tests y first
  auto cx = [&]() { return int(floor((p2x + amin * c - vx) / dx)); };
  auto cy = [&]() { return int(floor((p2y + amin * s - vy) / dy)); };
  const double axe = sx > 0 ? ax0 : axn; // entry through the x face
  const double aye = sy > 0 ? ay0 : ayn; // entry through the y face
  if (x_face_first) {
    if (amin == axe) {
      x = sx > 0 ? 0 : nxb - 1;
      if (sx < 0 && sy < 0 && amin == ayn)
        y = nyb - 1;
      else
        y = cy();
    } else if (amin == aye) {
      x = cx();
      y = sy > 0 ? 0 : nyb - 1;
    }
  } else {
    if (amin == aye) {
      x = cx();
      y = nyb - 1;
    } else if (amin == axe) {
      x = 0;
      y = cy();
    }
  }
  auto ax_at = [&](int i) { return (vx + double(i) * dx - p2x) * ic; };
  auto ay_at = [&](int j) { return (vy + double(j) * dy - p2y) * is; };
  const int ox = sx > 0 ? 1 : 0, oy = sy > 0 ? 1 : 0;
  double nxa = ax_at(x + ox), nya = ay_at(y + oy);
  double nxm = nxa - eps, nym = nya - eps;
  double ap = amin;
  const int ncol = g.nx * g.ny;
  const int cstep_x = sx * g.ny;
  int col = (bx0 + x) * g.ny + (by0 + y);
  while ((sx > 0 ? x < nxb : x >= 0) && (sy > 0 ? y < nyb : y >= 0)) {
    const int here = (unsigned(col) < unsigned(ncol)) ? col : -1;
    float len;
    if (nxa < nym) {
      len = float(nxa - ap);
      ap = nxa;
      x += sx;
      col += cstep_x;
      nxa = ax_at(x + ox);
      nxm = nxa - eps;
    } else if (nya < nxm) {
      len = float(nya - ap);
      ap = nya;
      y += sy;
      col += sy;
      nya = ay_at(y + oy);
      nym = nya - eps;
    } else {
      const double mx = dmax(nxa, nya);
      len = float(mx - ap);
      ap = mx;
      x += sx;
      y += sy;
      col += cstep_x + sy;
      nxa = ax_at(x + ox);
      nya = ay_at(y + oy);
      nxm = nxa - eps;
      nym = nya - eps;
    }
    emit(here, len);
  }
}

// All cells of ray (a, h) in the reference's accumulation order: blocks in
// (x-block, y-block) order, each applying the detector-column range rule.
// `room` is called before each block (it may flush staged cells).
template <class F, class R>
__device__ void pb_trace_ray(const Geom &g, int a, int h, F &emit, R &room) {
  const double eps = double(kEps);
  const double c = g.cosA[a], s = g.sinA[a], hv = g.hpix[h];
  const double p2x = c * g.det_x - s * hv;
  const double p2y = s * g.det_x + c * hv;
  const int nbx = (g.nx + kBlock - 1) / kBlock, nby = (g.ny + kBlock - 1) / kBlock;
  const double dx = g.size[0], dy = g.size[1];
  const int ncol = g.nx * g.ny;
  if (fabs(c) < eps && fabs(s) < eps)
    return;
  for (int bxi = 0; bxi < nbx; bxi++) {
    const int bx0 = bxi * kBlock, nxb = min(kBlock, g.nx - bx0);
    const double vx = g.origin[0] + double(bx0) * dx;
    const double wx = g.origin[0] + double(bx0 + nxb) * dx;
    int by_lo = 0, by_hi = nby - 1;
    int ix = 0;
    if (fabs(c) < eps) {
      // parallel to y: the block column that holds the ray by the floor rule
      ix = int(floor((p2x - vx) / dx));
      if (ix < 0 || ix >= nxb)
        continue;
    } else if (!(fabs(s) < eps)) {
      // prefilter: block rows the ray can cross inside this block column
      const double t = s / c;
      const double ya = p2y + (vx - p2x) * t, yb = p2y + (wx - p2x) * t;
      const double margin = 1e-3 * dy;
      const double ylo = fmin(ya, yb) - margin, yhi = fmax(ya, yb) + margin;
      const double bsz = double(kBlock) * dy;
      const double flo = floor((ylo - g.origin[1]) / bsz);
      const double fhi = floor((yhi - g.origin[1]) / bsz);
      if (fhi < 0.0 || flo > double(nby - 1))
        continue;
      by_lo = flo < 0.0 ? 0 : int(flo);
      by_hi = fhi > double(nby - 1) ? nby - 1 : int(fhi);
    }
    for (int byi = by_lo; byi <= by_hi; byi++) {
      const int by0 = byi * kBlock, nyb = min(kBlock, g.ny - by0);
      const double vy = g.origin[1] + double(by0) * dy;
      const double wy = g.origin[1] + double(by0 + nyb) * dy;
      int hmin, hmax;
      pb_hrange(g, vx, wx, vy, wy, c, s, hmin, hmax);
      if (h < hmin || h > hmax)
        continue;
      room();
      if (fabs(c) < eps) {
        const float len = float(dy);
        for (int t = 0; t < nyb; t++) {
          const int j = s < 0.0 ? nyb - 1 - t : t;
          const int col = (bx0 + ix) * g.ny + by0 + j;
          emit(unsigned(col) < unsigned(ncol) ? col : -1, len);
        }
      } else if (fabs(s) < eps) {
        const int jy = int(floor((p2y - vy) / dy));
        if (jy < 0 || jy >= nyb)
          continue;
        const float len = float(dx);
        for (int t = 0; t < nxb; t++) {
          const int i = c < 0.0 ? nxb - 1 - t : t;
          const int col = (bx0 + i) * g.ny + by0 + jy;
          emit(unsigned(col) < unsigned(ncol) ? col : -1, len);
        }
      } else {
        pb_walk_block(g, p2x, p2y, c, s, bx0, by0, nxb, nyb, vx, vy, emit);
      }
    }
  }
}

template <int EPI>
__device__ __forceinline__ float fp_epilogue(float acc, i64 idx, const Epi &e, double &ssq) {
  if (EPI == EPI_NORM) {
    ssq += double(acc) * double(acc);
    return acc;
  } else if (EPI == EPI_SIRT) {
    // sirt.cpp:60-62: r = (-1) r + b, then r *= R
    return __fmul_rn(__fadd_rn(-acc, e.b[idx]), e.w[idx]);
  } else if (EPI == EPI_MLEM) {
    // mlem.cpp:54,65 with blas.hpp div_xyz / clamp_min
    const float q = (acc != 0.0f) ? __fdiv_rn(e.b[idx], acc) : 0.0f;
    return (q < 0.0f) ? 0.0f : q;
  }
  return acc;
}

// One FP64 partial sum of squares per CTA.  A forward projection of more
// than 256 rows runs as several launches over row ranges on one stream with
// the same grid: the first (add == false) stores, the later ones add.
template <int NWARPS>
__device__ void store_partial(double ssq, const Epi &e, bool add = false) {
  __shared__ double red[NWARPS];
  const double t = cta_sum<NWARPS>(ssq, red);
  if (threadIdx.x == 0)
    e.partials[blockIdx.x] = add ? e.partials[blockIdx.x] + t : t;
}

// Staged cell lists: the warp-uniform walk emits (column, length) pairs into
// the warp's slice of shared memory; the lanes then accumulate them in
// order, four cells at a time with all loads issued before the adds.
constexpr int kFpWarps = 8;  // warps of a CTA trace one detector column at 8 angles
constexpr int kListCap = 256; // staged cells per warp
constexpr int kBlockCells = 72; // most cells one ray has in one 32x32 block

struct Cell {
  int col;
  float len;
};

// ---- forward, lane-parallel walk (row v -> slice v, nv and nz multiples of 4)
//
// One warp per ray.  The ray's blocks are first enumerated in the
// reference's order (lanes over block columns, prefix sum for positions).
// Then, 16 blocks at a time, every lane of a half-warp walks one block into
// its own slot of shared memory, and the warp replays the slots in block
// order with its lanes over detector rows, reading two staged cells per
// 16-byte shared load (all lanes read the same cells: broadcast).  The
// per-row additions are the same, in the same order, as a one-ray-at-a-time
// walk; only who evaluates the walk changes, so the instruction cost of the
// FP64 walk is shared by 16 blocks.
#ifndef PB_WALK_LANES
#define PB_WALK_LANES 16
#endif
#ifndef PB_FP_CTAS_PER_SM
#define PB_FP_CTAS_PER_SM 5
#endif
constexpr int kLaneWarps = 4;
constexpr int kWalkLanes = PB_WALK_LANES; // blocks walked in parallel per round
constexpr int kSlotCap = 66;    // cells of one ray in one block (<= 65); even, so
                                // every other entry starts a 16-byte pair
constexpr int kMaxBlocks = 192; // blocks one ray may visit (about nbx + nby)

// One staged cell: .x = the column's offset in float4 units (column * nz / 4),
// .y = the bits of its float length.  Cells outside the volume are dropped
// when staged (they add nothing).
struct LaneSmem {
  uint2 cell[kWalkLanes * kSlotCap];
  int blk[kMaxBlocks];
};

// Blocks of ray (c, s, p2) passing the reference's tests, counted (emit ==
// nullptr) or written in y-block order for one block column.
__device__ __forceinline__ int pb_column_blocks(const Geom &g, int h, double c, double s,
                                                double p2x, double p2y, bool par_y, bool par_x,
                                                int bxi, int *emit, int pos) {
  const double dx = g.size[0], dy = g.size[1];
  const int nby = (g.ny + kBlock - 1) / kBlock;
  const int bx0 = bxi * kBlock, nxb = min(kBlock, g.nx - bx0);
  const double vx = g.origin[0] + double(bx0) * dx;
  const double wx = g.origin[0] + double(bx0 + nxb) * dx;
  int lo = 0, hi = nby - 1;
  if (par_y) {
    const int ix = int(floor((p2x - vx) / dx));
    if (ix < 0 || ix >= nxb)
      return 0;
  } else if (!par_x) {
    const double tt = s / c;
    const double ya = p2y + (vx - p2x) * tt, yb = p2y + (wx - p2x) * tt;
    const double margin = 1e-3 * dy;
    const double ylo = fmin(ya, yb) - margin, yhi = fmax(ya, yb) + margin;
    const double bsz = double(kBlock) * dy;
    const double flo = floor((ylo - g.origin[1]) / bsz);
    const double fhi = floor((yhi - g.origin[1]) / bsz);
    if (fhi < 0.0 || flo > double(nby - 1))
      return 0;
    lo = flo < 0.0 ? 0 : int(flo);
    hi = fhi > double(nby - 1) ? nby - 1 : int(fhi);
  }
  int cnt = 0;
  for (int byi = lo; byi <= hi; byi++) {
    const int by0 = byi * kBlock, nyb = min(kBlock, g.ny - by0);
    const double vy = g.origin[1] + double(by0) * dy;
    const double wy = g.origin[1] + double(by0 + nyb) * dy;
    int hmin, hmax;
    pb_hrange(g, vx, wx, vy, wy, c, s, hmin, hmax);
    if (h < hmin || h > hmax)
      continue;
    if (par_x) {
      const int jy = int(floor((p2y - vy) / dy));
      if (jy < 0 || jy >= nyb)
        continue;
    }
    if (emit && pos + cnt < kMaxBlocks)
      emit[pos + cnt] = (bxi << 16) | byi;
    cnt++;
  }
  return cnt;
}

#ifndef PB_FP_MINB
#define PB_FP_MINB 5
#endif
#ifndef PB_FP_ORDER
#define PB_FP_ORDER 0
#endif
#ifndef PB_FP_BATCH
#define PB_FP_BATCH 4 // staged cells whose loads are issued together (4 or 2)
#endif
template <int NQ, int EPI>
__global__ void __launch_bounds__(kLaneWarps * 32, PB_FP_MINB)
    pb_fp_lanes(Geom g, const float *__restrict__ vol, float *__restrict__ pix, Epi e, int v0,
                int *err) {
  extern __shared__ unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  LaneSmem &S = reinterpret_cast<LaneSmem *>(smem_raw)[wib];
  const double eps = double(kEps);
  const double dx = g.size[0], dy = g.size[1];
  const int nbx = (g.nx + kBlock - 1) / kBlock;
  const int ncol = g.nx * g.ny;
  const unsigned nz4 = unsigned(g.nz) >> 2;
  // this lane's rows v0 + q*128 + 4*lane .. +3 of column 0, as float4
  const float4 *vb = reinterpret_cast<const float4 *>(vol) + (v0 >> 2) + lane;
  bool vok[NQ];
  int vq[NQ];
#pragma unroll
  for (int q = 0; q < NQ; q++) {
    vq[q] = v0 + q * 128 + lane * 4;
    vok[q] = vq[q] < g.nv;
  }
  double ssq = 0.0;
  const int nat = (g.na + kLaneWarps - 1) / kLaneWarps;
  const int ntiles = nat * g.nh;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
#if PB_FP_ORDER == 1
    // angle groups slow, detector columns fast: the resident CTAs trace
    // near-parallel rays that advance through the same block columns
    // together, so the volume strip they read stays in L2
    const int ag = t / g.nh;
    const int h = t - ag * g.nh;
    const int a = ag * kLaneWarps + wib;
#else
    const int h = t / nat;
    const int a = (t - h * nat) * kLaneWarps + wib;
#endif
    if (a >= g.na)
      continue;
    const int ray = a * g.nh + h;
    const double c = g.cosA[a], s = g.sinA[a], hv = g.hpix[h];
    const double p2x = c * g.det_x - s * hv;
    const double p2y = s * g.det_x + c * hv;
    const bool par_y = fabs(c) < eps, par_x = !par_y && fabs(s) < eps;
    float4 acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++)
      acc[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!(par_y && fabs(s) < eps)) {
      // ---- enumerate the blocks: x-block major, y-block ascending
      int nblk = 0;
      for (int bbase = 0; bbase < nbx; bbase += 32) {
        const int bxi = bbase + lane;
        const int cnt =
            bxi < nbx ? pb_column_blocks(g, h, c, s, p2x, p2y, par_y, par_x, bxi, nullptr, 0) : 0;
        int incl = cnt;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o)
            incl += y;
        }
        if (cnt)
          pb_column_blocks(g, h, c, s, p2x, p2y, par_y, par_x, bxi, S.blk, nblk + incl - cnt);
        nblk += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (nblk > kMaxBlocks) {
        if (lane == 0)
          atomicExch(err, 3);
        nblk = kMaxBlocks;
      }
      __syncwarp();
      const double ic = par_y ? 0.0 : 1.0 / c, is = par_x ? 0.0 : 1.0 / s;
      const int sx = c > 0.0 ? 1 : -1, sy = s > 0.0 ? 1 : -1;
      const int ox = sx > 0 ? 1 : 0, oy = sy > 0 ? 1 : 0;
      const bool x_face_first = !(sx > 0 && sy < 0);
      // ---- walk kWalkLanes blocks at a time, one per lane
      for (int r0 = 0; r0 < nblk; r0 += kWalkLanes) {
        const int j = r0 + lane;
        int n = 0;
        uint2 *myc = S.cell + (lane % kWalkLanes) * kSlotCap;
        auto put = [&](int col, float len) {
          if (unsigned(col) < unsigned(ncol))
            myc[n++] = make_uint2(unsigned(col) * nz4, __float_as_uint(len));
        };
        if (lane < kWalkLanes && j < nblk) {
          const int id = S.blk[j];
          const int bxi = id >> 16, byi = id & 0xffff;
          const int bx0 = bxi * kBlock, nxb = min(kBlock, g.nx - bx0);
          const int by0 = byi * kBlock, nyb = min(kBlock, g.ny - by0);
          const double vx = g.origin[0] + double(bx0) * dx;
          const double vy = g.origin[1] + double(by0) * dy;
          if (par_y) {
            const int ix = int(floor((p2x - vx) / dx));
            const float len = float(dy);
            for (int tt = 0; tt < nyb; tt++) {
              const int jj = s < 0.0 ? nyb - 1 - tt : tt;
              put((bx0 + ix) * g.ny + by0 + jj, len);
            }
          } else if (par_x) {
            const int jy = int(floor((p2y - vy) / dy));
            const float len = float(dx);
            for (int tt = 0; tt < nxb; tt++) {
              const int ii = c < 0.0 ? nxb - 1 - tt : tt;
              put((bx0 + ii) * g.ny + by0 + jy, len);
            }
          } else {
            const double xn = vx + double(nxb) * dx, yn = vy + double(nyb) * dy;
            const double ax0 = (vx - p2x) * ic, ay0 = (vy - p2y) * is;
            const double axn = (xn - p2x) * ic, ayn = (yn - p2y) * is;
            const double amin =
                dmax(dmax(dmin(ax0, axn), dmin(ay0, ayn)), double(-g.d_conv));
            const double amax = dmin(dmin(dmax(ax0, axn), dmax(ay0, ayn)), 0.0);
            if (amin < amax - eps) {
              int x = 0, y = 0;
              const double axe = sx > 0 ? ax0 : axn, aye = sy > 0 ? ay0 : ayn;
              if (x_face_first) {
                if (amin == axe) {
                  x = sx > 0 ? 0 : nxb - 1;
                  y = (sx < 0 && sy < 0 && amin == ayn)
                          ? nyb - 1
                          : int(floor((p2y + amin * s - vy) / dy));
                } else if (amin == aye) {
                  x = int(floor((p2x + amin * c - vx) / dx));
                  y = sy > 0 ? 0 : nyb - 1;
                }
              } else {
                if (amin == aye) {
                  x = int(floor((p2x + amin * c - vx) / dx));
                  y = nyb - 1;
                } else if (amin == axe) {
                  x = 0;
                  y = int(floor((p2y + amin * s - vy) / dy));
                }
              }
              double nxa = (vx + double(x + ox) * dx - p2x) * ic;
              double nya = (vy + double(y + oy) * dy - p2y) * is;
              double ap = amin;
              int col = (bx0 + x) * g.ny + (by0 + y);
              const int cstep_x = sx * g.ny;
              while ((sx > 0 ? x < nxb : x >= 0) && (sy > 0 ? y < nyb : y >= 0) &&
                     n < kSlotCap) {
                const bool tx = nxa < nya - eps;
                const bool ty = !tx && (nya < nxa - eps);
                const bool both = !tx && !ty;
                const double nxt = tx ? nxa : (ty ? nya : dmax(nxa, nya));
                put(col, float(nxt - ap));
                ap = nxt;
                if (tx || both) {
                  x += sx;
                  col += cstep_x;
                  nxa = (vx + double(x + ox) * dx - p2x) * ic;
                }
                if (ty || both) {
                  y += sy;
                  col += sy;
                  nya = (vy + double(y + oy) * dy - p2y) * is;
                }
              }
              if (n >= kSlotCap && (sx > 0 ? x < nxb : x >= 0) && (sy > 0 ? y < nyb : y >= 0))
                atomicExch(err, 3); // slot full before the ray left the block
            }
          }
        }
        __syncwarp();
        // ---- replay the slots in block order, lanes over rows
        const int nr = min(kWalkLanes, nblk - r0);
        for (int jj = 0; jj < nr; jj++) {
          const int nj = __shfl_sync(0xffffffffu, n, jj);
          const uint2 *cl = S.cell + jj * kSlotCap;
          int m = 0;
#if PB_FP_BATCH == 4
          for (; m + 4 <= nj; m += 4) {
            const uint4 p0 = *reinterpret_cast<const uint4 *>(cl + m);
            const uint4 p1 = *reinterpret_cast<const uint4 *>(cl + m + 2);
            const unsigned o[4] = {p0.x, p0.z, p1.x, p1.z};
            const float l[4] = {__uint_as_float(p0.y), __uint_as_float(p0.w),
                                __uint_as_float(p1.y), __uint_as_float(p1.w)};
#else
          for (; m + 2 <= nj; m += 2) {
            const uint4 p0 = *reinterpret_cast<const uint4 *>(cl + m);
            const unsigned o[2] = {p0.x, p0.z};
            const float l[2] = {__uint_as_float(p0.y), __uint_as_float(p0.w)};
#endif
            if (EPI == EPI_ONES) {
              (void)o;
#pragma unroll
              for (int u = 0; u < PB_FP_BATCH; u++)
#pragma unroll
                for (int q = 0; q < NQ; q++)
                  if (vok[q])
                    add_len4(acc[q], l[u]);
            } else {
              float4 xv[PB_FP_BATCH][NQ];
#pragma unroll
              for (int u = 0; u < PB_FP_BATCH; u++)
#pragma unroll
                for (int q = 0; q < NQ; q++)
                  if (vok[q])
                    xv[u][q] = __ldg(vb + o[u] + q * 32);
#pragma unroll
              for (int u = 0; u < PB_FP_BATCH; u++)
#pragma unroll
                for (int q = 0; q < NQ; q++)
                  if (vok[q])
                    axpy4(acc[q], xv[u][q], l[u]);
            }
          }
          for (; m < nj; m++) {
            const uint2 p = cl[m];
#pragma unroll
            for (int q = 0; q < NQ; q++)
              if (vok[q]) {
                if (EPI == EPI_ONES)
                  add_len4(acc[q], __uint_as_float(p.y));
                else
                  axpy4(acc[q], __ldg(vb + p.x + q * 32), __uint_as_float(p.y));
              }
          }
        }
        __syncwarp();
      }
    }
    const i64 rbase = i64(ray) * g.nv;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      if (vok[q]) {
        const int v = vq[q];
        float4 o;
        o.x = fp_epilogue<EPI>(acc[q].x, rbase + v + 0, e, ssq);
        o.y = fp_epilogue<EPI>(acc[q].y, rbase + v + 1, e, ssq);
        o.z = fp_epilogue<EPI>(acc[q].z, rbase + v + 2, e, ssq);
        o.w = fp_epilogue<EPI>(acc[q].w, rbase + v + 3, e, ssq);
        *reinterpret_cast<float4 *>(pix + rbase + v) = o;
      }
    }
  }
  if (EPI == EPI_NORM)
    store_partial<kLaneWarps>(ssq, e, v0 > 0);
}

// ---- forward, any row->slice mapping (p2D.cpp:63-213 cases 2, 4, default)
template <int NS, int EPI>
__global__ void __launch_bounds__(kFpWarps * 32) pb_fp_scalar(Geom g, const float *__restrict__ vol,
                                                              float *__restrict__ pix, Epi e, int v0) {
  __shared__ Cell lists[kFpWarps][kListCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  Cell *L = lists[wib];
  double ssq = 0.0;
  int zmap[NS];
#pragma unroll
  for (int q = 0; q < NS; q++) {
    const int v = v0 + q * 32 + lane;
    zmap[q] = (v < g.nv) ? g.map[v] : -1;
    if (zmap[q] >= g.nz)
      zmap[q] = -1; // the reference reads past the column here
  }
  const int nat = (g.na + kFpWarps - 1) / kFpWarps;
  const int ntiles = nat * g.nh;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int h = t / nat;
    const int a = (t - h * nat) * kFpWarps + wib;
    if (a >= g.na)
      continue;
    const int ray = a * g.nh + h;
    float acc[NS];
#pragma unroll
    for (int q = 0; q < NS; q++)
      acc[q] = 0.f;
    int n = 0;
    auto flush = [&]() {
      __syncwarp();
      for (int m = 0; m < n; m++) {
        const Cell c1 = L[m];
        if (c1.col < 0)
          continue;
        const float *colp = vol + i64(c1.col) * g.nz;
#pragma unroll
        for (int q = 0; q < NS; q++)
          if (zmap[q] >= 0)
            acc[q] = __fadd_rn(acc[q], __fmul_rn(__ldg(colp + zmap[q]), c1.len));
      }
      __syncwarp();
      n = 0;
    };
    auto emit = [&](int col, float len) {
      if (lane == 0)
        L[n] = Cell{col, len};
      n++;
    };
    auto room = [&]() {
      if (n > kListCap - kBlockCells)
        flush();
    };
    pb_trace_ray(g, a, h, emit, room);
    flush();
    const i64 rbase = i64(ray) * g.nv;
#pragma unroll
    for (int q = 0; q < NS; q++) {
      const int v = v0 + q * 32 + lane;
      if (v < g.nv)
        pix[rbase + v] = fp_epilogue<EPI>(acc[q], rbase + v, e, ssq);
    }
  }
  if (EPI == EPI_NORM)
    store_partial<kFpWarps>(ssq, e, v0 > 0);
}

// ---- backward
constexpr int kBpAngles = 16; // angles staged per pass
constexpr int kBpMaxRays = 8; // detector columns per (voxel column, angle)

struct BpEntry {
  int h0, cnt; // first detector column and number of rays; row index = a * nh + h0
  float w[kBpMaxRays];
};

// Detector columns and chord weights of voxel column [x0,xn) x [y0,yn) at
// angle a (bproject_ah, p2D.cpp:803-939).  Returns the count, or -1 when it
// exceeds the staging capacity (reported as an error by the host).
__device__ int pb_bp_rays(const Geom &g, double x0, double xn, double y0, double yn,
                          int a, BpEntry &E) {
  const double eps = double(kEps);
  const double c = g.cosA[a], s = g.sinA[a];
  int cnt = 0;
  E.h0 = 0;
  if (fabs(c) < eps || fabs(s) < eps) {
    int hmin, hmax;
    pb_hrange(g, x0, xn, y0, yn, c, s, hmin, hmax);
    const bool par_y = fabs(c) < eps;
    const double lo = par_y ? x0 : y0, hi = par_y ? xn : yn;
    const bool neg = par_y ? !(s < 0.0) : (c < 0.0);
    const float wt = float(par_y ? g.size[1] : g.size[0]);
    for (int h = hmin; h <= hmax; h++) {
      const double u = neg ? -g.hpix[h] : g.hpix[h];
      if (u >= lo && u < hi) {
        if (cnt == 0)
          E.h0 = h;
        else if (h != E.h0 + cnt)
          return -1; // not contiguous: cannot happen for monotone pixels
        if (cnt >= kBpMaxRays)
          return -1;
        E.w[cnt++] = wt;
      }
    }
    return cnt;
  }
  double ymin, ymax;
  if (c > 0.0) {
    if (s > 0.0) {
      ymin = y0 * c - xn * s;
      ymax = yn * c - x0 * s;
    } else {
      ymin = y0 * c - x0 * s;
      ymax = yn * c - xn * s;
    }
  } else {
    if (s > 0.0) {
      ymin = yn * c - xn * s;
      ymax = y0 * c - x0 * s;
    } else {
      ymin = yn * c - x0 * s;
      ymax = y0 * c - xn * s;
    }
  }
  const int hmin = (ymin < g.hpix[0]) ? 0 : int(floor(ymin * g.ihp - g.hp0));
  const int hmax = min(int(floor(ymax * g.ihp - g.hp0)), g.nh - 1);
  const double ybot = ymin + g.yoff[a], ytop = ymax - g.yoff[a];
  const double l = g.blen[a], io = g.ioff[a];
  for (int h = hmin; h <= hmax; h++) {
    if (h < 0)
      continue;
    const double hv = g.hpix[h];
    if (!(hv > ymin + eps))
      continue;
    float wt;
    if (hv < ybot)
      wt = float(l * (hv - ymin) * io);
    else if (hv <= ytop)
      wt = float(l);
    else if (hv < ymax - eps)
      wt = float(l * (ymax - hv) * io);
    else
      break;
    if (cnt == 0)
      E.h0 = h;
    if (cnt >= kBpMaxRays)
      return -1;
    E.w[cnt++] = wt;
  }
  return cnt;
}

template <int EPI>
__device__ __forceinline__ float bp_epilogue(float acc, i64 idx, const Epi &e, double &ssq) {
  if (EPI == EPI_NORM) {
    ssq += double(acc) * double(acc);
    return acc;
  } else if (EPI == EPI_SIRT) {
    // sirt.cpp:70-74: bp *= C; x += 1 * bp; x = max(x, 0)
    const float v = __fadd_rn(e.x[idx], __fmul_rn(1.0f, __fmul_rn(acc, e.w[idx])));
    return (v < 0.0f) ? 0.0f : v;
  } else if (EPI == EPI_MLEM) {
    // mlem.cpp:72-74: x *= (N * bp); x = max(x, 0)
    const float v = __fmul_rn(e.x[idx], __fmul_rn(e.w[idx], acc));
    return (v < 0.0f) ? 0.0f : v;
  }
  return acc;
}

// Stage the ray lists of this CTA's columns for angles [a0, a0 + kBpAngles).
__device__ void pb_bp_stage(const Geom &g, int tx0, int ty0, int tw, int th, int a0,
                            BpEntry *ent, int *err) {
  const int ncol = tw * th;
  for (int t = threadIdx.x; t < ncol * kBpAngles; t += blockDim.x) {
    const int col = t / kBpAngles, ai = t - col * kBpAngles;
    const int a = a0 + ai;
    BpEntry E;
    E.cnt = 0;
    E.h0 = 0;
    const int i = tx0 + col / th, j = ty0 + col % th;
    if (a < g.na && i < g.nx && j < g.ny) {
      const double x0 = g.origin[0] + double(i) * g.size[0];
      const double xn = g.origin[0] + double(i + 1) * g.size[0];
      const double y0 = g.origin[1] + double(j) * g.size[1];
      const double yn = g.origin[1] + double(j + 1) * g.size[1];
      const int n = pb_bp_rays(g, x0, xn, y0, yn, a, E);
      if (n < 0) {
        atomicExch(err, 1);
        E.cnt = 0;
      } else
        E.cnt = n;
    }
    ent[t] = E;
  }
}

// Vector over z (row v == slice z): each thread owns NP (column, group)
// pairs of VW = 16, 8 or 4 slices (four, two or one float4); groups are the fastest index so
// the lanes of a warp share a column and read its staged rays as
// broadcasts.  Group k holds float4 k, k + nzg, ... of the column (nzg =
// nz / VW groups), so each load instruction of a warp covers one contiguous
// 512-byte run of the sinogram row.
template <int NP, int VW, int EPI>
__global__ void __launch_bounds__(256, NP * VW <= 16 ? 4 : (NP * VW <= 32 ? 3 : 1)) pb_bp_vec(Geom g, const float *__restrict__ pix,
                                                 float *__restrict__ vol, Epi e, int tw, int th,
                                                 int *err) {
  extern __shared__ BpEntry ent[];
  constexpr int NF = VW / 4;
  const int ntx = (g.nx + tw - 1) / tw;
  const int tx0 = (blockIdx.x % ntx) * tw, ty0 = (blockIdx.x / ntx) * th;
  const int nzg = g.nz / VW;
  const int npairs = tw * th * nzg;
  const int fstride = 4 * nzg; // floats between a group's float4s
  float4 acc[NP][NF];
  int pcol[NP], pz[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) {
#pragma unroll
    for (int f = 0; f < NF; f++)
      acc[k][f] = make_float4(0.f, 0.f, 0.f, 0.f);
    const int p = threadIdx.x + k * blockDim.x;
    pcol[k] = (p < npairs) ? p / nzg : -1;
    pz[k] = (p < npairs) ? (p - (p / nzg) * nzg) * 4 : 0;
  }
  for (int a0 = 0; a0 < g.na; a0 += kBpAngles) {
    __syncthreads();
    pb_bp_stage(g, tx0, ty0, tw, th, a0, ent, err);
    __syncthreads();
    const int na_chunk = min(kBpAngles, g.na - a0);
#pragma unroll
    for (int k = 0; k < NP; k++) {
      if (pcol[k] < 0)
        continue;
      const BpEntry *E = ent + pcol[k] * kBpAngles;
      const float *base = pix + pz[k];
      for (int ai = 0; ai < na_chunk; ai++) {
        const int cnt = E[ai].cnt;
        const int row0 = (a0 + ai) * g.nh + E[ai].h0;
        for (int r = 0; r < cnt; r++) {
          const float w = E[ai].w[r];
          const float4 *p = reinterpret_cast<const float4 *>(base + i64(row0 + r) * g.nv);
          if (EPI == EPI_ONES) {
            (void)p;
#pragma unroll
            for (int f = 0; f < NF; f++)
              add_len4(acc[k][f], w);
          } else {
            float4 x[NF];
#pragma unroll
            for (int f = 0; f < NF; f++)
              x[f] = __ldg(p + f * nzg);
#pragma unroll
            for (int f = 0; f < NF; f++)
              axpy4_pa(acc[k][f], x[f], w);
          }
        }
      }
    }
  }
  double ssq = 0.0;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    if (pcol[k] < 0)
      continue;
    const int i = tx0 + pcol[k] / th, j = ty0 + pcol[k] % th;
    if (i >= g.nx || j >= g.ny)
      continue;
    const i64 base = (i64(i) * g.ny + j) * g.nz + pz[k];
#pragma unroll
    for (int f = 0; f < NF; f++) {
      float4 o;
      const i64 at = base + i64(f) * fstride;
      o.x = bp_epilogue<EPI>(acc[k][f].x, at + 0, e, ssq);
      o.y = bp_epilogue<EPI>(acc[k][f].y, at + 1, e, ssq);
      o.z = bp_epilogue<EPI>(acc[k][f].z, at + 2, e, ssq);
      o.w = bp_epilogue<EPI>(acc[k][f].w, at + 3, e, ssq);
      *reinterpret_cast<float4 *>(vol + at) = o;
    }
  }
  if (EPI == EPI_NORM)
    store_partial<8>(ssq, e);
}

// Scalar over z, any row->slice mapping (calc_ah_z cases, p2D.cpp:613-773).
template <int NP, int EPI>
__global__ void __launch_bounds__(256) pb_bp_scalar(Geom g, const float *__restrict__ pix,
                                                    float *__restrict__ vol, Epi e, int tw,
                                                    int th, int *err) {
  extern __shared__ BpEntry ent[];
  const int ntx = (g.nx + tw - 1) / tw;
  const int tx0 = (blockIdx.x % ntx) * tw, ty0 = (blockIdx.x / ntx) * th;
  const int npairs = tw * th * g.nz;
  float acc[NP];
  int pcol[NP], pz[NP];
#pragma unroll
  for (int k = 0; k < NP; k++) {
    acc[k] = 0.f;
    const int p = threadIdx.x + k * blockDim.x;
    pcol[k] = (p < npairs) ? p / g.nz : -1;
    pz[k] = (p < npairs) ? p - (p / g.nz) * g.nz : 0;
  }
  for (int a0 = 0; a0 < g.na; a0 += kBpAngles) {
    __syncthreads();
    pb_bp_stage(g, tx0, ty0, tw, th, a0, ent, err);
    __syncthreads();
    const int na_chunk = min(kBpAngles, g.na - a0);
#pragma unroll
    for (int k = 0; k < NP; k++) {
      if (pcol[k] < 0)
        continue;
      const int z = pz[k];
      const BpEntry *E = ent + pcol[k] * kBpAngles;
      for (int ai = 0; ai < na_chunk; ai++) {
        const int cnt = E[ai].cnt;
        const float *row = pix + (i64(a0 + ai) * g.nh + E[ai].h0) * g.nv;
        for (int r = 0; r < cnt; r++) {
          const float w = E[ai].w[r];
          const float *p = row + i64(r) * g.nv;
          switch (g.map_type) {
          case 1:
            if (z < g.nv)
              acc[k] = __fadd_rn(acc[k], __fmul_rn(p[z], w));
            break;
          case 2:
            if (2 * z + 1 < g.nv)
              acc[k] = __fadd_rn(acc[k], __fmul_rn(__fadd_rn(p[2 * z], p[2 * z + 1]), w));
            break;
          case 4:
            if (4 * z + 3 < g.nv) {
              const float t = __fadd_rn(__fadd_rn(__fadd_rn(p[4 * z], p[4 * z + 1]), p[4 * z + 2]),
                                        p[4 * z + 3]);
              acc[k] = __fadd_rn(acc[k], __fmul_rn(t, w));
            }
            break;
          default:
            for (int v = g.vlo[z]; v < g.vhi[z]; v++)
              acc[k] = __fadd_rn(acc[k], __fmul_rn(p[v], w));
            break;
          }
        }
      }
    }
  }
  double ssq = 0.0;
#pragma unroll
  for (int k = 0; k < NP; k++) {
    if (pcol[k] < 0)
      continue;
    const int i = tx0 + pcol[k] / th, j = ty0 + pcol[k] % th;
    if (i >= g.nx || j >= g.ny)
      continue;
    const i64 idx = (i64(i) * g.ny + j) * g.nz + pz[k];
    vol[idx] = bp_epilogue<EPI>(acc[k], idx, e, ssq);
  }
  if (EPI == EPI_NORM)
    store_partial<8>(ssq, e);
}

// The lane-parallel forward kernel applies: row v <-> slice v, float4 rows,
// float4 offsets of the columns fit 32 bits, and a ray's block list (at most
// about nbx + nby entries) fits its staging area.
bool pb_fp_vec4(const Geom &g) {
  const int nblocks = (g.nx + kBlock - 1) / kBlock + (g.ny + kBlock - 1) / kBlock;
  return g.map_type == 1 && (g.nv % 4) == 0 && (g.nz % 4) == 0 &&
         (long long)g.nx * g.ny * (g.nz / 4) < (1ll << 32) && nblocks + 16 <= kMaxBlocks;
}

template <int EPI>
int launch_fp(const Geom &g, const float *vol, float *pix, const Epi &e, int grid, int *err,
              cudaStream_t st) {
  if (pb_fp_vec4(g)) {
    const size_t smem = sizeof(LaneSmem) * kLaneWarps;
    for (int v0 = 0; v0 < g.nv; v0 += 256) {
      if (g.nv - v0 > 128)
        pb_fp_lanes<2, EPI><<<grid, kLaneWarps * 32, smem, st>>>(g, vol, pix, e, v0, err);
      else
        pb_fp_lanes<1, EPI><<<grid, kLaneWarps * 32, smem, st>>>(g, vol, pix, e, v0, err);
    }
  } else if (EPI != EPI_ONES) {
    for (int v0 = 0; v0 < g.nv; v0 += 256) {
      const int left = g.nv - v0;
      if (left > 128)
        pb_fp_scalar<8, EPI><<<grid, kFpWarps * 32, 0, st>>>(g, vol, pix, e, v0);
      else if (left > 32)
        pb_fp_scalar<4, EPI><<<grid, kFpWarps * 32, 0, st>>>(g, vol, pix, e, v0);
      else
        pb_fp_scalar<1, EPI><<<grid, kFpWarps * 32, 0, st>>>(g, vol, pix, e, v0);
    }
  }
  return 0;
}

#ifndef PB_BP_VW16
#define PB_BP_VW16 1 // 16 slices per (column, group) pair when nz % 16 == 0
#endif
#ifndef PB_BP_VW32
#define PB_BP_VW32 0 // 32 slices per pair when nz % 32 == 0
#endif

// Column tile and pairs per thread for the back projector: enough
// (column, slice group) pairs to fill 256 threads, at most 16 per thread.
struct BpShape {
  int vw, tw, th, np;
};

BpShape bp_shape(const Geom &g) {
  BpShape b;
  b.vw = 1;
  if (g.map_type == 1 && g.nv == g.nz) {
    if ((g.tune_vw == 4 || g.tune_vw == 8 || g.tune_vw == 16) && g.nz % g.tune_vw == 0)
      b.vw = g.tune_vw;
    else if (PB_BP_VW32 && g.nz % 32 == 0)
      b.vw = 32;
    else if (PB_BP_VW16 && g.nz % 16 == 0)
      b.vw = 16;
    else if (g.nz % 8 == 0)
      b.vw = 8;
    else if (g.nz % 4 == 0)
      b.vw = 4;
  }
  const int per_col = g.nz / b.vw;
  b.tw = 4;
  b.th = 4;
  if (per_col * 16 < 256) {
    b.tw = 8;
    b.th = per_col * 32 >= 256 ? 4 : 8;
  }
  b.np = (b.tw * b.th * per_col + 255) / 256;
  while (b.np > (b.vw >= 8 ? 8 : 16) && b.tw * b.th > 1) {
    if (b.tw >= b.th)
      b.tw = (b.tw + 1) / 2;
    else
      b.th = (b.th + 1) / 2;
    b.np = (b.tw * b.th * per_col + 255) / 256;
  }
  return b;
}

template <int EPI, int NP>
int launch_bp_np(const Geom &g, const BpShape &b, const float *pix, float *vol, const Epi &e,
                 int *err, cudaStream_t st) {
  const int tiles = ((g.nx + b.tw - 1) / b.tw) * ((g.ny + b.th - 1) / b.th);
  const size_t smem = sizeof(BpEntry) * b.tw * b.th * kBpAngles;
  if (PB_BP_VW32 && b.vw == 32)
    pb_bp_vec<NP, PB_BP_VW32 ? 32 : 16, EPI><<<tiles, 256, smem, st>>>(g, pix, vol, e, b.tw,
                                                                        b.th, err);
  else if (b.vw == 16)
    pb_bp_vec<NP, 16, EPI><<<tiles, 256, smem, st>>>(g, pix, vol, e, b.tw, b.th, err);
  else if (b.vw == 8)
    pb_bp_vec<NP, 8, EPI><<<tiles, 256, smem, st>>>(g, pix, vol, e, b.tw, b.th, err);
  else if (b.vw == 4)
    pb_bp_vec<NP, 4, EPI><<<tiles, 256, smem, st>>>(g, pix, vol, e, b.tw, b.th, err);
  else if (EPI != EPI_ONES)
    pb_bp_scalar<NP, EPI><<<tiles, 256, smem, st>>>(g, pix, vol, e, b.tw, b.th, err);
  return 0;
}

template <int EPI>
int launch_bp(const Geom &g, const float *pix, float *vol, const Epi &e, int *err,
              cudaStream_t st) {
  const BpShape b = bp_shape(g);
  if (b.np > 16)
    return 2; // more than 4096 slices per column: not supported
  if (b.np <= 1)
    return launch_bp_np<EPI, 1>(g, b, pix, vol, e, err, st);
  if (b.np <= 2)
    return launch_bp_np<EPI, 2>(g, b, pix, vol, e, err, st);
  if (b.np <= 4)
    return launch_bp_np<EPI, 4>(g, b, pix, vol, e, err, st);
  if (b.np <= 8)
    return launch_bp_np<EPI, 8>(g, b, pix, vol, e, err, st);
  if (b.vw >= 8)
    return 2;
  return launch_bp_np<EPI, 16>(g, b, pix, vol, e, err, st);
}

} // namespace

int pb_forward(const Geom &g, const float *vol, float *pix, int mode, const Epi &e,
               int grid, int *err, cudaStream_t st) {
  switch (mode) {
  case EPI_ONES:
    if (!pb_fp_vec4(g))
      return 3; // no ones form for this geometry: the caller projects a ones volume
    return launch_fp<EPI_ONES>(g, vol, pix, e, grid, err, st);
  case EPI_STORE:
    return launch_fp<EPI_STORE>(g, vol, pix, e, grid, err, st);
  case EPI_NORM:
    return launch_fp<EPI_NORM>(g, vol, pix, e, grid, err, st);
  case EPI_SIRT:
    return launch_fp<EPI_SIRT>(g, vol, pix, e, grid, err, st);
  case EPI_MLEM:
    return launch_fp<EPI_MLEM>(g, vol, pix, e, grid, err, st);
  }
  return 1;
}

// Opt the forward kernels into their shared memory (done once, outside any
// graph capture).
int pb_prepare() {
  const int smem = int(sizeof(LaneSmem) * kLaneWarps);
  const void *fns[] = {(const void *)pb_fp_lanes<1, EPI_STORE>, (const void *)pb_fp_lanes<2, EPI_STORE>,
                       (const void *)pb_fp_lanes<1, EPI_NORM>,  (const void *)pb_fp_lanes<2, EPI_NORM>,
                       (const void *)pb_fp_lanes<1, EPI_SIRT>,  (const void *)pb_fp_lanes<2, EPI_SIRT>,
                       (const void *)pb_fp_lanes<1, EPI_MLEM>,  (const void *)pb_fp_lanes<2, EPI_MLEM>,
                       (const void *)pb_fp_lanes<1, EPI_ONES>,  (const void *)pb_fp_lanes<2, EPI_ONES>};
  for (const void *f : fns)
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return 1;
  return 0;
}

int pb_fp_ctas(const Geom &g) {
  const long long tiles = (long long)((g.na + kLaneWarps - 1) / kLaneWarps) * g.nh;
  return int(tiles < 148 * PB_FP_CTAS_PER_SM ? tiles : 148 * PB_FP_CTAS_PER_SM);
}

int pb_backward(const Geom &g, const float *pix, float *vol, int mode, const Epi &e,
                int *err, cudaStream_t st) {
  switch (mode) {
  case EPI_ONES:
    if (bp_shape(g).vw < 4)
      return 3; // no ones form for this geometry: the caller projects a ones sinogram
    return launch_bp<EPI_ONES>(g, pix, vol, e, err, st);
  case EPI_STORE:
    return launch_bp<EPI_STORE>(g, pix, vol, e, err, st);
  case EPI_NORM:
    return launch_bp<EPI_NORM>(g, pix, vol, e, err, st);
  case EPI_SIRT:
    return launch_bp<EPI_SIRT>(g, pix, vol, e, err, st);
  case EPI_MLEM:
    return launch_bp<EPI_MLEM>(g, pix, vol, e, err, st);
  }
  return 1;
}

int pb_bp_tiles(const Geom &g) {
  const BpShape b = bp_shape(g);
  return ((g.nx + b.tw - 1) / b.tw) * ((g.ny + b.th - 1) / b.th);
}

} // namespace ccpi
