// Sinogram pre-processing of the reference's Diamond (parallel-beam)
// pipeline, on the GPU: the high-peaks filter (CCPi::Diamond::
// high_peaks_before, Core/src/diamond.cpp:513-617) and the column
// ring-artefact filter (CCPi::remove_column_ring_artefacts,
// diamond.cpp:619-658).  The reference runs them on the -log sinogram after
// reading a data file (diamond.cpp:383-387); the AML ring filter, the third
// of this group, is in aml.cu.
//
// Both work on the internal sinogram layout [angle][h][v] and treat every
// detector element (h, v) as an independent series over the angles, so one
// thread owns one (h, v) column and walks the angles in order; consecutive
// threads own consecutive v, so every access of a warp is one contiguous run.
// The float and FP64 operations are the reference's, unfused (this file is
// compiled with --fmad=false; neither filter multiplies), in its order, so the
// results are the reference's bit for bit.
#include <algorithm>

#include "../../include/ccpi_b200.h"
#include "engine.h"
#include "kernels.h"

namespace ccpi {
namespace {

constexpr int kPfThreads = 256;

// The clamp of both high-peaks passes: a difference below -jump (compared in
// FP64, as the reference compares its float difference with the real jump)
// becomes float(-jump).
__device__ __forceinline__ float hp_clamp(float t, double neg_jump, float neg_jump_f) {
  return (double(t) < neg_jump) ? neg_jump_f : t;
}

// num_pix rounds of the high-peaks filter on every (h, v) series.  One round
// is the reference's top-to-bottom pass, q[a] = p[a+1] + clamp(p[a] - p[a+1])
// for a < na - 1 (q[na-1] = p[na-1]), then its bottom-to-top pass on q,
// r[a+1] = q[a] + clamp(q[a+1] - q[a]) (r[0] = q[0]).  Each pass reads only
// values from before it, so one streaming walk over the angles forms r with
// p[a+1] and q[a-1] held in registers, one read and one write per element.
__global__ void __launch_bounds__(kPfThreads)
    high_peaks_kernel(float *__restrict__ px, int na, i64 ncol, double neg_jump, float neg_jump_f,
                      int num_pix) {
  for (i64 c = blockIdx.x * i64(blockDim.x) + threadIdx.x; c < ncol;
       c += i64(gridDim.x) * blockDim.x) {
    float *col = px + c;
    for (int it = 0; it < num_pix; it++) {
      float p0 = col[0], qprev = 0.0f;
      for (int a = 0; a < na; a++) {
        float q = p0;
        if (a + 1 < na) {
          const float p1 = col[i64(a + 1) * ncol];
          q = __fadd_rn(p1, hp_clamp(__fsub_rn(p0, p1), neg_jump, neg_jump_f));
          p0 = p1;
        }
        const float r =
            a == 0 ? q : __fadd_rn(qprev, hp_clamp(__fsub_rn(q, qprev), neg_jump, neg_jump_f));
        col[i64(a) * ncol] = r;
        qprev = q;
      }
    }
  }
}

// Column ring filter: every series loses its angular mean, summed in FP64 in
// angle order, divided by the angle count and rounded to float once.
__global__ void __launch_bounds__(kPfThreads)
    column_ring_kernel(float *__restrict__ px, int na, i64 ncol) {
  for (i64 c = blockIdx.x * i64(blockDim.x) + threadIdx.x; c < ncol;
       c += i64(gridDim.x) * blockDim.x) {
    float *col = px + c;
    double acc = 0.0;
    for (int a = 0; a < na; a++)
      acc = __dadd_rn(acc, double(col[i64(a) * ncol]));
    const float m = __double2float_rn(__ddiv_rn(acc, double(na)));
    for (int a = 0; a < na; a++)
      col[i64(a) * ncol] = __fsub_rn(col[i64(a) * ncol], m);
  }
}

int pf_grid(i64 n) {
  const i64 b = (n + kPfThreads - 1) / kPfThreads;
  return int(std::min<i64>(std::max<i64>(b, 1), 148 * 16));
}

} // namespace

int high_peaks_check(int na, double jump, int num_pix) {
  // the reference's two checks (diamond.cpp:520-527); it reports them and
  // leaves the data as it is, here they are errors
  if (jump < 0.0) {
    set_error("high peaks filter: negative jump");
    return 1;
  }
  if (num_pix < 1 || num_pix >= na) {
    set_error("high peaks filter: the number of neighbours must be in [1, n_angles)");
    return 1;
  }
  return 0;
}

int high_peaks_filter(float *d_sino, int na, int nh, int nv, double jump, int num_pix,
                      cudaStream_t st) {
  if (!d_sino || na < 1 || nh < 1 || nv < 1) {
    set_error("high peaks filter: need a sinogram of >= 1 angle, column and row");
    return 1;
  }
  if (high_peaks_check(na, jump, num_pix))
    return 1;
  const i64 ncol = i64(nh) * nv;
  high_peaks_kernel<<<pf_grid(ncol), kPfThreads, 0, st>>>(d_sino, na, ncol, -jump, float(-jump),
                                                           num_pix);
  return cuda_ok(cudaGetLastError(), "high peaks filter") ? 0 : 2;
}

int column_ring_filter(float *d_sino, int na, int nh, int nv, cudaStream_t st) {
  if (!d_sino || na < 1 || nh < 1 || nv < 1) {
    set_error("column ring filter: need a sinogram of >= 1 angle, column and row");
    return 1;
  }
  const i64 ncol = i64(nh) * nv;
  column_ring_kernel<<<pf_grid(ncol), kPfThreads, 0, st>>>(d_sino, na, ncol);
  return cuda_ok(cudaGetLastError(), "column ring filter") ? 0 : 2;
}

} // namespace ccpi
