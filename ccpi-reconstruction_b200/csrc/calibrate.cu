// Gather-bandwidth calibration for the projectors' roofline.
//
// The projectors' inner loops are gathers: every ray-cell visit reads one
// voxel column (nz floats, 1 KB at nz = 256) at a data-dependent offset,
// served from L2 and L1 rather than streamed from HBM.  Their ceiling is
// therefore the rate at which the SMs can pull whole columns at random out of
// an L2-resident working set, which this kernel measures: each warp reads
// 1 KB columns at hashed offsets, eight columns' loads in flight per lane.
// bench.py reports it beside the measured HBM copy bandwidth.  No
// counterpart in the reference.
#include <cstdint>

#include "../../include/ccpi_b200.h"
#include "engine.h"
#include "kernels.h"

namespace ccpi {
namespace {

constexpr int kCalThreads = 256;
constexpr int kCalBatch = 8;
constexpr int kCalPerWarp = 2048; // columns per warp per launch

__device__ __forceinline__ unsigned cal_hash(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Column c of the working set is float4s [64 c, 64 c + 64); lane l reads
// float4s l and l + 32 of it.  mask + 1 (a power of two) columns are
// allocated, c = hash & mask.
__global__ void __launch_bounds__(kCalThreads)
    gather_probe(const float4 *__restrict__ cols, unsigned mask, float *__restrict__ out) {
  const int lane = threadIdx.x & 31;
  const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0;
  for (int m = 0; m < kCalPerWarp; m += kCalBatch) {
    float4 x[kCalBatch][2];
#pragma unroll
    for (int u = 0; u < kCalBatch; u++) {
      const unsigned c = cal_hash(warp * kCalPerWarp + unsigned(m + u)) & mask;
      x[u][0] = __ldg(cols + size_t(c) * 64 + lane);
      x[u][1] = __ldg(cols + size_t(c) * 64 + 32 + lane);
    }
#pragma unroll
    for (int u = 0; u < kCalBatch; u++) {
      a0.x += x[u][0].x;
      a0.y += x[u][0].y;
      a0.z += x[u][0].z;
      a0.w += x[u][0].w;
      a1.x += x[u][1].x;
      a1.y += x[u][1].y;
      a1.z += x[u][1].z;
      a1.w += x[u][1].w;
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] =
      a0.x + a0.y + a0.z + a0.w + a1.x + a1.y + a1.z + a1.w;
}

} // namespace
} // namespace ccpi

extern "C" int ccpi_measure_gather(unsigned long long working_set_bytes, void *stream,
                                   double *gbs) {
  using namespace ccpi;
  g_last_error.clear();
  if (!gbs || working_set_bytes < 1024) {
    set_error("ccpi_measure_gather: need an output and a working set of >= 1 KB");
    return 1;
  }
  cudaStream_t st = cudaStream_t(stream);
  unsigned long long ncols = 1;
  while (ncols * 2 * 1024 <= working_set_bytes)
    ncols *= 2; // a power of two, so a mask picks the column
  if (ncols > 0x80000000ull) {
    set_error("ccpi_measure_gather: working set too large");
    return 1;
  }
  const unsigned mask = unsigned(ncols - 1);
  // four CTAs per SM of the current device (148 SMs on a B200)
  const int grid = sm_count() * 4;
  float4 *cols = nullptr;
  float *out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  if (!cuda_ok(cudaMalloc(&cols, ncols * 1024), "gather probe: working set") ||
      !cuda_ok(cudaMalloc(&out, size_t(grid) * kCalThreads * sizeof(float)), "gather probe") ||
      !cuda_ok(cudaMemsetAsync(cols, 0, ncols * 1024, st), "gather probe: clear") ||
      !cuda_ok(cudaEventCreate(&e0), "gather probe: event") ||
      !cuda_ok(cudaEventCreate(&e1), "gather probe: event"))
    rc = 2;
  const int reps = 3;
  if (rc == 0) {
    gather_probe<<<grid, kCalThreads, 0, st>>>(cols, mask, out); // warm-up
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; r++)
      gather_probe<<<grid, kCalThreads, 0, st>>>(cols, mask, out);
    cudaEventRecord(e1, st);
    float ms = 0.f;
    if (!cuda_ok(cudaEventSynchronize(e1), "gather probe") ||
        !cuda_ok(cudaEventElapsedTime(&ms, e0, e1), "gather probe: timing") || ms <= 0.f) {
      rc = 2;
    } else {
      const double bytes =
          double(reps) * grid * (kCalThreads / 32) * double(kCalPerWarp) * 1024.0;
      *gbs = bytes / (double(ms) * 1e-3) / 1e9;
    }
  }
  if (e0)
    cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
  cudaFree(cols);
  cudaFree(out);
  return rc;
}
