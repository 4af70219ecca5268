// ccpi_solve_noalloc: ccpi_solve for callers that must not allocate device
// memory during a solve.
//
// Who needs it: a host that owns every byte of device memory through its own
// pool (and forbids other allocations once it has reserved the device), or a
// latency-sensitive loop running other streams, where a cudaMalloc/cudaFree
// pair around each solve would add device-wide synchronisation.  ccpi_solve
// with d_workspace == NULL allocates and frees its workspace; this entry
// point instead uses a fixed scratch area compiled into the library.
//
// The scratch is a file-scope __device__ array of kStaticScratchBytes
// (16 MiB per device).  Its address is looked up once per device, on the
// first call on that device (cudaGetSymbolAddress; this may load the
// library's module), so make one call before any stream capture begins.
// Problems whose solver workspace exceeds the scratch are rejected with an
// error naming both sizes; ccpi_solve_workspace_bytes() gives the need.
// Nothing in the scratch has to start at zero: the solver initialises every
// buffer it uses.  The solve runs host-driven (the CCPI_SOLVE_PLAIN
// schedule), so no graph is instantiated.
//
// All calls on one device share the one scratch area: calls that overlap in
// time (from several host threads) race and corrupt each other's results.
// Each call is synchronous, so calls made one after another are safe.
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/ccpi_b200.h"
#include "engine.h"

namespace {

constexpr size_t kStaticScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_lock;

// Address of this device's scratch, looked up on the first call.
void *static_scratch(int device) {
  std::lock_guard<std::mutex> guard(g_setup_lock);
  if (!g_scratch_addr[device]) {
    void *p = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&p, g_static_scratch);
    if (rc != cudaSuccess) {
      ccpi::set_error(std::string("ccpi_solve_noalloc: static scratch lookup failed: ") +
                      cudaGetErrorString(rc));
      return nullptr;
    }
    g_scratch_addr[device] = p;
  }
  return g_scratch_addr[device];
}

} // namespace

extern "C" int ccpi_solve_noalloc(const ccpi_plan *plan, int alg, const float *d_sino,
                                  float *d_x, int niterations, double regularize,
                                  double *h_norms, void *stream) {
  ccpi::g_last_error.clear();
  if (!plan || !d_sino || !d_x) {
    ccpi::set_error("ccpi_solve_noalloc: null argument");
    return 1;
  }
  if ((reinterpret_cast<uintptr_t>(d_sino) | reinterpret_cast<uintptr_t>(d_x)) & 15u) {
    ccpi::set_error("ccpi_solve_noalloc: device buffers must be 16-byte aligned");
    return 1;
  }
  if (alg < CCPI_CGLS || alg > CCPI_CGLS_TV || niterations < 0) {
    ccpi::set_error("ccpi_solve_noalloc: unknown algorithm or negative iteration count");
    return 1;
  }
  const size_t need = ccpi::solve_workspace_bytes(plan, alg, niterations);
  if (need > kStaticScratchBytes) {
    ccpi::set_error("ccpi_solve_noalloc: this problem needs " + std::to_string(need) +
                    " bytes of solver scratch; the static scratch holds " +
                    std::to_string(kStaticScratchBytes) +
                    " bytes (use ccpi_solve with a workspace)");
    return 1;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
    ccpi::set_error("ccpi_solve_noalloc: no usable current device");
    return 2;
  }
  // the scratch used is the current device's: it must be the plan's device,
  // where the plan's tables and the caller's buffers live
  if (device != plan->device) {
    ccpi::set_error("ccpi_solve_noalloc: the current device (" + std::to_string(device) +
                    ") is not the plan's device (" + std::to_string(plan->device) +
                    "); make the plan's device current first");
    return 1;
  }
  void *scratch = static_scratch(device);
  if (!scratch)
    return 2;
  return ccpi::solve(plan, alg, d_sino, d_x, niterations, regularize, h_norms,
                     CCPI_SOLVE_PLAIN, scratch, kStaticScratchBytes, cudaStream_t(stream));
}
