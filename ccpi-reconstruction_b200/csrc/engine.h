// Internal engine interface shared by the C ABI (capi.cu) and engine.cu.
#pragma once

#include <string>
#include <vector>

#include "../../include/ccpi_b200.h"
#include "common.cuh"

struct ccpi_plan {
  ccpi::Geom g{};
  int device = 0;
  long long nvox = 0, npix = 0;
  int fp_grid = 1;  // CTAs of the forward projector (= its partial sums)
  int bp_parts = 1; // CTAs of the back projector (= its partial sums)
  int2 *hrange = nullptr; // cone: detector columns seeing the volume, per angle
  int *err = nullptr;     // device error flag set by the projectors
  std::vector<void *> bufs;
  ~ccpi_plan();
};

namespace ccpi {

extern thread_local std::string g_last_error;
void set_error(const std::string &m);
bool cuda_ok(cudaError_t e, const char *what);
// Streaming multiprocessors of the current device (148 on a B200).
int sm_count();

int plan_create(const ccpi_geometry *g, ccpi_plan **out);
int forward(const ccpi_plan *p, const float *vol, float *pix, int mode, const Epi &e,
            cudaStream_t st);
int backward(const ccpi_plan *p, const float *pix, float *vol, int mode, const Epi &e,
             cudaStream_t st);
// Pick the fastest launch shapes for this plan on scratch data; chosen (may
// be NULL) receives {forward grid or cone rows per lane, back projector
// slices per lane or 0}.
int plan_autotune(ccpi_plan *p, cudaStream_t st, int *chosen);
// Cone plans: 1 selects the ray-driven scatter back projector for the plain
// and norm forms, 0 the deterministic voxel gather (the default).
int set_cone_backprojector(ccpi_plan *p, int scatter);
size_t solve_workspace_bytes(const ccpi_plan *p, int alg, int niter);
int solve(const ccpi_plan *p, int alg, const float *sino, float *x, int niter, double lambda,
          double *h_norms, int flags, void *ws, size_t ws_bytes, cudaStream_t st);
void *session_create(const ccpi_plan *p, int alg, const float *sino, float *x, double lambda,
                     int max_iter, int flags, cudaStream_t st, int *rc);
int session_run(void *s, int n);
int session_finish(void *s, double *h_norms);
void session_destroy(void *s);
int solve_batched(int n, const ccpi_plan *const *plans, int alg, const float *const *sino,
                  float *const *x, int niter, const double *lambda, cudaStream_t st);
// z-sharded CGLS family (see engine.cu); stages as CCPI_SHARD_* in the C ABI
enum ShardStage { SHARD_SETUP = 0, SHARD_FORWARD = 1, SHARD_UPDATE = 2, SHARD_BACKWARD = 3,
                  SHARD_NEXT = 4 };
void *shard_create(const ccpi_plan *p, int alg, const float *sino, float *x, double lambda,
                   int max_iter, double *sum, float *edges, const float *halo_lo,
                   const float *halo_hi, cudaStream_t st, int *rc);
int shard_stage(void *s, int stage);
int shard_finish(void *s, double *h_norms);
void shard_destroy(void *s);
// AML ring-artefact filter on a device sinogram [angle][h][v], in place
// (aml.cu); synchronises st.
int aml_ring_filter(float *d_sino, int na, int nh, int nv, double param_n, double param_r,
                    int num_series, cudaStream_t st);
// High-peaks and column ring-artefact filters on a device sinogram
// [angle][h][v], in place (prefilter.cu); launched on st, not waited for.
int high_peaks_filter(float *d_sino, int na, int nh, int nv, double jump, int num_pix,
                      cudaStream_t st);
int column_ring_filter(float *d_sino, int na, int nh, int nv, cudaStream_t st);
// The high-peaks parameter checks alone (no CUDA call); 1 and an error
// message when jump < 0 or num_pix is outside [1, na).
int high_peaks_check(int na, double jump, int num_pix);

} // namespace ccpi
