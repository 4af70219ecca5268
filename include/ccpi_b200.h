/* ccpi_b200.h -- C ABI of the B200-native CCPi iterative reconstruction path.
 *
 * One shared library (ccpi-reconstruction_b200/libccpi_b200.so) exports
 * everything below.  Signatures use plain pointers, sizes and doubles only;
 * CUDA streams are passed as `void *` (a cudaStream_t, NULL = the legacy
 * default stream).  Every entry point returns 0 on success and a nonzero
 * code on failure; ccpi_last_error() then holds a message (per thread).
 *
 * Layouts are the reference's:
 *   parallel-beam numpy sinogram  (n_angles, n_v, n_h), float32
 *   cone-beam numpy sinogram      (n_angles, n_h, n_v), float32
 *   internal / device sinogram    (n_angles, n_h, n_v), v fastest
 *   volume                        (nx, ny, nz), z fastest
 * Angles are degrees at the reference-facing calls (read as float32, as the
 * reference's wrappers read them) and radians in ccpi_geometry.
 */
#ifndef CCPI_B200_H
#define CCPI_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CCPI_CGLS = 0,
  CCPI_SIRT = 1,
  CCPI_MLEM = 2,
  CCPI_CGLS_TIKHONOV = 3,
  CCPI_CGLS_TV = 4
};

enum { CCPI_PARALLEL = 0, CCPI_CONE = 1 };

/* Solver flags. */
enum {
  CCPI_SOLVE_PLAIN = 1 /* host-driven loop, one launch sequence per
                          iteration, host reads the step scalars back every
                          iteration (no CUDA graph) */
};

/* Explicit projector geometry in the reference's frame
 * (Core/src/instruments.hpp:22-143): rays of detector column h and row v
 * at angle a; parallel beam uses h_pixels/v_pixels as detector coordinates,
 * cone beam places the source at `source` and the detector plane at
 * x = detector_x before rotation. */
typedef struct ccpi_geometry {
  int kind; /* CCPI_PARALLEL or CCPI_CONE */
  int n_angles, n_h, n_v;
  const double *angles;   /* n_angles, radians */
  const double *h_pixels; /* n_h, increasing, evenly spaced */
  const double *v_pixels; /* n_v, increasing, evenly spaced */
  double source[3];       /* cone beam only */
  double detector_x;      /* cone beam only */
  double origin[3];       /* corner of voxel (0, 0, 0) */
  double voxel_size[3];
  int nx, ny, nz;
} ccpi_geometry;

typedef struct ccpi_plan ccpi_plan; /* device tables for one geometry */

/* Message of the last failure on this thread ("" if none). */
const char *ccpi_last_error(void);
/* Library version as major * 10000 + minor * 100 + patch. */
int ccpi_version(void);

/* ---------------------------------------------------------------------
 * Reference-facing calls (host buffers in, host buffers out).
 * ------------------------------------------------------------------- */

/* Voxel grid the parallel-beam path derives from a sinogram shape.
 * Replaces Diamond::setup_experimental_geometry + calculate_block_sizes +
 * Diamond::get_xy_size (Core/src/diamond.cpp:35-86, :479-501,
 * Core/src/voxels.cpp:12-46).  dims = {nx, ny, nz, n_v_padded, v_offset}. */
int ccpi_pb_grid(int n_angles, int n_v, int n_h, double rotation_centre,
                 int pixels_per_voxel, int dims[5]);

/* The explicit geometry ccpi_pb_reconstruct derives from a sinogram shape
 * (the same front-end as ccpi_pb_grid: Core/src/diamond.cpp:35-86,
 * :479-501), for callers that keep their data on the device and use
 * ccpi_plan_create.  The caller provides angles_rad (n_angles),
 * h_pixels (n_h) and v_pixels (n_v_padded from ccpi_pb_grid); `geometry`
 * is filled and points into them. */
int ccpi_pb_geometry(int n_angles, int n_v, int n_h, const float *angles_deg,
                     double rotation_centre, int pixels_per_voxel,
                     double *angles_rad, double *h_pixels, double *v_pixels,
                     ccpi_geometry *geometry);

/* Device-side layout change of a parallel-beam sinogram: numpy layout
 * (n_angles, n_v, n_h) -> (n_angles, n_h, n_v_padded) with the data in
 * rows [v_offset, v_offset + n_v) and zeros elsewhere, as the reference's
 * Diamond::read_scans stores it (Core/src/diamond.cpp:394-451).
 * Asynchronous on `stream`. */
int ccpi_pb_pack(const float *d_pixels, int n_angles, int n_v, int n_h,
                 int n_v_padded, int v_offset, float *d_sino, void *stream);

/* parallelbeam.alg.{cgls,sirt,mlem,cgls_conv,cgls_tikhonov,cgls_TVreg}
 * and their *_step forms.  Replaces reconstruct_iter
 * (Wrappers/Python/src/diamond_wrapper.cpp:53-137; *_step: :140-257).
 * pixels: (n_angles, n_v, n_h); volume: nx*ny*nz floats (ccpi_pb_grid);
 * x0: NULL, or the previous volume for the *_step forms; norms: NULL or
 * niterations doubles receiving |A^T r| per iteration (CGLS family);
 * nthreads is accepted and ignored (the work runs on the current GPU). */
int ccpi_pb_reconstruct(int alg, const float *pixels, int n_angles, int n_v,
                        int n_h, const float *angles_deg,
                        double rotation_centre, int pixels_per_voxel,
                        int niterations, int nthreads, int is_pixels_in_log,
                        double regularize, const float *x0, double *norms,
                        float *volume);

/* n independent ccpi_pb_reconstruct problems of uneven sizes solved
 * together: one CUDA graph per iteration holds every problem's kernels.
 * The reference has no batched call; each problem i gives the same volume
 * as ccpi_pb_reconstruct(alg, pixels[i], na[i], nv[i], nh[i],
 * angles_deg[i], cor[i], pixels_per_voxel, niterations, -, is_log,
 * regularize[i], NULL, NULL, volumes[i]) (reconstruct_iter,
 * Wrappers/Python/src/diamond_wrapper.cpp:53-137, called n times).
 * regularize: NULL (all 0) or n weights; volumes[i]: ccpi_pb_grid's
 * nx*ny*nz floats for problem i. */
int ccpi_pb_reconstruct_batched(int n, int alg, const float *const *pixels,
                                const int *n_angles, const int *n_v,
                                const int *n_h, const float *const *angles_deg,
                                const double *rotation_centre,
                                int pixels_per_voxel, int niterations,
                                int is_pixels_in_log, const double *regularize,
                                float *const *volumes);

/* parallelbeam.filters.aml_ring_artefacts: the AML ring-artefact filter
 * (Wrappers/Python/src/diamond_wrapper.cpp:18-51 over
 * CCPi::remove_aml_ring_artefacts, Core/src/diamond.cpp:660-808).
 * pixels and out: (n_angles, n_v, n_h) transmission data; the filter runs
 * on -log(pixels) and out = exp(-filtered).  Parameters the reference
 * rejects (param_n < 0, param_r <= 0, num_series outside [1, 100]) are
 * errors. */
int ccpi_pb_aml_ring_artefacts(const float *pixels, int n_angles, int n_v,
                               int n_h, float param_n, float param_r,
                               int num_series, float *out);

/* The same filter on a device log sinogram in the internal layout
 * (n_angles, n_h, n_v), in place, on `stream` (the call waits for it). */
int ccpi_ring_filter_aml(float *d_sino, int n_angles, int n_h, int n_v,
                         double param_n, double param_r, int num_series,
                         void *stream);

/* The high-peaks filter of the reference's Diamond pre-processing
 * (CCPi::Diamond::high_peaks_before, Core/src/diamond.cpp:513-617; the
 * reference runs it on the -log sinogram when its configuration asks,
 * diamond.cpp:383-384, and has no Python call for it).  pixels and out:
 * (n_angles, n_v, n_h); with is_pixels_in_log == 0 they are transmission
 * (filtered as -log, returned as exp(-filtered)), else logs.  jump < 0 and
 * num_pix outside [1, n_angles) are errors (the reference prints them and
 * leaves the data unfiltered). */
int ccpi_pb_high_peaks(const float *pixels, int n_angles, int n_v, int n_h,
                       double jump, int num_pix, int is_pixels_in_log,
                       float *out);

/* The column ring-artefact filter (CCPi::remove_column_ring_artefacts,
 * Core/src/diamond.cpp:619-658, reached through the reference's
 * configuration, diamond.cpp:814-816): every detector element loses its
 * mean over the angles.  Layout and is_pixels_in_log as ccpi_pb_high_peaks. */
int ccpi_pb_column_ring_artefacts(const float *pixels, int n_angles, int n_v,
                                  int n_h, int is_pixels_in_log, float *out);

/* The two filters above on a device log sinogram in the internal layout
 * (n_angles, n_h, n_v), in place, launched on `stream` (not waited for). */
int ccpi_high_peaks(float *d_sino, int n_angles, int n_h, int n_v, double jump,
                    int num_pix, void *stream);
int ccpi_ring_filter_column(float *d_sino, int n_angles, int n_h, int n_v,
                            void *stream);

/* parallelbeam.alg.pb_forward_project (diamond_wrapper.cpp:421-556):
 * volume (vx, vy, vz) -> (n_angles, n_v_padded, max(vx, vy)).  With
 * out == NULL only out_dims is filled. */
int ccpi_pb_forward_project(const float *volume, int vx, int vy, int vz,
                            const float *angles_deg, int n_angles,
                            int resolution, float *out, int out_dims[3]);

/* parallelbeam.alg.pb_backward_project (diamond_wrapper.cpp:633-757):
 * stack (n_angles, n_v, n_h) -> volume on the ccpi_pb_grid grid. */
int ccpi_pb_backward_project(const float *stack, int n_angles, int n_v,
                             int n_h, const float *angles_deg,
                             double rotation_center, int resolution,
                             float *out, int out_dims[3]);

/* Voxel grid and detector of the cone-beam numpy path
 * (Core/src/Readers/xtek.cpp:57-129, :367-380, :760-798).
 * dims = {nx, ny, nz, n_v_padded, v_offset};
 * geom = {voxel size xy, voxel size z, origin x, y, z}. */
int ccpi_cb_grid(int n_angles, int n_h, int n_v, int pixels_per_voxel,
                 double source_to_sample, double source_to_detector,
                 double pixel_h_size, double pixel_v_size,
                 double mask_radius, int dims[5], double geom[5]);

/* Centre-of-rotation search of the cone-beam path (Nikon_XTek::find_centre,
 * xtek.cpp:671-758; T. Liu, Opt. Eng. 48(4) 046501, 2009) on the padded,
 * log sinogram (n_angles, n_h, n_v_padded) of ccpi_cb_grid's geometry.
 * Returns the source y offset the reference applies (*y_centre). */
int ccpi_cb_find_centre(const float *sino, int n_angles, int n_h,
                        int n_v_padded, const float *angles_deg,
                        double source_to_sample, double source_to_detector,
                        double pixel_h_size, double *y_centre);

/* conebeam.alg.{cgls,sirt,mlem,cgls_conv,cgls_tikhonov,cgls_TVreg}.
 * Replaces conebeam_reconstruct_iter
 * (Wrappers/Python/src/conebeam_wrapper.cpp:14-121).
 * pixels: (n_angles, n_h, n_v); volume: nx*ny*nz (ccpi_cb_grid). */
int ccpi_cb_reconstruct(int alg, const float *pixels, int n_angles, int n_h,
                        int n_v, const float *angles_deg,
                        int pixels_per_voxel, double source_to_sample,
                        double source_to_detector, double pixel_h_size,
                        double pixel_v_size, double mask_radius,
                        int niterations, int nthreads, int is_pixels_in_log,
                        double regularize, double *norms, float *volume);

/* conebeam.alg.create_sinogram (conebeam_wrapper.cpp:346-400): the cone
 * forward projection of an explicit geometry; out (n_angles, n_h, n_v). */
int ccpi_cb_create_sinogram(const ccpi_geometry *geometry,
                            const float *volume, float *out);

/* A solver on an explicit geometry with host buffers: the reference's core
 * call reconstruction_alg::reconstruct (Core/src/algorithms.hpp:13-20) on an
 * instrument whose geometry is set explicitly (as its Avizo and Matlab
 * front-ends do, Wrappers/Avizo/src/CCPiReconstruction/Cone_Beam_recon.cpp:
 * 114-180), followed by the clamp at zero of Core/src/voxels.cpp:187.
 * sino: (n_angles, n_h, n_v) log data; volume: nx*ny*nz floats (written);
 * norms: NULL or niter doubles (|A^T r| per CGLS-family iteration).  The
 * call uploads, solves on the current device and downloads; it blocks. */
int ccpi_reconstruct(const ccpi_geometry *geometry, int alg, const float *sino, int niter,
                     double regularize, double *norms, float *volume);

/* Flags of ccpi_reconstruct_flags. */
enum {
  CCPI_RECON_CONE_SCATTER = 1 /* cone beam: the CGLS family back-projects with
                                 the ray-driven scatter
                                 (ccpi_plan_set_cone_backprojector 1): faster,
                                 equal to the gather to float rounding, the
                                 order of its additions not fixed; SIRT and
                                 MLEM are unchanged */
};

/* ccpi_reconstruct with flags (0 gives ccpi_reconstruct).  No reference
 * counterpart beyond ccpi_reconstruct's: the flags choose among this
 * build's equivalent forms.  Unknown flag bits are an error. */
int ccpi_reconstruct_flags(const ccpi_geometry *geometry, int alg, const float *sino, int niter,
                           double regularize, double *norms, float *volume, int flags);

/* ---------------------------------------------------------------------
 * Device-level calls (device buffers; asynchronous on `stream` unless
 * stated).  Replace the core projector and solver entry points the
 * wrappers above drive: parallel_beam::f2D / b2D (Core/src/p2D.cpp:468,
 * :950), cone_beam::f2D / b2D (Core/src/c2D.cpp:469, :1052) and
 * reconstruction_alg::reconstruct (Core/src/algorithms.hpp:13-20).
 * ------------------------------------------------------------------- */

/* Build the device tables of a geometry on the current device (blocking).
 * The geometry's arrays are copied; the caller may free them. */
int ccpi_plan_create(const ccpi_geometry *geometry, ccpi_plan **plan);
void ccpi_plan_destroy(ccpi_plan *plan);
/* Time this plan's projector launch shapes on scratch data and keep the
 * fastest: the forward projector's grid (parallel beam) or rows per lane
 * (cone beam), the parallel back projector's slices per lane, and the cone
 * back projector's form (ccpi_plan_set_cone_backprojector; both forms timed
 * on a sinogram pre-scaled by d_conv, as the CGLS iterations run them).  No
 * counterpart in the reference (its block sizes are fixed).  Parallel
 * projections do not depend on the choice; CGLS step scalars may change in
 * the last FP64 bits (the number of partial sums follows the grid); the
 * cone scatter form changes the back projection at float rounding.  Call it
 * after ccpi_plan_create and before any solve or session on the plan.
 * chosen (may be NULL) receives {grid or rows per lane, slices per lane (parallel)
 * or 1 when the cone scatter was picked}.  Allocates and frees scratch of
 * one volume and one sinogram. */
int ccpi_plan_autotune(ccpi_plan *plan, void *stream, int chosen[2]);
/* Cone beam: the form of the back projector used by ccpi_backward and the
 * CGLS family (SIRT and MLEM always use the gather).  0 (the default): the
 * voxel-driven gather, the reference's design (cone_beam::b2D,
 * Core/src/c2D.cpp:948-1119) and equal to it bit for bit.  1: a ray-driven
 * scatter over the forward projector's walk (c2D.cpp:193-467) that applies
 * b2D's per-column row rules (c2D.cpp:657-750); each lane sums runs of its
 * consecutive detector rows that feed the same voxels in registers and adds
 * them with float atomics.  Equal to the reference to float rounding (the
 * order of the additions is not fixed).
 * ccpi_plan_autotune picks the faster for the plan's geometry. */
int ccpi_plan_set_cone_backprojector(ccpi_plan *plan, int scatter);

/* Measured ceiling of the projectors' gathers: GB/s at which the GPU reads
 * whole 1 KB columns at random offsets out of a working set of
 * working_set_bytes (rounded down to a power of two; pick one that fits L2,
 * e.g. 64 MiB), eight columns in
 * flight per lane.  A roofline denominator for ray-driven kernels whose
 * traffic is L2 -> SM rather than HBM.  No counterpart in the reference.
 * Allocates and frees the working set; waits for `stream`. */
int ccpi_measure_gather(unsigned long long working_set_bytes, void *stream,
                        double *gbs);
/* Sizes of a plan's volume and sinogram in elements. */
long long ccpi_plan_voxels(const ccpi_plan *plan);
long long ccpi_plan_pixels(const ccpi_plan *plan);

/* sino = A vol (overwritten). */
int ccpi_forward(const ccpi_plan *plan, const float *d_volume, float *d_sino,
                 void *stream);
/* vol = A^T sino (overwritten). */
int ccpi_backward(const ccpi_plan *plan, const float *d_sino, float *d_volume,
                  void *stream);
/* The same for n items of one plan stored one after another (volumes
 * nx*ny*nz floats apart, sinograms n_angles*n_h*n_v apart), e.g. a batch
 * of volumes under torch autograd.  Cone beam runs one launch per
 * direction, the batch sharing each ray's xy walk and each column's ray
 * list (f2D / b2D, Core/src/c2D.cpp:469-625, :948-1119, called once per
 * item in the reference); parallel beam one launch per item.  The cone
 * batch back projection is one gather launch on a gather plan; on a plan
 * set to the scatter (ccpi_plan_set_cone_backprojector 1) it runs the
 * scatter item by item.  Every item must start on a 16-byte boundary. */
int ccpi_forward_batch(const ccpi_plan *plan, int n, const float *d_volumes, float *d_sinos,
                       void *stream);
int ccpi_backward_batch(const ccpi_plan *plan, int n, const float *d_sinos, float *d_volumes,
                        void *stream);

/* Device bytes ccpi_solve needs as workspace for `alg` and `niterations`. */
size_t ccpi_solve_workspace_bytes(const ccpi_plan *plan, int alg,
                                  int niterations);

/* Run `alg` for `niterations` on the device.  d_x holds the starting volume
 * (zeros for a plain call) and receives the clamped result; d_sino is the
 * log sinogram (n_angles, n_h, n_v) and is not modified.  d_workspace may
 * be NULL (the library allocates and frees it).  h_norms (NULL or
 * niterations doubles) receives |A^T r| per CGLS-family iteration.  Blocks
 * until done. */
int ccpi_solve(const ccpi_plan *plan, int alg, const float *d_sino,
               float *d_x, int niterations, double regularize,
               double *h_norms, int flags, void *d_workspace,
               size_t workspace_bytes, void *stream);

/* Solve n independent problems (uneven sizes allowed) together: each
 * iteration of all problems is one captured CUDA graph whose branches run
 * concurrently.  regularize: n values (or NULL for 0).  Blocks until done. */
int ccpi_solve_batched(int n, const ccpi_plan *const *plans, int alg,
                       const float *const *d_sino, float *const *d_x,
                       int niterations, const double *regularize,
                       void *stream);

/* A prepared solver for iteration-by-iteration control (the reference's
 * reconstruction_alg::reconstruct loop of Core/src/Algorithms/cgls.cpp,
 * sirt.cpp and mlem.cpp, split
 * into set-up, iterations and the final clamp of voxels.cpp:187).
 * create: allocates the workspace, runs the set-up (initial back
 * projection / normalisations) and captures one iteration as a CUDA graph;
 * run: enqueues niterations graph launches on the session's stream
 * (asynchronous), at most max_iterations over the session's life;
 * finish: clamps d_x at zero, waits, checks the projectors' error flag and
 * copies the per-iteration |A^T r| (CGLS family) to h_norms (NULL or one
 * double per iteration run). */
typedef struct ccpi_session ccpi_session;
int ccpi_session_create(const ccpi_plan *plan, int alg, const float *d_sino,
                        float *d_x, double regularize, int max_iterations,
                        int flags, void *stream, ccpi_session **session);
int ccpi_session_run(ccpi_session *session, int niterations);
int ccpi_session_finish(ccpi_session *session, double *h_norms);
void ccpi_session_destroy(ccpi_session *session);

/* A CGLS-family solve (CCPI_CGLS, CCPI_CGLS_TIKHONOV, CCPI_CGLS_TV) of one
 * z slab of a parallel-beam volume that is cut into slabs over several
 * ranks (the reference's MPI split of the volume into z blocks,
 * Core/src/voxels.cpp:27-45; rows map to their own slices, so each rank
 * projects its slab alone).  The plan is the slab's geometry (its rows, its
 * slices).  The iteration of cgls.cpp:87-157 / :343-423 is run in stages;
 * between two stages the caller makes the exchange the next stage needs:
 *   SETUP     then all-reduce (sum) *d_sum; TV: swap halos
 *   FORWARD   then all-reduce *d_sum
 *   UPDATE    then TV: swap halos
 *   BACKWARD  then all-reduce *d_sum
 *   NEXT      then TV: swap halos; continue with FORWARD
 * d_sum: one device double, written by SETUP / FORWARD / BACKWARD with this
 * rank's FP64 partial sum and read back (all-reduced in place by the
 * caller) by the next stage.  d_edges: 2 * nx * ny device floats, the
 * slab's first and last z planes ([x][y]) after the stages marked "swap
 * halos"; d_halo_lo / d_halo_hi: nx * ny device floats holding the
 * neighbouring slabs' adjacent planes (the lower neighbour's last plane,
 * the upper neighbour's first plane), or NULL at the volume's ends, where
 * the TV stencil mirrors as in the reference (total_v.cpp:31-52).  One rank
 * with no halos gives ccpi_solve's result bit for bit.  Stages are enqueued
 * on `stream` and are not waited for; out-of-order stages are an error.
 * finish (after NEXT): clamps d_x at zero, waits, returns the per-iteration
 * |A^T r| of the whole volume. */
typedef struct ccpi_shard ccpi_shard;
enum {
  CCPI_SHARD_SETUP = 0,
  CCPI_SHARD_FORWARD = 1,
  CCPI_SHARD_UPDATE = 2,
  CCPI_SHARD_BACKWARD = 3,
  CCPI_SHARD_NEXT = 4
};
int ccpi_shard_create(const ccpi_plan *plan, int alg, const float *d_sino, float *d_x,
                      double regularize, int max_iterations, double *d_sum, float *d_edges,
                      const float *d_halo_lo, const float *d_halo_hi, void *stream,
                      ccpi_shard **shard);
int ccpi_shard_stage(ccpi_shard *shard, int stage);
int ccpi_shard_finish(ccpi_shard *shard, double *h_norms);
void ccpi_shard_destroy(ccpi_shard *shard);

/* ccpi_solve for callers that must not allocate device memory during a
 * solve: a host that owns all device memory through its own pool, or a
 * loop running other streams that cannot take the device-wide
 * synchronisation of a cudaMalloc/cudaFree pair per call.  No counterpart
 * in the reference (its solvers allocate on the host heap per call).
 * The solver workspace is a 16 MiB scratch area compiled into the library
 * (per device); problems needing more (ccpi_solve_workspace_bytes) are
 * rejected with an error naming both sizes.  The scratch needs no zeroing:
 * every buffer is initialised by the solve.  The first call on a device
 * looks up the scratch address (this may load the library's module): make
 * it before any stream capture begins.  Iterations are host-driven (the
 * CCPI_SOLVE_PLAIN schedule).  All calls on one device share the scratch,
 * so calls that overlap in time (several host threads) race; each call
 * blocks until done, so sequential calls are safe.  The plan's device must
 * be the current device (an error otherwise).  Arguments and results are as
 * for ccpi_solve. */
int ccpi_solve_noalloc(const ccpi_plan *plan, int alg, const float *d_sino,
                       float *d_x, int niterations, double regularize,
                       double *h_norms, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CCPI_B200_H */
