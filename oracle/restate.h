/* CPU restatement of CCPi-Reconstruction's iterative hot path (oracle).
 *
 * TEST INFRASTRUCTURE ONLY.  Loaded by tests/, by the smoke check and by
 * bench.py's CPU-baseline leg as the checker; the product never links it.
 *
 * Two builds of every routine: *_f32 uses the reference's own arithmetic
 * types (float data, float "recon_type" intermediates, double geometry) and
 * operation order, and is expected to agree bit for bit with the reference
 * compiled from its sources (oracle/_ref); *_f64 runs the same algorithm
 * entirely in double and is the FP64 oracle used to state the error of
 * both the reference and the CUDA path.
 *
 * Layout (the reference's): sinogram (n_angles, n_h, n_v), v fastest;
 * volume (nx, ny, nz), z fastest.  Angles in radians.
 */
#ifndef CCPI_ORACLE_RESTATE_H
#define CCPI_ORACLE_RESTATE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int kind; /* 0 parallel beam, 1 cone beam */
  int na, nh, nv;
  const double *angles;   /* na, radians */
  const double *h_pixels; /* nh detector column positions */
  const double *v_pixels; /* nv detector row positions */
  double source[3];       /* cone only */
  double detector_x;      /* cone only */
  double origin[3];       /* voxel grid corner */
  double size[3];         /* voxel size */
  int nx, ny, nz;
} rs_geometry;

enum { RS_CGLS = 0, RS_SIRT = 1, RS_MLEM = 2, RS_TIKHONOV = 3, RS_TV = 4 };

/* Projectors: the output is accumulated into (callers zero it first, as the
 * reference's fresh arrays are). */
void rs_fp_f32(const rs_geometry *g, const float *vol, float *pix);
void rs_bp_f32(const rs_geometry *g, const float *pix, float *vol);
void rs_fp_f64(const rs_geometry *g, const double *vol, double *pix);
void rs_bp_f64(const rs_geometry *g, const double *pix, double *vol);

/* Solvers.  x holds the starting volume on entry (zeros for the plain
 * call; the previous volume for the *_step calls) and the clamped result on
 * exit; sino is not modified.  norms (may be NULL) receives |R| per
 * iteration for the CGLS family. */
int rs_solve_f32(const rs_geometry *g, int alg, const float *sino, float *x,
                 int niter, double lambda, double *norms);
int rs_solve_f64(const rs_geometry *g, int alg, const double *sino, double *x,
                 int niter, double lambda, double *norms);

/* Regularisers (Tikhonov xy stencil, 3-D TV divergence). */
void rs_regularize_f32(int alg, int nx, int ny, int nz, const float *a,
                       float *b);
void rs_regularize_f64(int alg, int nx, int ny, int nz, const double *a,
                       double *b);

/* AML ring-artefact filter (Core/src/diamond.cpp:660-808) on a log
 * sinogram in the layout [angle][h][v], in place.  Returns 1 (and leaves p
 * unchanged) for parameters the reference rejects. */
int rs_aml_ring_f32(float *p, int na, int nh, int nv, double param_n,
                    double param_r, int num_series);

/* High-peaks filter (Core/src/diamond.cpp:513-617) on a log sinogram
 * [angle][h][v], in place: num_pix rounds of a top-to-bottom and a
 * bottom-to-top pass that limit every drop between neighbouring angles to
 * jump.  Returns 1 (p unchanged) for the parameters the reference rejects. */
int rs_high_peaks_f32(float *p, int na, int nh, int nv, double jump,
                      int num_pix);

/* Column ring-artefact filter (Core/src/diamond.cpp:619-658), in place:
 * every (h, v) element loses its FP64 mean over the angles. */
void rs_column_ring_f32(float *p, int na, int nh, int nv);

/* -log(p) with the C library's logf, as the reference's read_scans does. */
void rs_neglog_f32(const float *in, float *out, long long n);

/* exp(-p) with the C library's expf, as the reference's filter wrapper
 * turns logs back into transmission (diamond_wrapper.cpp:45-48). */
void rs_expneg_f32(const float *in, float *out, long long n);

#ifdef __cplusplus
}
#endif
#endif
