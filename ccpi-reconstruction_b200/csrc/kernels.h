// Host-callable launchers for the device kernels (internal to the library).
#pragma once

#include "common.cuh"

namespace ccpi {

// projectors (pb_project.cu, cb_project.cu); out is overwritten
int pb_forward(const Geom &g, const float *vol, float *pix, int mode, const Epi &e,
               int grid, int *err, cudaStream_t st);
int pb_prepare();
int pb_fp_ctas(const Geom &g);
int pb_backward(const Geom &g, const float *pix, float *vol, int mode, const Epi &e,
                int *err, cudaStream_t st);
int pb_bp_tiles(const Geom &g);
int cb_prepare(const Geom &g);
// band[i * ny + j] = the back projector's band rows [x, y) of voxel column
// (i, j) (c2D.cpp:657-676); the cone back projectors read it as g.colband
int cb_column_bands(const Geom &g, int2 *band, cudaStream_t st);
size_t cb_fp_smem(const Geom &g);
size_t cb_bp_smem(const Geom &g);
// nb / nbatch: that many volumes and sinograms one after another, one launch
// (EPI_STORE); the walk, row regimes and band limits are shared
int cb_forward(const Geom &g, const float *vol, float *pix, int mode, const Epi &e,
               const int2 *hrange, int grid, cudaStream_t st, int nb = 1);
int cb_backward(const Geom &g, const float *pix, float *vol, int mode, const Epi &e,
                int *err, cudaStream_t st, int nbatch = 1);
// The ray-driven cone back projector (each lane sums runs of its rows in
// registers and adds them with float atomics; order of the additions not
// fixed): vol = A^T pix, EPI_STORE semantics; pre: pix is already scaled
// by d_conv.  Launch shape of the forward projector.
int cb_backward_scatter(const Geom &g, const float *pix, float *vol, int pre,
                        const int2 *hrange, int grid, cudaStream_t st);
// The cone back projector accepts a sinogram pre-scaled by d_conv (Epi::pre)
// for this geometry; cb_prescale writes that scaled copy.
bool cb_bp_takes_prescaled(const Geom &g);
void cb_prescale(const Geom &g, const float *in, float *out, cudaStream_t st);
// Streaming multiprocessors of the current device (engine.cu).
int sm_count();

// vector kernels (vec_ops.cu)
void k_fill(float *p, i64 n, float v, cudaStream_t st);
void k_invert_pos(float *p, i64 n, cudaStream_t st);    // p > 0 ? 1/p : 0
void k_invert_nonzero(float *p, i64 n, cudaStream_t st); // p != 0 ? 1/p : p
void k_clamp0(float *p, i64 n, cudaStream_t st);
void k_sumsq_partials(const float *x, i64 n, double *partials, int nblocks, cudaStream_t st);
int sumsq_blocks();

// CGLS scalar updates from FP64 partials.  s[] layout: see solver.cpp.
enum ScalarOp { S_INIT = 0, S_ALPHA = 1, S_ALPHA2 = 2, S_BETA = 3 };
void k_cgls_scalars(int op, const double *p1, int n1, const double *p2, int n2, double *s,
                    double *norms, cudaStream_t st);
// y += sign * alpha * x   (alpha = s[idx])
void k_axpy_scalar(float *y, const float *x, i64 n, const double *s, int idx, float sign,
                   cudaStream_t st);
// x += alpha d; d = s_vec + beta d
void k_cgls_xd(float *x, float *d, const float *sv, i64 n, const double *s, cudaStream_t st);
// d = s_vec + beta d
void k_cgls_d(float *d, const float *sv, i64 n, const double *s, cudaStream_t st);
// out = in + alpha * d   (alpha = s[1])
void k_add_scaled(float *out, const float *in, const float *d, i64 n, const double *s,
                  cudaStream_t st);

// regularisers (vec_ops.cu).  alg 3 Tikhonov, 4 TV.  lo / hi (may be NULL):
// the z planes just below and above a slab of a volume cut along z ([x][y]
// each), read by the TV stencil in place of the mirrored neighbour.
// acc += lambda * L(a), with per-CTA FP64 sum of squares of the new acc
void k_reg_accumulate(int alg, const float *a, float *acc, int nx, int ny, int nz,
                      float lambda, double *partials, int nblocks, cudaStream_t st,
                      const float *lo = nullptr, const float *hi = nullptr);
// out = a + lambda * L(a)
void k_reg_step(int alg, const float *a, float *out, int nx, int ny, int nz, float lambda,
                cudaStream_t st, const float *lo = nullptr, const float *hi = nullptr);
// Step scalars of a z-sharded solve (sum[0]: the value the ranks
// all-reduce between stages).
enum ShardOp { SH_LOCAL = 0, SH_INIT = 1, SH_ALPHA = 2, SH_BETA = 3 };
void k_shard_scalars(int op, const double *p1, int n1, const double *p2, int n2, double *sum,
                     double *s, double *norms, cudaStream_t st);
// lo / hi = the first / last z plane of a slab ([x][y] each)
void k_pack_edges(const float *a, int nx, int ny, int nz, float *lo, float *hi, cudaStream_t st);
// out = L(a)
void k_reg_apply(int alg, const float *a, float *out, int nx, int ny, int nz,
                 cudaStream_t st);

// numpy front-end layouts
// (na, nv, nh) -> (na, nh, nv_pad) with rows [voff, voff + nv) holding data
void k_pack_parallel(const float *in, float *out, int na, int nv, int nh, int nv_pad,
                     int voff, cudaStream_t st);
// (na, nh, nv) -> (na, nh, nv_pad)
void k_pack_cone(const float *in, float *out, int na, int nh, int nv, int nv_pad, int voff,
                 cudaStream_t st);
// (na, nh, nv) -> (na, nv, nh)
void k_unpack_parallel(const float *in, float *out, int na, int nh, int nv, cudaStream_t st);

} // namespace ccpi
