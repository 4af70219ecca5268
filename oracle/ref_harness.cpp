// Test infrastructure: C entry points into the reference's own iterative
// core (CCPi-Reconstruction Core/src), compiled by oracle/Makefile into
// oracle/_ref/libccpi_ref.so.  Each function mirrors the marshalling of the
// reference's boost.python wrapper it names, so that tests can run the
// reference exactly as a Python user of `ccpi.reconstruction.*.alg` would.
// Only tests/, the smoke check and bench.py's CPU-baseline leg load this.
//
// Two hazards in the reference are contained here rather than fixed (the
// reference is the oracle and must run unmodified):
//  * cone_beam::bproject_ah writes its scratch lists past their capacity
//    when a voxel's shadow spans more than two detector columns per angle
//    (Core/src/c2D.cpp:808-814, checked only after the fact at :939-940);
//  * cgls_regularize::reconstruct updates r_vox with sinogram extents
//    (Core/src/Algorithms/cgls.cpp:386), out of bounds when n_angles > nx.
// Both only write memory that is never read back for the result, so every
// allocation made by the reference is padded (operator new below).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "base_types.hpp"
#include "instruments.hpp"
#include "algorithms.hpp"
#include "cgls.hpp"
#include "sirt.hpp"
#include "mlem.hpp"
#include "results.hpp"
#include "voxels.hpp"
#include "mpi.hpp"

// ---------------------------------------------------------------- padding
static double g_pad_factor = 0.0;
static const std::size_t g_pad_bytes = 1 << 18;

void *operator new(std::size_t n) {
  std::size_t extra = g_pad_bytes + std::size_t(g_pad_factor * double(n));
  void *p = std::calloc(1, n + extra);
  if (!p)
    throw std::bad_alloc();
  return p;
}
void *operator new[](std::size_t n) { return operator new(n); }
void operator delete(void *p) noexcept { std::free(p); }
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete(void *p, std::size_t) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }

extern "C" void ref_set_pad_factor(double f) { g_pad_factor = f < 0 ? 0 : f; }

// ------------------------------------------------------------- helpers
namespace {

enum { ALG_CGLS = 0, ALG_SIRT = 1, ALG_MLEM = 2, ALG_TIKHONOV = 3, ALG_TV = 4 };

CCPi::reconstruction_alg *make_alg(int alg, int niter, double lambda) {
  switch (alg) {
  case ALG_CGLS:
    return new CCPi::cgls_3d(niter);
  case ALG_SIRT:
    return new CCPi::sirt(niter);
  case ALG_MLEM:
    return new CCPi::mlem(niter);
  case ALG_TIKHONOV:
    return new CCPi::cgls_tikhonov(niter, lambda);
  case ALG_TV:
    return new CCPi::cgls_tv_reg(niter, lambda);
  }
  return 0;
}

// Parallel-beam instrument that also exposes its detector coordinates.
class probe_diamond : public CCPi::Diamond {
public:
  using CCPi::instrument::get_h_pixels;
  using CCPi::instrument::get_v_pixels;
};

class probe_xtek : public CCPi::Nikon_XTek {
public:
  using CCPi::instrument::get_h_pixels;
  using CCPi::instrument::get_v_pixels;
};

// Cone-beam instrument with caller-given geometry: the explicit-grid case
// (no voxel-grid choice, no centre search), solved by the reference's own
// algorithms on the reference's own cone_beam projectors.
class explicit_cone : public CCPi::cone_beam {
public:
  bool setup_experimental_geometry(const std::string, const std::string,
                                   const real, const int, const bool) {
    return false;
  }
  bool setup_experimental_geometry(const numpy_3d &, const numpy_1d &,
                                   const real, const int) {
    return false;
  }
  bool setup_experimental_geometry(const numpy_3d &, const numpy_1d &,
                                   const numpy_1d &, const numpy_1d &,
                                   const int, const real, const real,
                                   const real, const real, const real,
                                   const bool) {
    return false;
  }
  bool read_scans(const std::string, const int, const int, const bool,
                  const bool) {
    return false;
  }
  bool read_scans(const numpy_3d &, const int, const int, bool) {
    return false;
  }
  bool finish_voxel_geometry(real *, real *, const int, const int,
                             const int) const {
    return true;
  }
  void get_xy_size(int &, int &, const int) {}
  void apply_beam_hardening() {}
  void load(const float *sino, int na, int nh, int nv) {
    pixel_3d &p = create_pixel_data();
    std::memcpy(p.data(), sino, sizeof(float) * std::size_t(na) * nh * nv);
  }
};

void to_real(real_1d &dst, const double *src, int n) {
  dst.resize(n);
  for (int i = 0; i < n; i++)
    dst[i] = src[i];
}

} // namespace

// ------------------------------------------------ parallel beam (Diamond)

// Geometry the reference derives for a parallel-beam numpy call
// (Core/src/diamond.cpp:35-86, :453-501, voxels.cpp:12-46).
// geom[0..3] = h_pixels[0], v_pixels[0], h_vox_size(xy), v_vox_size(z)
// dims[0..3] = nx, ny, nz, nv_padded
extern "C" int ref_pb_geometry(int na, int nv, int nh, double cor, int ppv,
                               int *dims, double *geom) {
  probe_diamond d;
  numpy_3d pix((float *)0, boost::extents[na][nv][nh]);
  std::vector<float> ang(na, 0.0f);
  numpy_1d angles(ang.data(), boost::extents[na]);
  if (!d.setup_experimental_geometry(pix, angles, cor, ppv))
    return 1;
  int nx = 0, ny = 0, nz = 0, maxz = 0, bs = 0, bstep = 0;
  calculate_block_sizes(nx, ny, nz, maxz, bs, bstep, 1, 0, ppv, &d, false);
  real origin[3], size[3];
  d.finish_voxel_geometry(origin, size, nx, ny, maxz);
  dims[0] = nx;
  dims[1] = ny;
  dims[2] = maxz;
  dims[3] = d.get_num_v_pixels();
  geom[0] = d.get_h_pixels()[0];
  geom[1] = d.get_v_pixels()[0];
  geom[2] = size[0];
  geom[3] = size[2];
  return 0;
}

// Mirrors reconstruct_iter (Wrappers/Python/src/diamond_wrapper.cpp:53-137)
// and its *_step variant (:140-257) when x0 != NULL.  pixels: (na, nv, nh)
// float32; angles in degrees (float32, as the wrapper reads them); out must
// hold nx*ny*nz floats (ref_pb_geometry).
extern "C" int ref_pb_reconstruct(int alg, const float *pixels, int na, int nv,
                                  int nh, const float *angles_deg, double cor,
                                  int ppv, int niter, int nthreads, int is_log,
                                  double lambda, const float *x0, float *out) {
  numpy_3d pix(const_cast<float *>(pixels), boost::extents[na][nv][nh]);
  numpy_1d angles(const_cast<float *>(angles_deg), boost::extents[na]);
  CCPi::reconstruction_alg *algorithm = make_alg(alg, niter, lambda);
  if (!algorithm)
    return 2;
  CCPi::instrument *instrument = new CCPi::Diamond();
  machine::initialise(nthreads);
  voxel_data *voxels = 0;
  voxel_data *input = 0;
  if (x0) {
    int dims[4];
    double geom[4];
    ref_pb_geometry(na, nv, nh, cor, ppv, dims, geom);
    input = new voxel_data(boost::extents[dims[0]][dims[1]][dims[2]]);
    std::memcpy(input->data(), x0,
                sizeof(float) * std::size_t(dims[0]) * dims[1] * dims[2]);
    voxels = reconstruct(instrument, algorithm, pix, angles, cor, ppv, 0,
                         false, is_log != 0, input);
  } else {
    voxels = reconstruct(instrument, algorithm, pix, angles, cor, ppv, 0,
                         false, is_log != 0);
  }
  machine::exit();
  delete instrument;
  delete algorithm;
  if (!voxels)
    return 3;
  const voxel_data::size_type *s = voxels->shape();
  std::memcpy(out, voxels->data(), sizeof(float) * s[0] * s[1] * s[2]);
  delete voxels;
  return 0;
}

// Mirrors pb_forward_project (diamond_wrapper.cpp:421-556): the detector is
// derived from the volume shape (width max(vx, vy), height vz, centre at
// width/2); out is (na, nv_padded, width) float32.
extern "C" int ref_pb_forward_project(const float *vol, int vx, int vy, int vz,
                                      const float *angles_deg, int na, int ppv,
                                      float *out, int *nv_pad_out) {
  probe_diamond d;
  int width = vx > vy ? vx : vy;
  numpy_3d pix((float *)0, boost::extents[na][vz][width]);
  numpy_1d angles(const_cast<float *>(angles_deg), boost::extents[na]);
  if (!d.setup_experimental_geometry(pix, angles, double(width) / 2.0, ppv))
    return 1;
  int nx = 0, ny = 0, nz = 0, maxz = 0, bs = 0, bstep = 0;
  calculate_block_sizes(nx, ny, nz, maxz, bs, bstep, 1, 0, ppv, &d, false);
  d.set_v_block(bs * ppv);
  int n_h = d.get_num_h_pixels();
  int n_v = d.get_num_v_pixels();
  *nv_pad_out = n_v;
  if (!out)
    return 0;
  real origin[3], size[3];
  d.finish_voxel_geometry(origin, size, vx, vy, vz);
  pixel_data Ad(boost::extents[na][n_h][n_v]);
  voxel_data v(boost::extents[vx][vy][vz]);
  std::memcpy(v.data(), vol, sizeof(float) * std::size_t(vx) * vy * vz);
  d.forward_project(Ad, v, origin, size, vx, vy, vz);
  for (int i = 0; i < na; i++)
    for (int j = 0; j < n_v; j++)
      for (int k = 0; k < n_h; k++)
        out[(std::size_t(i) * n_v + j) * n_h + k] = Ad[i][k][j];
  return 0;
}

// Mirrors pb_backward_project (diamond_wrapper.cpp:633-757): stack is
// (na, nv, nh); out is the API grid (nx, ny, nz) of ref_pb_geometry.
// Note the wrapper copies stack[i][k][j] for k < n_v (the padded count).
extern "C" int ref_pb_backward_project(const float *stack, int na, int nv,
                                       int nh, const float *angles_deg,
                                       double cor, int ppv, float *out) {
  probe_diamond d;
  numpy_3d pix(const_cast<float *>(stack), boost::extents[na][nv][nh]);
  numpy_1d angles(const_cast<float *>(angles_deg), boost::extents[na]);
  if (!d.setup_experimental_geometry(pix, angles, cor, ppv))
    return 1;
  int nx = 0, ny = 0, nz = 0, maxz = 0, bs = 0, bstep = 0;
  calculate_block_sizes(nx, ny, nz, maxz, bs, bstep, 1, 0, ppv, &d, false);
  d.set_v_block(bs * ppv);
  int n_h = d.get_num_h_pixels();
  int n_v = d.get_num_v_pixels();
  real origin[3], size[3];
  d.finish_voxel_geometry(origin, size, nx, ny, maxz);
  pixel_data Ad(boost::extents[na][n_h][n_v]);
  voxel_data v(boost::extents[nx][ny][maxz]);
  // the wrapper reads rows k < n_v of an array that has nv rows; rows past
  // nv do not exist in the caller's array, so they are taken as zero here.
  for (int k = 0; k < n_v && k < nv; k++)
    for (int j = 0; j < n_h; j++)
      for (int i = 0; i < na; i++)
        Ad[i][j][k] = stack[(std::size_t(i) * nv + k) * nh + j];
  d.backward_project(Ad, v, origin, size, nx, ny, maxz);
  std::memcpy(out, v.data(), sizeof(float) * std::size_t(nx) * ny * maxz);
  return 0;
}

// Direct parallel_beam::f2D / b2D with explicit geometry (the core-level
// projector call of Wrappers/Matlab/mex/PBproject_single_newgeom_c.cpp).
// pixels are (na, nh, nv), voxels (nx, ny, nz); out accumulates (zero it).
extern "C" void ref_pb_f2d(const double *h_pixels, int nh,
                           const double *v_pixels, int nv,
                           const double *angles_rad, int na,
                           const double *origin, const double *size, int nx,
                           int ny, int nz, const float *vol, float *pix_out) {
  real_1d h, v, a;
  to_real(h, h_pixels, nh);
  to_real(v, v_pixels, nv);
  to_real(a, angles_rad, na);
  pixel_data p(boost::extents[na][nh][nv]);
  voxel_data x(boost::extents[nx][ny][nz]);
  std::memcpy(x.data(), vol, sizeof(float) * std::size_t(nx) * ny * nz);
  real o[3] = {origin[0], origin[1], origin[2]};
  real s[3] = {size[0], size[1], size[2]};
  CCPi::parallel_beam::f2D(h, v, a, na, nh, nv, o, s, nx, ny, nz, p, x);
  std::memcpy(pix_out, p.data(), sizeof(float) * std::size_t(na) * nh * nv);
}

extern "C" void ref_pb_b2d(const double *h_pixels, int nh,
                           const double *v_pixels, int nv,
                           const double *angles_rad, int na,
                           const double *origin, const double *size, int nx,
                           int ny, int nz, const float *pix, float *vol_out) {
  real_1d h, v, a;
  to_real(h, h_pixels, nh);
  to_real(v, v_pixels, nv);
  to_real(a, angles_rad, na);
  pixel_data p(boost::extents[na][nh][nv]);
  std::memcpy(p.data(), pix, sizeof(float) * std::size_t(na) * nh * nv);
  voxel_data x(boost::extents[nx][ny][nz]);
  real o[3] = {origin[0], origin[1], origin[2]};
  real s[3] = {size[0], size[1], size[2]};
  CCPi::parallel_beam::b2D(h, v, a, p, x, na, nh, nv, o, s, nx, ny, nz);
  std::memcpy(vol_out, x.data(), sizeof(float) * std::size_t(nx) * ny * nz);
}

// ------------------------------------------------- cone beam (Nikon XTek)

// Geometry the reference derives for a cone-beam numpy call
// (Core/src/Readers/xtek.cpp:57-129, :367-380, :519-564, :671-798) including
// the centre-of-rotation search when pixels != NULL.
// dims[0..3] = nx, ny, nz, nv_padded
// geom[0..6] = voxel size xy, voxel size z, origin x, y, z,
//              source_y after find_centre, h_pixels[0] after find_centre
extern "C" int ref_cb_geometry(const float *pixels, int na, int nh, int nv,
                               const float *angles_deg, int ppv,
                               double source_to_sample,
                               double source_to_detector, double pixel_h,
                               double pixel_v, double mask_radius, int is_log,
                               int *dims, double *geom) {
  probe_xtek d;
  numpy_3d pix(const_cast<float *>(pixels), boost::extents[na][nh][nv]);
  std::vector<float> zeros_ang(na, 0.0f);
  numpy_1d angles(angles_deg ? const_cast<float *>(angles_deg)
                             : zeros_ang.data(),
                  boost::extents[na]);
  float off = 0.0f;
  numpy_1d hoff(&off, boost::extents[1]);
  real source_x = -source_to_sample;
  real detector_x = source_to_detector + source_x;
  if (!d.setup_experimental_geometry(pix, angles, hoff, hoff, ppv, source_x,
                                     detector_x, pixel_h, pixel_v,
                                     mask_radius, false))
    return 1;
  int nx = 0, ny = 0, nz = 0, maxz = 0, bs = 0, bstep = 0;
  calculate_block_sizes(nx, ny, nz, maxz, bs, bstep, 1, 0, ppv, &d, false);
  d.set_v_block(bs * ppv);
  real origin[3], size[3];
  d.finish_voxel_geometry(origin, size, nx, ny, maxz);
  dims[0] = nx;
  dims[1] = ny;
  dims[2] = maxz;
  dims[3] = d.get_num_v_pixels();
  geom[0] = size[0];
  geom[1] = size[2];
  geom[2] = origin[0];
  geom[3] = origin[1];
  geom[4] = origin[2];
  geom[5] = d.get_source_y();
  geom[6] = d.get_h_pixels()[0];
  if (pixels) {
    if (!d.read_scans(pix, 0, bs * ppv, is_log != 0))
      return 2;
    geom[5] = d.get_source_y();
    geom[6] = d.get_h_pixels()[0];
  }
  return 0;
}

// Mirrors conebeam_reconstruct_iter
// (Wrappers/Python/src/conebeam_wrapper.cpp:14-121).  pixels (na, nh, nv).
extern "C" int ref_cb_reconstruct(int alg, const float *pixels, int na, int nh,
                                  int nv, const float *angles_deg, int ppv,
                                  double source_to_sample,
                                  double source_to_detector, double pixel_h,
                                  double pixel_v, double mask_radius,
                                  int niter, int nthreads, int is_log,
                                  double lambda, float *out) {
  numpy_3d pix(const_cast<float *>(pixels), boost::extents[na][nh][nv]);
  numpy_1d angles(const_cast<float *>(angles_deg), boost::extents[na]);
  float off = 0.0f;
  numpy_1d hoff(&off, boost::extents[1]);
  real source_x = -source_to_sample;
  real detector_x = source_to_detector + source_x;
  CCPi::reconstruction_alg *algorithm = make_alg(alg, niter, lambda);
  if (!algorithm)
    return 2;
  CCPi::instrument *instrument = new CCPi::Nikon_XTek();
  machine::initialise(nthreads);
  real vox_origin[3] = {0, 0, 0};
  real vox_size[3] = {0, 0, 0};
  voxel_data *voxels =
      reconstruct(instrument, algorithm, pix, angles, hoff, hoff, ppv,
                  source_x, detector_x, pixel_h, pixel_v, mask_radius, false,
                  vox_origin, vox_size, false, is_log != 0);
  machine::exit();
  delete instrument;
  delete algorithm;
  if (!voxels)
    return 3;
  const voxel_data::size_type *s = voxels->shape();
  std::memcpy(out, voxels->data(), sizeof(float) * s[0] * s[1] * s[2]);
  delete voxels;
  return 0;
}

// Direct cone_beam::f2D / b2D with explicit geometry (the call
// conebeam.create_sinogram makes, conebeam_wrapper.cpp:346-400, with angles
// in radians).  pixels (na, nh, nv), voxels (nx, ny, nz).
extern "C" void ref_cb_f2d(double sx, double sy, double sz, double det_x,
                           const double *h_pixels, int nh,
                           const double *v_pixels, int nv,
                           const double *angles_rad, int na,
                           const double *origin, const double *size, int nx,
                           int ny, int nz, const float *vol, float *pix_out) {
  real_1d h, v, a;
  to_real(h, h_pixels, nh);
  to_real(v, v_pixels, nv);
  to_real(a, angles_rad, na);
  pixel_data p(boost::extents[na][nh][nv]);
  voxel_data x(boost::extents[nx][ny][nz]);
  std::memcpy(x.data(), vol, sizeof(float) * std::size_t(nx) * ny * nz);
  real o[3] = {origin[0], origin[1], origin[2]};
  real s[3] = {size[0], size[1], size[2]};
  CCPi::cone_beam::f2D(sx, sy, sz, det_x, h, v, a, p, x, na, nh, nv, o, s, nx,
                       ny, nz);
  std::memcpy(pix_out, p.data(), sizeof(float) * std::size_t(na) * nh * nv);
}

extern "C" void ref_cb_b2d(double sx, double sy, double sz, double det_x,
                           const double *h_pixels, int nh,
                           const double *v_pixels, int nv,
                           const double *angles_rad, int na,
                           const double *origin, const double *size, int nx,
                           int ny, int nz, const float *pix, float *vol_out) {
  real_1d h, v, a;
  to_real(h, h_pixels, nh);
  to_real(v, v_pixels, nv);
  to_real(a, angles_rad, na);
  pixel_data p(boost::extents[na][nh][nv]);
  std::memcpy(p.data(), pix, sizeof(float) * std::size_t(na) * nh * nv);
  voxel_data x(boost::extents[nx][ny][nz]);
  real o[3] = {origin[0], origin[1], origin[2]};
  real s[3] = {size[0], size[1], size[2]};
  CCPi::cone_beam::b2D(sx, sy, sz, det_x, h, v, a, p, x, na, nh, nv, o, s, nx,
                       ny, nz);
  std::memcpy(vol_out, x.data(), sizeof(float) * std::size_t(nx) * ny * nz);
}

// The reference's solvers on an explicit cone geometry (no grid choice, no
// centre search, no output clamp: the clamp is voxels.cpp:272's job and is
// applied here too so the result matches the numpy path's semantics).
extern "C" int ref_cb_solve_explicit(int alg, double sx, double sy, double sz,
                                     double det_x, const double *h_pixels,
                                     int nh, const double *v_pixels, int nv,
                                     const double *angles_rad, int na,
                                     const float *sino, const double *origin,
                                     const double *size, int nx, int ny,
                                     int nz, int niter, double lambda,
                                     int nthreads, float *out) {
  explicit_cone dev;
  std::vector<real> hp(h_pixels, h_pixels + nh), vp(v_pixels, v_pixels + nv),
      ap(angles_rad, angles_rad + na);
  dev.set_params(sx, sy, sz, det_x, hp.data(), vp.data(), ap.data(), nh, nv,
                 na);
  dev.load(sino, na, nh, nv);
  CCPi::reconstruction_alg *algorithm = make_alg(alg, niter, lambda);
  if (!algorithm)
    return 2;
  machine::initialise(nthreads);
  voxel_data x(boost::extents[nx][ny][nz]);
  real o[3] = {origin[0], origin[1], origin[2]};
  real s[3] = {size[0], size[1], size[2]};
  bool ok = algorithm->reconstruct(&dev, x, o, s);
  machine::exit();
  delete algorithm;
  if (!ok)
    return 3;
  float *xd = x.data();
  std::size_t n = std::size_t(nx) * ny * nz;
  for (std::size_t i = 0; i < n; i++)
    out[i] = xd[i] < 0.0f ? 0.0f : xd[i];
  return 0;
}

// The reference's regularisers (Core/src/tikhonov.cpp:5-33,
// Core/src/total_v.cpp:21-195) on a (nx, ny, nz) volume.
#include "regularize.hpp"
extern "C" void ref_regularize(int alg, int nx, int ny, int nz, const float *a,
                               float *b) {
  voxel_data in(boost::extents[nx][ny][nz]);
  voxel_data out(boost::extents[nx][ny][nz]);
  std::memcpy(in.data(), a, sizeof(float) * std::size_t(nx) * ny * nz);
  if (alg == ALG_TIKHONOV)
    CCPi::tikhonov_regularize(out, in, nx, ny, nz);
  else
    CCPi::tv_regularize(out, in, nx, ny, nz);
  std::memcpy(b, out.data(), sizeof(float) * std::size_t(nx) * ny * nz);
}

// The reference's AML ring-artefact filter (CCPi::remove_aml_ring_artefacts,
// Core/src/diamond.cpp:660-808) on a log sinogram in its pixel layout
// [angle][h][v], in place.
extern "C" void ref_aml_ring(float *p, int na, int nh, int nv, double param_n, double param_r,
                             int num_series) {
  pixel_data px(boost::extents[na][nh][nv]);
  std::memcpy(px.data(), p, sizeof(float) * std::size_t(na) * nh * nv);
  CCPi::remove_aml_ring_artefacts(px, na, nh, nv, param_n, param_r, num_series);
  std::memcpy(p, px.data(), sizeof(float) * std::size_t(na) * nh * nv);
}

// The reference's high-peaks filter is a private member of CCPi::Diamond
// (Core/src/instruments.hpp:371, diamond.cpp:513-617).  An explicit template
// instantiation may name a private member; it hands the member pointer to a
// friend function, through which the harness calls the reference's own code
// on a Diamond whose sizes and pixels it sets.
struct hp_member {
  typedef void (CCPi::Diamond::*type)(const real, const int);
  friend type hp_get(hp_member);
};
template <typename Tag, typename Tag::type M> struct hp_expose {
  friend typename Tag::type hp_get(Tag) { return M; }
};
template struct hp_expose<hp_member, &CCPi::Diamond::high_peaks_before>;

class hp_diamond : public CCPi::Diamond {
public:
  void load(const float *p, int na, int nh, int nv) {
    set_phi(na);
    set_h_pixels(nh);
    set_v_pixels(nv);
    pixel_3d &px = create_pixel_data();
    std::memcpy(px.data(), p, sizeof(float) * std::size_t(na) * nh * nv);
  }
};

// CCPi::Diamond::high_peaks_before on a log sinogram [angle][h][v], in place.
extern "C" void ref_high_peaks(float *p, int na, int nh, int nv, double jump, int num_pix) {
  hp_diamond d;
  d.load(p, na, nh, nv);
  (d.*hp_get(hp_member()))(jump, num_pix);
  std::memcpy(p, d.get_pixel_data().data(), sizeof(float) * std::size_t(na) * nh * nv);
}

// CCPi::remove_column_ring_artefacts (diamond.cpp:619-658), in place.
extern "C" void ref_column_ring(float *p, int na, int nh, int nv) {
  pixel_data px(boost::extents[na][nh][nv]);
  std::memcpy(px.data(), p, sizeof(float) * std::size_t(na) * nh * nv);
  CCPi::remove_column_ring_artefacts(px, na, nh, nv);
  std::memcpy(p, px.data(), sizeof(float) * std::size_t(na) * nh * nv);
}

// parallelbeam.filters.aml_ring_artefacts as the reference's wrapper runs it
// (Wrappers/Python/src/diamond_wrapper.cpp:18-51): pixels (na, nv, nh)
// transmission in, exp(-filtered -log) out, same layout.
extern "C" void ref_aml_ring_artefacts(const float *pixels, int na, int nv, int nh, float param_n,
                                       float param_r, int num_series, float *out) {
  pixel_3d p(boost::extents[na][nh][nv]);
  for (int i = 0; i < na; i++)
    for (int j = 0; j < nh; j++)
      for (int k = 0; k < nv; k++)
        p[i][j][k] = -std::log(pixels[(std::size_t(i) * nv + k) * nh + j]);
  CCPi::remove_aml_ring_artefacts(p, na, nh, nv, param_n, param_r, num_series);
  for (int i = 0; i < na; i++)
    for (int j = 0; j < nv; j++)
      for (int k = 0; k < nh; k++)
        out[(std::size_t(i) * nv + j) * nh + k] = std::exp(-p[i][k][j]);
}

// conebeam.create_phantom_volume as the reference's wrapper builds it
// (Wrappers/Python/src/conebeam_wrapper.cpp:270-310 over
// Nikon_XTek::initialise_phantom_volume, Core/src/Readers/xtek.cpp:825-894):
// vol (512^3), angles (250, degrees), h and v pixels (512 each) and
// scalars {source_x, detector_x, pixel_h, pixel_v, mask_radius}.
extern "C" void ref_cb_phantom_volume(float *vol, float *angles, float *h, float *v,
                                      double *scalars) {
  CCPi::Nikon_XTek *instrument = new CCPi::Nikon_XTek();
  real_1d hp(512), vp(512);
  voxel_data x = instrument->initialise_phantom_volume(hp, vp);
  std::memcpy(vol, x.data(), sizeof(float) * std::size_t(512) * 512 * 512);
  const double source_x = -1 * instrument->get_source_x();
  const double detector_x = instrument->get_detector_x() + source_x;
  real_1d phi = instrument->get_phi();
  for (int i = 0; i < instrument->get_num_angles(); i++)
    angles[i] = float(phi[i] * 180.0 / M_PI);
  for (int i = 0; i < 512; i++) {
    h[i] = float(hp[i]);
    v[i] = float(vp[i]);
  }
  scalars[0] = source_x;
  scalars[1] = detector_x;
  scalars[2] = 0.390625;
  scalars[3] = 0.390625;
  scalars[4] = instrument->get_mask_radius();
  delete instrument;
}
