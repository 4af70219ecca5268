// C ABI of the library (declared in include/ccpi_b200.h).
//
// The reference-facing calls restate the numpy front-ends of the
// reference's Python wrappers: the Diamond parallel-beam geometry
// (Core/src/diamond.cpp:35-86, :394-501, instruments.cpp:35-64,
// voxels.cpp:12-46, :131-205), the Nikon XTek cone-beam geometry and its
// centre-of-rotation search (Core/src/Readers/xtek.cpp:57-129, :367-380,
// :519-564, :566-798), and the wrappers' marshalling
// (Wrappers/Python/src/diamond_wrapper.cpp, conebeam_wrapper.cpp).  Host
// work is limited to O(geometry) tables, the -log of transmission data
// (done with the C library's logf, as the reference does) and the centre
// search; the sinogram layout change and all projection work run on the
// GPU.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <omp.h>

#include "../../include/ccpi_b200.h"
#include "engine.h"
#include "kernels.h"

using ccpi::i64;
using ccpi::set_error;

namespace {

struct HostGeometry {
  ccpi_geometry g{};
  std::vector<double> angles, h, v;
  int nv_pad = 0, v_offset = 0;
  void bind() {
    g.angles = angles.data();
    g.h_pixels = h.data();
    g.v_pixels = v.data();
    g.n_angles = int(angles.size());
    g.n_h = int(h.size());
    g.n_v = int(v.size());
  }
};

// instrument::calc_v_alignment (instruments.cpp:35-64) with the conda
// build's 16-byte allocator alignment: rows padded to a multiple of
// 4 slices' worth of rows, data centred.
void v_alignment(int n, int ppv, int &npix, int &offset) {
  int nvox = n / ppv;
  if (n % ppv != 0)
    nvox++;
  const int align = 4;
  int blocks = nvox / align;
  if (nvox % align != 0)
    blocks++;
  npix = blocks * align * ppv;
  offset = (npix - n) / 2;
}

void degrees_to_radians(const float *deg, int n, std::vector<double> &out) {
  out.resize(n);
  for (int i = 0; i < n; i++)
    out[i] = M_PI * (double(deg[i]) / 180.0); // diamond.cpp:81-82, xtek.cpp:123-124
}

// Diamond numpy geometry (diamond.cpp:35-86) and voxel grid
// (diamond.cpp:479-501 via voxels.cpp:12-46, :453-477).
bool pb_geometry(int na, int nv, int nh, double cor, int ppv, const float *angles_deg,
                 HostGeometry &G) {
  if (na < 1 || nv < 1 || nh < 2 || ppv < 1) {
    set_error("parallel beam: need n_angles >= 1, n_v >= 1, n_h >= 2, resolution >= 1");
    return false;
  }
  const double hsize = 1.0, vsize = 1.0;
  v_alignment(nv, ppv, G.nv_pad, G.v_offset);
  double shift = 0.0;
  if (cor > 0.0)
    shift = hsize * (cor - double(nh) / 2.0);
  G.h.resize(nh);
  G.h[0] = -((nh - 1) * hsize) / 2.0 - shift;
  for (int i = 1; i < nh; i++)
    G.h[i] = G.h[0] + double(i) * hsize;
  G.v.resize(G.nv_pad);
  G.v[0] = -((G.nv_pad - 1) * vsize) / 2.0;
  for (int i = 1; i < G.nv_pad; i++)
    G.v[i] = G.v[0] + double(i) * vsize;
  if (angles_deg)
    degrees_to_radians(angles_deg, na, G.angles);
  else
    G.angles.assign(na, 0.0);
  const double hrange = G.h[1] - G.h[0];
  const double hmax = std::max(std::abs(G.h[0]), std::abs(G.h[nh - 1]));
  const int n = int(std::ceil((2.0 * hmax) / hrange));
  int nx = n / ppv;
  if (n % ppv != 0)
    nx++;
  const double hvox = hrange * double(ppv);
  double xmin = -hvox * double(nx) / 2.0, xmax = hvox * double(nx) / 2.0;
  while (xmin >= G.h[0] || xmax <= G.h[nh - 1]) {
    nx++;
    xmin = -hvox * double(nx) / 2.0;
    xmax = hvox * double(nx) / 2.0;
  }
  const double vvox = (G.v[1 < G.nv_pad ? 1 : 0] - G.v[0]) * double(ppv);
  int nz = G.nv_pad / ppv;
  if (G.nv_pad % ppv != 0)
    nz++;
  G.g.kind = CCPI_PARALLEL;
  G.g.nx = nx;
  G.g.ny = nx;
  G.g.nz = nz;
  G.g.voxel_size[0] = hvox;
  G.g.voxel_size[1] = hvox;
  G.g.voxel_size[2] = G.nv_pad > 1 ? vvox : vsize * double(ppv);
  for (int i = 0; i < 3; i++) {
    const int nn = i == 0 ? nx : (i == 1 ? nx : nz);
    G.g.origin[i] = -G.g.voxel_size[i] * double(nn) / 2.0;
  }
  G.bind();
  return true;
}

// Nikon XTek numpy geometry (xtek.cpp:57-129) and grid (xtek.cpp:760-798,
// :367-380).
bool cb_geometry(int na, int nh, int nv, int ppv, double s2s, double s2d, double px_h,
                 double px_v, double mask_radius, const float *angles_deg, HostGeometry &G) {
  if (na < 1 || nv < 1 || nh < 2 || ppv < 1) {
    set_error("cone beam: need n_angles >= 1, n_v >= 1, n_h >= 2, pixels_per_voxel >= 1");
    return false;
  }
  if (!(px_h > 0.0) || !(px_v > 0.0) || !(mask_radius > 0.0) || !(s2d > s2s) || !(s2s > 0.0)) {
    set_error("cone beam: need positive pixel sizes and mask radius, and "
              "0 < source_to_sample < source_to_detector");
    return false;
  }
  const double source_x = -s2s, detector_x = s2d + source_x;
  v_alignment(nv, ppv, G.nv_pad, G.v_offset);
  G.h.resize(nh);
  G.h[0] = -((nh - 1) * px_h) / 2.0;
  for (int i = 1; i < nh; i++)
    G.h[i] = G.h[0] + double(i) * px_h;
  G.v.resize(G.nv_pad);
  G.v[0] = -((G.nv_pad - 1) * px_v) / 2.0;
  for (int i = 1; i < G.nv_pad; i++)
    G.v[i] = G.v[0] + double(i) * px_v;
  if (angles_deg)
    degrees_to_radians(angles_deg, na, G.angles);
  else
    G.angles.assign(na, 0.0);
  int n = nh / ppv;
  if (nh % ppv != 0)
    n++;
  double vsize = 2.0 * mask_radius / double(n);
  double vox_x = vsize * double(n) / 2.0;
  const int nvp = G.nv_pad;
  int nz = nvp / ppv;
  if (nvp % ppv != 0)
    nz++;
  double max_z = vsize * double(nz) / 2.0;
  double v_pos = G.v[nvp - 1];
  v_pos *= (vox_x - source_x) / (detector_x - source_x);
  if (max_z < v_pos) {
    vsize = -2.0 * source_x * G.v[nvp - 1] /
            (nz * (detector_x - source_x) - n * G.v[nvp - 1]);
    vsize *= (1.0 + 1.0 / double(nvp));
  }
  G.g.kind = CCPI_CONE;
  G.g.nx = n;
  G.g.ny = n;
  G.g.nz = nz;
  for (int i = 0; i < 3; i++)
    G.g.voxel_size[i] = vsize;
  G.g.origin[0] = -vsize * double(n) / 2.0;
  G.g.origin[1] = -vsize * double(n) / 2.0;
  G.g.origin[2] = -vsize * double(nz) / 2.0;
  G.g.source[0] = source_x;
  G.g.source[1] = 0.0;
  G.g.source[2] = 0.0;
  G.g.detector_x = detector_x;
  G.bind();
  return true;
}

// ---- centre-of-rotation search (xtek.cpp:566-758) ----
float linear_i(double x1, double x2, float f1, float f2, double x) {
  return float((f1 * (x2 - x) + f2 * (x - x1)) / (x2 - x1));
}
float bilinear_i(double x1, double x2, double y1, double y2, float f11, float f12, float f21,
                 float f22, double x, double y) {
  return float((f11 * (x2 - x) * (y2 - y) + f21 * (x - x1) * (y2 - y) +
                f12 * (x2 - x) * (y - y1) + f22 * (x - x1) * (y - y1)) /
               ((x2 - x1) * (y2 - y1)));
}

struct CentreData {
  const float *px; // (na, nh, nvp)
  int na, nh, nvp, vs;
  const double *h, *ang;
  bool sorted_angles;
  float at(int a, int k) const { return px[(i64(a) * nh + k) * nvp + vs]; }
  // first index i in [0, n-1) with x[i+1] > val, else n - 1
  static int bracket(const double *x, int n, double val, bool sorted) {
    if (sorted) {
      const double *u = std::upper_bound(x + 1, x + n, val);
      return int(u - (x + 1));
    }
    int i = 0;
    for (; i < n - 1; i++)
      if (x[i + 1] > val)
        break;
    return i;
  }
  float angles_linear(int ph1, double na_) const {
    if (na_ < ang[0])
      return linear_i(ang[na - 1] - 2.0 * M_PI, ang[0], at(na - 1, ph1), at(0, ph1), na_);
    const int pa1 = bracket(ang, na, na_, sorted_angles);
    if (ang[pa1] == na_)
      return at(pa1, ph1);
    if (pa1 == na - 1)
      return linear_i(ang[pa1], ang[0] + 2.0 * M_PI, at(pa1, ph1), at(0, ph1), na_);
    return linear_i(ang[pa1], ang[pa1 + 1], at(pa1, ph1), at(pa1 + 1, ph1), na_);
  }
  float angles_bilinear(int ph1, double nh_, double na_) const {
    if (na_ < ang[0])
      return bilinear_i(h[ph1], h[ph1 + 1], ang[na - 1] - 2.0 * M_PI, ang[0], at(na - 1, ph1),
                        at(0, ph1), at(na - 1, ph1 + 1), at(0, ph1 + 1), nh_, na_);
    const int pa1 = bracket(ang, na, na_, sorted_angles);
    if (ang[pa1] == na_)
      return linear_i(h[ph1], h[ph1 + 1], at(pa1, ph1), at(pa1, ph1 + 1), nh_);
    if (pa1 == na - 1)
      return bilinear_i(h[ph1], h[ph1 + 1], ang[pa1], ang[0] + 2.0 * M_PI, at(pa1, ph1),
                        at(0, ph1), at(pa1, ph1 + 1), at(0, ph1 + 1), nh_, na_);
    return bilinear_i(h[ph1], h[ph1 + 1], ang[pa1], ang[pa1 + 1], at(pa1, ph1),
                      at(pa1 + 1, ph1), at(pa1, ph1 + 1), at(pa1 + 1, ph1 + 1), nh_, na_);
  }
  float interpolate(double nh_, double na_) const {
    const int ph1 = bracket(h, nh, nh_, true);
    if (h[ph1] == nh_)
      return angles_linear(ph1, na_);
    return angles_bilinear(ph1, nh_, na_);
  }
};

// Returns the centre offset along h in the detector frame (the reference's
// "midpoint"), or NaN on failure.
double find_centre_midpoint(const CentreData &D, double distance) {
  const int nsamples = 21, nprec = 5;
  const double precision[nprec] = {1, 0.1, 0.01, 0.001, 0.0001};
  double midpoint = 0.0;
  const int nh = D.nh, na = D.na;
  std::vector<double> gamma_i(nh), beta(nh), s2(nh);
  std::vector<float> terms(size_t(na) * nh);
  std::vector<unsigned char> valid(nh);
  for (int k = 0; k < nh; k++)
    gamma_i[k] = std::atan(D.h[k] / distance);
  for (int i = 0; i < nprec; i++) {
    const double scor = midpoint - double(nsamples / 2) * precision[i];
    float M[nsamples];
    for (int j = 0; j < nsamples; j++) {
      const double gamma_c = std::atan((midpoint + (j - nsamples / 2) * precision[i]) / distance);
      for (int k = 0; k < nh; k++) {
        beta[k] = double(M_PI) + 2.0 * (gamma_i[k] - gamma_c);
        s2[k] = distance * std::tan(2.0 * gamma_c - gamma_i[k]);
        valid[k] = (s2[k] >= D.h[0] && s2[k] <= D.h[nh - 1]) ? 1 : 0;
      }
#pragma omp parallel for schedule(static)
      for (int a = 0; a < na; a++) {
        for (int k = 0; k < nh; k++) {
          if (!valid[k])
            continue;
          double ab = D.ang[a] + beta[k];
          while (ab < D.ang[0])
            ab += 2.0 * M_PI;
          while (ab > D.ang[na - 1])
            ab -= 2.0 * M_PI;
          const float p = D.interpolate(s2[k], ab);
          const float t = D.at(a, k) - p;
          terms[size_t(a) * nh + k] = t * t;
        }
      }
      // the reference sums in float, in (angle, column) order
      int count = 0;
      float sum = 0.0f;
      for (int a = 0; a < na; a++)
        for (int k = 0; k < nh; k++)
          if (valid[k]) {
            sum += terms[size_t(a) * nh + k];
            count++;
          }
      M[j] = sum / float(count);
    }
    int ind = -1;
    double min_m = 1e20;
    for (int j = 0; j < nsamples; j++)
      if (min_m > M[j]) {
        ind = j;
        min_m = M[j];
      }
    if (ind < 0)
      return std::nan("");
    midpoint = scor + ind * precision[i];
  }
  return midpoint;
}

// -log(p) with the C library's float log (diamond.cpp:442, xtek.cpp:556).
void neglog_host(const float *in, float *out, i64 n) {
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < n; i++)
    out[i] = -std::log(in[i]);
}

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p)
      cudaFree(p);
  }
  bool alloc(size_t bytes) {
    return ccpi::cuda_ok(cudaMalloc(&p, bytes ? bytes : 4), "device allocation");
  }
  float *f() { return static_cast<float *>(p); }
};

struct PlanHolder {
  ccpi_plan *p = nullptr;
  ~PlanHolder() { delete p; }
};

// Upload a sinogram, lay it out as (n_angles, n_h, n_v_padded), solve and
// download the volume.  raw_parallel: the host array is the parallel-beam
// numpy layout (na, nv, nh); otherwise it is already padded and laid out.
int solve_on_host_data(HostGeometry &G, int alg, const float *sino_host, bool raw_parallel,
                       int na, int nv, int nh, const float *x0, int niter, double lambda,
                       double *norms, float *volume) {
  PlanHolder P;
  if (ccpi::plan_create(&G.g, &P.p))
    return 2;
  const i64 V = P.p->nvox, Pn = P.p->npix;
  const i64 raw = raw_parallel ? i64(na) * nv * nh : Pn;
  DevBuf draw, dsino, dx;
  if ((raw_parallel && !draw.alloc(raw * 4)) || !dsino.alloc(Pn * 4) || !dx.alloc(V * 4))
    return 2;
  cudaStream_t st = 0;
  if (!ccpi::cuda_ok(cudaMemcpyAsync(raw_parallel ? draw.p : dsino.p, sino_host, raw * 4,
                                     cudaMemcpyHostToDevice, st),
                     "upload sinogram"))
    return 2;
  if (raw_parallel)
    ccpi::k_pack_parallel(draw.f(), dsino.f(), na, nv, nh, G.nv_pad, G.v_offset, st);
  if (x0) {
    if (!ccpi::cuda_ok(cudaMemcpyAsync(dx.p, x0, V * 4, cudaMemcpyHostToDevice, st),
                       "upload x0"))
      return 2;
  } else {
    cudaMemsetAsync(dx.p, 0, V * 4, st);
  }
  const int rc = ccpi::solve(P.p, alg, dsino.f(), dx.f(), niter, lambda, norms, 0, nullptr, 0, st);
  if (rc)
    return rc;
  if (!ccpi::cuda_ok(cudaMemcpy(volume, dx.p, V * 4, cudaMemcpyDeviceToHost), "download volume"))
    return 2;
  return 0;
}

} // namespace

namespace {
// A sinogram filter on host pixels (n_angles, n_v, n_h): -log unless the
// data are already logs, the internal layout [a][h][v], the filter, back to
// (n_angles, n_v, n_h) and, for transmission input, exp(-x) with the C
// library's expf, as the reference's filter wrapper does
// (diamond_wrapper.cpp:28-48).
template <class F>
int host_sino_filter(const char *name, const float *pixels, int na, int nv, int nh, int is_log,
                     float *out, F &&filter) {
  if (!pixels || !out || na < 1 || nv < 1 || nh < 1) {
    set_error(std::string(name) + ": need pixels (n_angles, n_v, n_h >= 1) and an output buffer");
    return 1;
  }
  const i64 n = i64(na) * nv * nh;
  std::vector<float> logged(size_t(n), 0.0f);
  if (is_log)
    std::memcpy(logged.data(), pixels, size_t(n) * 4);
  else
    neglog_host(pixels, logged.data(), n);
  DevBuf raw, sino;
  if (!raw.alloc(n * 4) || !sino.alloc(n * 4))
    return 2;
  cudaStream_t st = 0;
  if (!ccpi::cuda_ok(cudaMemcpy(raw.p, logged.data(), n * 4, cudaMemcpyHostToDevice),
                     "upload pixels"))
    return 2;
  ccpi::k_pack_parallel(raw.f(), sino.f(), na, nv, nh, nv, 0, st); // -> [a][h][v]
  const int rc = filter(sino.f(), st);
  if (rc)
    return rc;
  ccpi::k_unpack_parallel(sino.f(), raw.f(), na, nh, nv, st); // -> [a][v][h]
  if (!ccpi::cuda_ok(cudaMemcpy(logged.data(), raw.p, n * 4, cudaMemcpyDeviceToHost),
                     "download pixels"))
    return 2;
  if (is_log) {
    std::memcpy(out, logged.data(), size_t(n) * 4);
  } else {
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; i++)
      out[i] = std::exp(-logged[size_t(i)]);
  }
  return 0;
}
} // namespace

extern "C" {

const char *ccpi_last_error(void) { return ccpi::g_last_error.c_str(); }

int ccpi_version(void) { return 100; }

int ccpi_pb_grid(int na, int nv, int nh, double cor, int ppv, int dims[5]) {
  HostGeometry G;
  if (!pb_geometry(na, nv, nh, cor, ppv, nullptr, G))
    return 1;
  dims[0] = G.g.nx;
  dims[1] = G.g.ny;
  dims[2] = G.g.nz;
  dims[3] = G.nv_pad;
  dims[4] = G.v_offset;
  return 0;
}

int ccpi_pb_geometry(int na, int nv, int nh, const float *angles_deg, double cor, int ppv,
                     double *angles_rad, double *h_pixels, double *v_pixels,
                     ccpi_geometry *geometry) {
  ccpi::g_last_error.clear();
  if (!angles_deg || !angles_rad || !h_pixels || !v_pixels || !geometry) {
    set_error("ccpi_pb_geometry: null argument");
    return 1;
  }
  HostGeometry G;
  if (!pb_geometry(na, nv, nh, cor, ppv, angles_deg, G))
    return 1;
  std::copy(G.angles.begin(), G.angles.end(), angles_rad);
  std::copy(G.h.begin(), G.h.end(), h_pixels);
  std::copy(G.v.begin(), G.v.end(), v_pixels);
  *geometry = G.g;
  geometry->angles = angles_rad;
  geometry->h_pixels = h_pixels;
  geometry->v_pixels = v_pixels;
  return 0;
}

int ccpi_pb_pack(const float *d_pixels, int na, int nv, int nh, int nv_pad, int v_offset,
                 float *d_sino, void *stream) {
  ccpi::g_last_error.clear();
  if (!d_pixels || !d_sino || na < 1 || nv < 1 || nh < 1 || v_offset < 0 ||
      v_offset + nv > nv_pad) {
    set_error("ccpi_pb_pack: bad arguments");
    return 1;
  }
  // writes every element of d_sino, padding rows included (zeros)
  ccpi::k_pack_parallel(d_pixels, d_sino, na, nv, nh, nv_pad, v_offset, cudaStream_t(stream));
  return ccpi::cuda_ok(cudaGetLastError(), "ccpi_pb_pack: launch") ? 0 : 2;
}

int ccpi_pb_reconstruct(int alg, const float *pixels, int na, int nv, int nh,
                        const float *angles_deg, double cor, int ppv, int niter, int nthreads,
                        int is_log, double lambda, const float *x0, double *norms,
                        float *volume) {
  (void)nthreads;
  ccpi::g_last_error.clear();
  if (!pixels || !angles_deg || !volume) {
    set_error("ccpi_pb_reconstruct: null buffer");
    return 1;
  }
  HostGeometry G;
  if (!pb_geometry(na, nv, nh, cor, ppv, angles_deg, G))
    return 1;
  const float *src = pixels;
  std::vector<float> logged;
  if (!is_log) {
    logged.resize(size_t(na) * nv * nh);
    neglog_host(pixels, logged.data(), i64(logged.size()));
    src = logged.data();
  }
  return solve_on_host_data(G, alg, src, true, na, nv, nh, x0, niter, lambda, norms, volume);
}

int ccpi_pb_reconstruct_batched(int n, int alg, const float *const *pixels, const int *na,
                                const int *nv, const int *nh, const float *const *angles_deg,
                                const double *cor, int ppv, int niter, int is_log,
                                const double *lambda, float *const *volumes) {
  ccpi::g_last_error.clear();
  if (n < 0 || (n > 0 && (!pixels || !na || !nv || !nh || !angles_deg || !cor || !volumes))) {
    set_error("ccpi_pb_reconstruct_batched: bad arguments");
    return 1;
  }
  if (n == 0)
    return 0;
  std::vector<HostGeometry> G(n);
  std::vector<PlanHolder> P(n);
  std::vector<i64> off_raw(n + 1, 0), off_sino(n + 1, 0), off_x(n + 1, 0);
  for (int i = 0; i < n; i++) {
    if (!pixels[i] || !angles_deg[i] || !volumes[i]) {
      set_error("ccpi_pb_reconstruct_batched: null buffer for problem " + std::to_string(i));
      return 1;
    }
    if (!pb_geometry(na[i], nv[i], nh[i], cor[i], ppv, angles_deg[i], G[i]))
      return 1;
    if (ccpi::plan_create(&G[i].g, &P[i].p))
      return 2;
    // 16-byte aligned sub-buffers
    auto up4 = [](i64 x) { return (x + 3) & ~i64(3); };
    off_raw[i + 1] = off_raw[i] + up4(i64(na[i]) * nv[i] * nh[i]);
    off_sino[i + 1] = off_sino[i] + up4(P[i].p->npix);
    off_x[i + 1] = off_x[i] + up4(P[i].p->nvox);
  }
  DevBuf draw, dsino, dx;
  if (!draw.alloc(off_raw[n] * 4) || !dsino.alloc(off_sino[n] * 4) || !dx.alloc(off_x[n] * 4))
    return 2;
  cudaStream_t st = 0;
  std::vector<float> logged;
  std::vector<const float *> ds(n);
  std::vector<float *> dv(n);
  std::vector<const ccpi_plan *> pl(n);
  for (int i = 0; i < n; i++) {
    const i64 raw = i64(na[i]) * nv[i] * nh[i];
    const float *src = pixels[i];
    if (!is_log) {
      logged.resize(size_t(raw));
      neglog_host(pixels[i], logged.data(), raw);
      src = logged.data();
    }
    float *r = draw.f() + off_raw[i];
    // synchronous copy: `logged` is reused by the next problem
    if (!ccpi::cuda_ok(cudaMemcpy(r, src, raw * 4, cudaMemcpyHostToDevice), "upload sinogram"))
      return 2;
    float *s = dsino.f() + off_sino[i];
    ccpi::k_pack_parallel(r, s, na[i], nv[i], nh[i], G[i].nv_pad, G[i].v_offset, st);
    ds[i] = s;
    dv[i] = dx.f() + off_x[i];
    pl[i] = P[i].p;
  }
  cudaMemsetAsync(dx.p, 0, off_x[n] * 4, st);
  const int rc = ccpi::solve_batched(n, pl.data(), alg, ds.data(), dv.data(), niter, lambda, st);
  if (rc)
    return rc;
  for (int i = 0; i < n; i++)
    if (!ccpi::cuda_ok(cudaMemcpy(volumes[i], dv[i], P[i].p->nvox * 4, cudaMemcpyDeviceToHost),
                       "download volume"))
      return 2;
  return 0;
}

int ccpi_pb_aml_ring_artefacts(const float *pixels, int na, int nv, int nh, float param_n,
                               float param_r, int num_series, float *out) {
  ccpi::g_last_error.clear();
  if (!pixels || !out || na < 1 || nv < 1 || nh < 2) {
    set_error("ccpi_pb_aml_ring_artefacts: need pixels (n_angles >= 1, n_v >= 1, n_h >= 2) "
              "and an output buffer");
    return 1;
  }
  const i64 n = i64(na) * nv * nh;
  // p = -log(pixels) with the C library's logf (diamond_wrapper.cpp:28-34)
  std::vector<float> logged(size_t(n), 0.0f);
  neglog_host(pixels, logged.data(), n);
  DevBuf raw, sino;
  if (!raw.alloc(n * 4) || !sino.alloc(n * 4))
    return 2;
  cudaStream_t st = 0;
  if (!ccpi::cuda_ok(cudaMemcpy(raw.p, logged.data(), n * 4, cudaMemcpyHostToDevice),
                     "upload pixels"))
    return 2;
  ccpi::k_pack_parallel(raw.f(), sino.f(), na, nv, nh, nv, 0, st); // -> [a][h][v]
  const int rc = ccpi::aml_ring_filter(sino.f(), na, nh, nv, param_n, param_r, num_series, st);
  if (rc)
    return rc;
  ccpi::k_unpack_parallel(sino.f(), raw.f(), na, nh, nv, st); // -> [a][v][h]
  if (!ccpi::cuda_ok(cudaMemcpy(logged.data(), raw.p, n * 4, cudaMemcpyDeviceToHost),
                     "download pixels"))
    return 2;
  // back to transmission with the C library's expf (diamond_wrapper.cpp:45-48)
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < n; i++)
    out[i] = std::exp(-logged[size_t(i)]);
  return 0;
}

int ccpi_ring_filter_aml(float *d_sino, int n_angles, int n_h, int n_v, double param_n,
                         double param_r, int num_series, void *stream) {
  ccpi::g_last_error.clear();
  return ccpi::aml_ring_filter(d_sino, n_angles, n_h, n_v, param_n, param_r, num_series,
                               cudaStream_t(stream));
}

int ccpi_pb_high_peaks(const float *pixels, int na, int nv, int nh, double jump, int num_pix,
                       int is_pixels_in_log, float *out) {
  ccpi::g_last_error.clear();
  if (pixels && out && na >= 1 && ccpi::high_peaks_check(na, jump, num_pix))
    return 1;
  return host_sino_filter("ccpi_pb_high_peaks", pixels, na, nv, nh, is_pixels_in_log, out,
                          [&](float *d, cudaStream_t st) {
                            return ccpi::high_peaks_filter(d, na, nh, nv, jump, num_pix, st);
                          });
}

int ccpi_pb_column_ring_artefacts(const float *pixels, int na, int nv, int nh,
                                  int is_pixels_in_log, float *out) {
  ccpi::g_last_error.clear();
  return host_sino_filter("ccpi_pb_column_ring_artefacts", pixels, na, nv, nh, is_pixels_in_log,
                          out, [&](float *d, cudaStream_t st) {
                            return ccpi::column_ring_filter(d, na, nh, nv, st);
                          });
}

int ccpi_high_peaks(float *d_sino, int n_angles, int n_h, int n_v, double jump, int num_pix,
                    void *stream) {
  ccpi::g_last_error.clear();
  return ccpi::high_peaks_filter(d_sino, n_angles, n_h, n_v, jump, num_pix,
                                 cudaStream_t(stream));
}

int ccpi_ring_filter_column(float *d_sino, int n_angles, int n_h, int n_v, void *stream) {
  ccpi::g_last_error.clear();
  return ccpi::column_ring_filter(d_sino, n_angles, n_h, n_v, cudaStream_t(stream));
}

int ccpi_pb_forward_project(const float *volume, int vx, int vy, int vz, const float *angles_deg,
                            int na, int ppv, float *out, int out_dims[3]) {
  ccpi::g_last_error.clear();
  const int width = vx > vy ? vx : vy;
  HostGeometry G;
  if (!pb_geometry(na, vz, width, double(width) / 2.0, ppv, angles_deg, G))
    return 1;
  out_dims[0] = na;
  out_dims[1] = G.nv_pad;
  out_dims[2] = width;
  if (!out)
    return 0;
  // the volume's own shape, centred, voxel size = resolution (diamond.cpp:453-477)
  G.g.nx = vx;
  G.g.ny = vy;
  G.g.nz = vz;
  const int nn[3] = {vx, vy, vz};
  for (int i = 0; i < 3; i++)
    G.g.origin[i] = -G.g.voxel_size[i] * double(nn[i]) / 2.0;
  PlanHolder P;
  if (ccpi::plan_create(&G.g, &P.p))
    return 2;
  DevBuf dv, dp, dq;
  const i64 V = P.p->nvox, Pn = P.p->npix;
  if (!dv.alloc(V * 4) || !dp.alloc(Pn * 4) || !dq.alloc(Pn * 4))
    return 2;
  cudaMemcpy(dv.p, volume, V * 4, cudaMemcpyHostToDevice);
  ccpi::Epi e{};
  if (ccpi::forward(P.p, dv.f(), dp.f(), ccpi::EPI_STORE, e, 0))
    return 3;
  ccpi::k_unpack_parallel(dp.f(), dq.f(), na, width, G.nv_pad, 0);
  if (!ccpi::cuda_ok(cudaMemcpy(out, dq.p, Pn * 4, cudaMemcpyDeviceToHost), "pb_forward_project"))
    return 2;
  return 0;
}

int ccpi_pb_backward_project(const float *stack, int na, int nv, int nh, const float *angles_deg,
                             double cor, int ppv, float *out, int out_dims[3]) {
  ccpi::g_last_error.clear();
  HostGeometry G;
  if (!pb_geometry(na, nv, nh, cor, ppv, angles_deg, G))
    return 1;
  out_dims[0] = G.g.nx;
  out_dims[1] = G.g.ny;
  out_dims[2] = G.g.nz;
  if (!out)
    return 0;
  PlanHolder P;
  if (ccpi::plan_create(&G.g, &P.p))
    return 2;
  DevBuf draw, dp, dv;
  const i64 V = P.p->nvox, Pn = P.p->npix;
  if (!draw.alloc(i64(na) * nv * nh * 4) || !dp.alloc(Pn * 4) || !dv.alloc(V * 4))
    return 2;
  cudaMemcpy(draw.p, stack, i64(na) * nv * nh * 4, cudaMemcpyHostToDevice);
  // the wrapper copies the stack's rows to padded rows [0, n_v) without the
  // centring offset (diamond_wrapper.cpp:702-710)
  ccpi::k_pack_parallel(draw.f(), dp.f(), na, nv, nh, G.nv_pad, 0, 0);
  ccpi::Epi e{};
  if (ccpi::backward(P.p, dp.f(), dv.f(), ccpi::EPI_STORE, e, 0))
    return 3;
  if (!ccpi::cuda_ok(cudaMemcpy(out, dv.p, V * 4, cudaMemcpyDeviceToHost), "pb_backward_project"))
    return 2;
  return 0;
}

int ccpi_cb_grid(int na, int nh, int nv, int ppv, double s2s, double s2d, double px_h,
                 double px_v, double mask_radius, int dims[5], double geom[5]) {
  HostGeometry G;
  if (!cb_geometry(na, nh, nv, ppv, s2s, s2d, px_h, px_v, mask_radius, nullptr, G))
    return 1;
  dims[0] = G.g.nx;
  dims[1] = G.g.ny;
  dims[2] = G.g.nz;
  dims[3] = G.nv_pad;
  dims[4] = G.v_offset;
  geom[0] = G.g.voxel_size[0];
  geom[1] = G.g.voxel_size[2];
  geom[2] = G.g.origin[0];
  geom[3] = G.g.origin[1];
  geom[4] = G.g.origin[2];
  return 0;
}

int ccpi_cb_find_centre(const float *sino, int na, int nh, int nvp, const float *angles_deg,
                        double s2s, double s2d, double px_h, double *y_centre) {
  if (!sino || !angles_deg || na < 1 || nh < 2 || nvp < 1) {
    set_error("ccpi_cb_find_centre: bad arguments");
    return 1;
  }
  std::vector<double> h(nh), ang;
  h[0] = -((nh - 1) * px_h) / 2.0;
  for (int i = 1; i < nh; i++)
    h[i] = h[0] + double(i) * px_h;
  degrees_to_radians(angles_deg, na, ang);
  CentreData D{sino, na, nh, nvp, nvp / 2, h.data(), ang.data(), true};
  for (int a = 1; a < na; a++)
    if (!(ang[a] > ang[a - 1]))
      D.sorted_angles = false;
  const double source_x = -s2s, detector_x = s2d + source_x;
  const double distance = detector_x - source_x;
  const double mid = find_centre_midpoint(D, distance);
  if (std::isnan(mid)) {
    set_error("ccpi_cb_find_centre: no detector column inside the search window");
    return 3;
  }
  *y_centre = mid * source_x / distance;
  return 0;
}

int ccpi_cb_reconstruct(int alg, const float *pixels, int na, int nh, int nv,
                        const float *angles_deg, int ppv, double s2s, double s2d, double px_h,
                        double px_v, double mask_radius, int niter, int nthreads, int is_log,
                        double lambda, double *norms, float *volume) {
  (void)nthreads;
  ccpi::g_last_error.clear();
  if (!pixels || !angles_deg || !volume) {
    set_error("ccpi_cb_reconstruct: null buffer");
    return 1;
  }
  HostGeometry G;
  if (!cb_geometry(na, nh, nv, ppv, s2s, s2d, px_h, px_v, mask_radius, angles_deg, G))
    return 1;
  // read_scans (xtek.cpp:519-563): pad rows, -log, then the centre search
  std::vector<float> packed(size_t(na) * nh * G.nv_pad, 0.0f);
  for (i64 ah = 0; ah < i64(na) * nh; ah++) {
    const float *in = pixels + ah * nv;
    float *o = packed.data() + ah * G.nv_pad + G.v_offset;
    if (is_log)
      std::memcpy(o, in, sizeof(float) * nv);
    else
      for (int k = 0; k < nv; k++)
        o[k] = -std::log(in[k]);
  }
  double yc = 0.0;
  if (ccpi_cb_find_centre(packed.data(), na, nh, G.nv_pad, angles_deg, s2s, s2d, px_h, &yc))
    return 3;
  G.g.source[1] += yc;
  for (auto &hh : G.h)
    hh += yc;
  G.bind();
  return solve_on_host_data(G, alg, packed.data(), false, na, G.nv_pad, nh, nullptr, niter,
                            lambda, norms, volume);
}

int ccpi_cb_create_sinogram(const ccpi_geometry *geometry, const float *volume, float *out) {
  ccpi::g_last_error.clear();
  if (!geometry || geometry->kind != CCPI_CONE || !volume || !out) {
    set_error("ccpi_cb_create_sinogram: need a cone geometry and buffers");
    return 1;
  }
  PlanHolder P;
  if (ccpi::plan_create(geometry, &P.p))
    return 2;
  DevBuf dv, dp;
  const i64 V = P.p->nvox, Pn = P.p->npix;
  if (!dv.alloc(V * 4) || !dp.alloc(Pn * 4))
    return 2;
  cudaMemcpy(dv.p, volume, V * 4, cudaMemcpyHostToDevice);
  ccpi::Epi e{};
  if (ccpi::forward(P.p, dv.f(), dp.f(), ccpi::EPI_STORE, e, 0))
    return 3;
  if (!ccpi::cuda_ok(cudaMemcpy(out, dp.p, Pn * 4, cudaMemcpyDeviceToHost), "create_sinogram"))
    return 2;
  return 0;
}

int ccpi_reconstruct(const ccpi_geometry *geometry, int alg, const float *sino, int niter,
                     double regularize, double *norms, float *volume) {
  return ccpi_reconstruct_flags(geometry, alg, sino, niter, regularize, norms, volume, 0);
}

int ccpi_reconstruct_flags(const ccpi_geometry *geometry, int alg, const float *sino, int niter,
                           double regularize, double *norms, float *volume, int flags) {
  ccpi::g_last_error.clear();
  if (!geometry || !sino || !volume) {
    set_error("ccpi_reconstruct: need a geometry and host buffers");
    return 1;
  }
  if (alg < CCPI_CGLS || alg > CCPI_CGLS_TV || niter < 0) {
    set_error("ccpi_reconstruct: unknown algorithm or negative iteration count");
    return 1;
  }
  if (flags & ~CCPI_RECON_CONE_SCATTER) {
    set_error("ccpi_reconstruct_flags: unknown flag bits");
    return 1;
  }
  PlanHolder P;
  if (ccpi::plan_create(geometry, &P.p))
    return 2;
  if ((flags & CCPI_RECON_CONE_SCATTER) && geometry->kind == CCPI_CONE &&
      ccpi::set_cone_backprojector(P.p, 1))
    return 1;
  const i64 V = P.p->nvox, Pn = P.p->npix;
  DevBuf dsino, dx;
  if (!dsino.alloc(Pn * 4) || !dx.alloc(V * 4))
    return 2;
  cudaStream_t st = 0;
  if (!ccpi::cuda_ok(cudaMemcpyAsync(dsino.p, sino, Pn * 4, cudaMemcpyHostToDevice, st),
                     "ccpi_reconstruct: upload sinogram"))
    return 2;
  cudaMemsetAsync(dx.p, 0, V * 4, st);
  const int rc =
      ccpi::solve(P.p, alg, dsino.f(), dx.f(), niter, regularize, norms, 0, nullptr, 0, st);
  if (rc)
    return rc;
  if (!ccpi::cuda_ok(cudaMemcpy(volume, dx.p, V * 4, cudaMemcpyDeviceToHost),
                     "ccpi_reconstruct: download volume"))
    return 2;
  return 0;
}

int ccpi_plan_create(const ccpi_geometry *geometry, ccpi_plan **plan) {
  ccpi::g_last_error.clear();
  if (!plan) {
    set_error("ccpi_plan_create: null output");
    return 1;
  }
  return ccpi::plan_create(geometry, plan);
}

void ccpi_plan_destroy(ccpi_plan *plan) { delete plan; }

int ccpi_plan_autotune(ccpi_plan *plan, void *stream, int chosen[2]) {
  ccpi::g_last_error.clear();
  if (!plan) {
    set_error("ccpi_plan_autotune: null plan");
    return 1;
  }
  return ccpi::plan_autotune(plan, cudaStream_t(stream), chosen);
}

int ccpi_plan_set_cone_backprojector(ccpi_plan *plan, int scatter) {
  ccpi::g_last_error.clear();
  if (!plan) {
    set_error("ccpi_plan_set_cone_backprojector: null plan");
    return 1;
  }
  return ccpi::set_cone_backprojector(plan, scatter);
}

long long ccpi_plan_voxels(const ccpi_plan *plan) { return plan ? plan->nvox : 0; }
long long ccpi_plan_pixels(const ccpi_plan *plan) { return plan ? plan->npix : 0; }

// Device buffers are read and written as float4 rows: 16-byte alignment.
bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int ccpi_forward(const ccpi_plan *plan, const float *d_volume, float *d_sino, void *stream) {
  if (!plan || !d_volume || !d_sino) {
    set_error("ccpi_forward: null argument");
    return 1;
  }
  if (!aligned16(d_volume) || !aligned16(d_sino)) {
    set_error("ccpi_forward: device buffers must be 16-byte aligned");
    return 1;
  }
  ccpi::Epi e{};
  if (ccpi::forward(plan, d_volume, d_sino, ccpi::EPI_STORE, e, cudaStream_t(stream)))
    return 3;
  return ccpi::cuda_ok(cudaGetLastError(), "ccpi_forward") ? 0 : 2;
}

int ccpi_backward(const ccpi_plan *plan, const float *d_sino, float *d_volume, void *stream) {
  if (!plan || !d_volume || !d_sino) {
    set_error("ccpi_backward: null argument");
    return 1;
  }
  if (!aligned16(d_volume) || !aligned16(d_sino)) {
    set_error("ccpi_backward: device buffers must be 16-byte aligned");
    return 1;
  }
  ccpi::Epi e{};
  if (ccpi::backward(plan, d_sino, d_volume, ccpi::EPI_STORE, e, cudaStream_t(stream)))
    return 3;
  return ccpi::cuda_ok(cudaGetLastError(), "ccpi_backward") ? 0 : 2;
}

// n projections of one plan: cone beam in one launch per direction (the
// rays' walks and the columns' band limits are shared by the batch),
// parallel beam one launch per item.
static int project_batch(const char *what, const ccpi_plan *plan, int n, const float *in,
                         float *out, bool fwd, void *stream) {
  if (!plan || !in || !out || n < 0) {
    set_error(std::string(what) + ": null argument or negative batch");
    return 1;
  }
  const i64 nin = fwd ? plan->nvox : plan->npix, nout = fwd ? plan->npix : plan->nvox;
  if (!aligned16(in) || !aligned16(out) ||
      (n > 1 && ((nin * 4) % 16 != 0 || (nout * 4) % 16 != 0))) {
    set_error(std::string(what) + ": every item must start on a 16-byte boundary");
    return 1;
  }
  const cudaStream_t st = cudaStream_t(stream);
  ccpi::Epi e{};
  // cone: one launch for the batch, except back projection on a plan set to
  // the ray-driven scatter, which runs the scatter item by item
  if (plan->g.kind == CCPI_CONE && n > 0 && (fwd || !plan->g.tune_scatter)) {
    const int rc = fwd ? ccpi::cb_forward(plan->g, in, out, ccpi::EPI_STORE, e, plan->hrange,
                                          plan->fp_grid, st, n)
                       : ccpi::cb_backward(plan->g, in, out, ccpi::EPI_STORE, e, plan->err, st, n);
    if (rc)
      return 3;
  } else {
    for (int b = 0; b < n; b++) {
      const float *src = in + i64(b) * nin;
      float *dst = out + i64(b) * nout;
      if (fwd ? ccpi::forward(plan, src, dst, ccpi::EPI_STORE, e, st)
              : ccpi::backward(plan, src, dst, ccpi::EPI_STORE, e, st))
        return 3;
    }
  }
  return ccpi::cuda_ok(cudaGetLastError(), what) ? 0 : 2;
}

int ccpi_forward_batch(const ccpi_plan *plan, int n, const float *d_volumes, float *d_sinos,
                       void *stream) {
  return project_batch("ccpi_forward_batch", plan, n, d_volumes, d_sinos, true, stream);
}

int ccpi_backward_batch(const ccpi_plan *plan, int n, const float *d_sinos, float *d_volumes,
                        void *stream) {
  return project_batch("ccpi_backward_batch", plan, n, d_sinos, d_volumes, false, stream);
}

size_t ccpi_solve_workspace_bytes(const ccpi_plan *plan, int alg, int niterations) {
  return plan ? ccpi::solve_workspace_bytes(plan, alg, niterations) : 0;
}

int ccpi_solve(const ccpi_plan *plan, int alg, const float *d_sino, float *d_x, int niterations,
               double regularize, double *h_norms, int flags, void *d_workspace,
               size_t workspace_bytes, void *stream) {
  ccpi::g_last_error.clear();
  if (!plan || !d_sino || !d_x) {
    set_error("ccpi_solve: null argument");
    return 1;
  }
  if (!aligned16(d_sino) || !aligned16(d_x) || (d_workspace && !aligned16(d_workspace))) {
    set_error("ccpi_solve: device buffers must be 16-byte aligned");
    return 1;
  }
  return ccpi::solve(plan, alg, d_sino, d_x, niterations, regularize, h_norms, flags,
                     d_workspace, workspace_bytes, cudaStream_t(stream));
}

int ccpi_solve_batched(int n, const ccpi_plan *const *plans, int alg, const float *const *d_sino,
                       float *const *d_x, int niterations, const double *regularize,
                       void *stream) {
  ccpi::g_last_error.clear();
  if (n < 0 || (n > 0 && (!plans || !d_sino || !d_x))) {
    set_error("ccpi_solve_batched: bad arguments");
    return 1;
  }
  for (int i = 0; i < n; i++)
    if (!plans[i] || !aligned16(d_sino[i]) || !aligned16(d_x[i])) {
      set_error("ccpi_solve_batched: null plan or device buffer not 16-byte aligned");
      return 1;
    }
  return ccpi::solve_batched(n, plans, alg, d_sino, d_x, niterations, regularize,
                             cudaStream_t(stream));
}

int ccpi_session_create(const ccpi_plan *plan, int alg, const float *d_sino, float *d_x,
                        double regularize, int max_iterations, int flags, void *stream,
                        ccpi_session **session) {
  ccpi::g_last_error.clear();
  if (!plan || !d_sino || !d_x || !session) {
    set_error("ccpi_session_create: null argument");
    return 1;
  }
  if (!aligned16(d_sino) || !aligned16(d_x)) {
    set_error("ccpi_session_create: device buffers must be 16-byte aligned");
    return 1;
  }
  int rc = 0;
  *session = static_cast<ccpi_session *>(ccpi::session_create(
      plan, alg, d_sino, d_x, regularize, max_iterations, flags, cudaStream_t(stream), &rc));
  return rc;
}

int ccpi_session_run(ccpi_session *session, int niterations) {
  if (!session) {
    set_error("ccpi_session_run: null session");
    return 1;
  }
  return ccpi::session_run(session, niterations);
}

int ccpi_session_finish(ccpi_session *session, double *h_norms) {
  if (!session) {
    set_error("ccpi_session_finish: null session");
    return 1;
  }
  return ccpi::session_finish(session, h_norms);
}

void ccpi_session_destroy(ccpi_session *session) {
  if (session)
    ccpi::session_destroy(session);
}

int ccpi_shard_create(const ccpi_plan *plan, int alg, const float *d_sino, float *d_x,
                      double regularize, int max_iterations, double *d_sum, float *d_edges,
                      const float *d_halo_lo, const float *d_halo_hi, void *stream,
                      ccpi_shard **shard) {
  ccpi::g_last_error.clear();
  if (!plan || !d_sino || !d_x || !shard) {
    set_error("ccpi_shard_create: null argument");
    return 1;
  }
  int rc = 0;
  *shard = static_cast<ccpi_shard *>(ccpi::shard_create(plan, alg, d_sino, d_x, regularize,
                                                         max_iterations, d_sum, d_edges,
                                                         d_halo_lo, d_halo_hi,
                                                         cudaStream_t(stream), &rc));
  return rc;
}

int ccpi_shard_stage(ccpi_shard *shard, int stage) {
  ccpi::g_last_error.clear();
  if (!shard) {
    set_error("ccpi_shard_stage: null shard");
    return 1;
  }
  return ccpi::shard_stage(shard, stage);
}

int ccpi_shard_finish(ccpi_shard *shard, double *h_norms) {
  ccpi::g_last_error.clear();
  if (!shard) {
    set_error("ccpi_shard_finish: null shard");
    return 1;
  }
  return ccpi::shard_finish(shard, h_norms);
}

void ccpi_shard_destroy(ccpi_shard *shard) {
  if (shard)
    ccpi::shard_destroy(shard);
}

} // extern "C"
