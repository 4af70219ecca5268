// Plans (device geometry tables), projector dispatch and the solver loops.
//
// Solvers restate Core/src/Algorithms/cgls.cpp (cgls_base + cgls_3d,
// cgls_regularize), sirt.cpp and mlem.cpp.  Every iteration runs without a
// host round trip: the CGLS step scalars live in device memory (FP64), the
// SIRT/MLEM updates and the sums of squares are fused into the projector
// epilogues, and one iteration is captured once as a CUDA graph and
// replayed.  CCPI_SOLVE_PLAIN instead launches each iteration from the
// host and reads the scalars back every iteration, the way a host-driven
// port of the reference's loop runs; it is kept as the comparison path.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ccpi_b200.h"
#include "engine.h"
#include "kernels.h"

ccpi_plan::~ccpi_plan() {
  for (void *b : bufs)
    cudaFree(b);
}

namespace ccpi {

thread_local std::string g_last_error;

void set_error(const std::string &m) { g_last_error = m; }

bool cuda_ok(cudaError_t e, const char *what) {
  if (e == cudaSuccess)
    return true;
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  // the failure is reported through the status and ccpi_last_error(); clear
  // the runtime's last-error slot so that a recoverable failure (an
  // allocation refused for lack of memory) does not surface later in the
  // caller's own error checks
  cudaGetLastError();
  return false;
}

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
    return 148;
  return n;
}

namespace {

template <class T> T *upload(ccpi_plan *p, const std::vector<T> &h) {
  if (h.empty())
    return nullptr;
  void *d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(T)) != cudaSuccess)
    return nullptr;
  p->bufs.push_back(d);
  cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
  return static_cast<T *>(d);
}

bool evenly_increasing(const double *p, int n) {
  for (int i = 1; i < n; i++)
    if (!(p[i] > p[i - 1]))
      return false;
  return true;
}

} // namespace

int plan_create(const ccpi_geometry *gi, ccpi_plan **out) {
  *out = nullptr;
  if (!gi || (gi->kind != CCPI_PARALLEL && gi->kind != CCPI_CONE)) {
    set_error("ccpi_plan_create: geometry kind must be CCPI_PARALLEL or CCPI_CONE");
    return 1;
  }
  if (gi->n_angles < 1 || gi->n_h < 2 || gi->n_v < 1 || gi->nx < 1 || gi->ny < 1 ||
      gi->nz < 1 || !gi->angles || !gi->h_pixels || !gi->v_pixels) {
    set_error("ccpi_plan_create: empty geometry (need >= 1 angle, >= 2 detector "
              "columns, >= 1 row and a non-empty voxel grid)");
    return 1;
  }
  if (!evenly_increasing(gi->h_pixels, gi->n_h) || !evenly_increasing(gi->v_pixels, gi->n_v)) {
    set_error("ccpi_plan_create: detector coordinates must be increasing");
    return 1;
  }
  for (int i = 0; i < 3; i++)
    if (!(gi->voxel_size[i] > 0.0)) {
      set_error("ccpi_plan_create: voxel sizes must be positive");
      return 1;
    }
  if (i64(gi->nx) * gi->ny * gi->nz > (i64(1) << 40) ||
      i64(gi->n_angles) * gi->n_h * gi->n_v > (i64(1) << 40)) {
    set_error("ccpi_plan_create: problem too large");
    return 1;
  }
  if (i64(gi->nx) * gi->ny >= (i64(1) << 31)) {
    set_error("ccpi_plan_create: more than 2^31 voxel columns");
    return 1;
  }
  ccpi_plan *p = new ccpi_plan();
  cudaGetDevice(&p->device);
  Geom &g = p->g;
  std::memset(&g, 0, sizeof(g));
  g.kind = gi->kind;
  g.na = gi->n_angles;
  g.nh = gi->n_h;
  g.nv = gi->n_v;
  g.nx = gi->nx;
  g.ny = gi->ny;
  g.nz = gi->nz;
  for (int i = 0; i < 3; i++) {
    g.origin[i] = gi->origin[i];
    g.size[i] = gi->voxel_size[i];
  }
  p->nvox = i64(g.nx) * g.ny * g.nz;
  p->npix = i64(g.na) * g.nh * g.nv;
  const int na = g.na, nh = g.nh, nv = g.nv, nz = g.nz;
  std::vector<double> ca(na), sa(na), hp(gi->h_pixels, gi->h_pixels + nh),
      vp(gi->v_pixels, gi->v_pixels + nv);
  for (int a = 0; a < na; a++) {
    // the host C library's cos/sin, as the reference evaluates them
    ca[a] = std::cos(gi->angles[a]);
    sa[a] = std::sin(gi->angles[a]);
  }
  g.cosA = upload(p, ca);
  g.sinA = upload(p, sa);
  g.hpix = upload(p, hp);
  g.vpix = upload(p, vp);
  bool ok = g.cosA && g.sinA && g.hpix && g.vpix;
  if (g.kind == CCPI_PARALLEL) {
    // p2D.cpp:477-494 forward constants
    g.det_x = 2.0 * std::max(std::abs(g.origin[0]),
                             std::max(std::abs(g.origin[1]), std::abs(g.origin[2])));
    g.d_conv = float(3.0 * g.det_x);
    g.ihp = 1.0 / (hp[1] - hp[0]);
    g.hp0 = hp[0] / (hp[1] - hp[0]);
    // p2D.cpp:995-1049 per-angle trapezoid tables of the (0,0) voxel
    std::vector<double> yoff(na), ioff(na), blen(na);
    const double o0 = g.origin[0], o1 = g.origin[1], d0 = g.size[0], d1 = g.size[1];
    for (int a = 0; a < na; a++) {
      const double c = ca[a], s = sa[a];
      const double y00 = o1 * c - o0 * s;
      const double y01 = (o1 + d1) * c - o0 * s;
      const double y10 = o1 * c - (o0 + d0) * s;
      const double y11 = (o1 + d1) * c - (o0 + d0) * s;
      double ymin, ybot;
      if (c > 0.0) {
        if (s > 0.0) {
          ymin = y10;
          ybot = (y11 < y00) ? y11 : y00;
        } else {
          ymin = y00;
          ybot = (y01 < y10) ? y01 : y10;
        }
      } else {
        if (s > 0.0) {
          ymin = y11;
          ybot = (y01 < y10) ? y01 : y10;
        } else {
          ymin = y01;
          ybot = (y11 < y00) ? y11 : y00;
        }
      }
      yoff[a] = ybot - ymin;
      ioff[a] = 1.0 / yoff[a];
      blen[a] = (std::abs(c) > std::abs(s)) ? d0 / std::abs(c) : d1 / std::abs(s);
    }
    g.yoff = upload(p, yoff);
    g.ioff = upload(p, ioff);
    g.blen = upload(p, blen);
    // p2D.cpp:22-61 row -> slice mapping
    std::vector<int> map(nv), vlo(nz, 0), vhi(nz, 0);
    for (int v = 0; v < nv; v++)
      map[v] = int(std::floor((vp[v] - g.origin[2]) / g.size[2]));
    g.map_type = 0;
    for (int per : {1, 2, 4}) {
      bool same = true;
      for (int v = 0; v < nv && same; v++)
        same = map[v] == v / per;
      // the fast paths index the column without a bound: rows must land in it
      if (same && map[nv - 1] < nz) {
        g.map_type = per;
        break;
      }
    }
    // rows of each slice, in row order (the mapping is non-decreasing)
    for (int z = 0; z < nz; z++) {
      vlo[z] = nv;
      vhi[z] = nv;
    }
    for (int v = nv - 1; v >= 0; v--)
      if (map[v] >= 0 && map[v] < nz) {
        if (vhi[map[v]] == nv && vlo[map[v]] == nv)
          vhi[map[v]] = v + 1;
        vlo[map[v]] = v;
      }
    for (int z = 0; z < nz; z++)
      if (vlo[z] == nv)
        vhi[z] = nv;
    g.map = upload(p, map);
    g.vlo = upload(p, vlo);
    g.vhi = upload(p, vhi);
    ok = ok && g.yoff && g.ioff && g.blen && g.map && g.vlo && g.vhi;
    p->fp_grid = pb_fp_ctas(g);
    ok = ok && pb_prepare() == 0;
    p->bp_parts = pb_bp_tiles(g);
  } else {
    if (nv < 2) {
      set_error("ccpi_plan_create: cone beam needs at least 2 detector rows");
      delete p;
      return 1;
    }
    const double sx = gi->source[0], sy = gi->source[1], sz = gi->source[2];
    g.src[0] = sx;
    g.src[1] = sy;
    g.src[2] = sz;
    g.detx = gi->detector_x;
    // c2D.cpp:480-492: first row above the source
    g.mid = -1;
    for (int i = 0; i < nv; i++)
      if (vp[i] > sz) {
        g.mid = i;
        break;
      }
    if (g.mid <= 0) {
      set_error("ccpi_plan_create: the source height must lie strictly inside the "
                "detector's row range");
      delete p;
      return 1;
    }
    g.cl = g.detx - sx;
    const double step = hp[1] - hp[0];
    g.cipix = 1.0 / step;
    g.chpix0 = (sy - hp[0]) / step;
    std::vector<double> p1x(na), p1y(na), cdx(na), sdx(na);
    for (int a = 0; a < na; a++) {
      p1x[a] = ca[a] * sx - sa[a] * sy;
      p1y[a] = sa[a] * sx + ca[a] * sy;
      cdx[a] = ca[a] * g.detx;
      sdx[a] = sa[a] * g.detx;
    }
    g.p1x = upload(p, p1x);
    g.p1y = upload(p, p1y);
    g.cdx = upload(p, cdx);
    g.sdx = upload(p, sdx);
    // c2D.cpp:495-516 and :993-1010 tables
    std::vector<float> dconv(size_t(nh) * nv), dz(nv), iz(nv), vz(nz + 1);
    const double x2 = (g.detx - sx) * (g.detx - sx);
    for (int i = 0; i < nh; i++) {
      const double xy2 = x2 + (hp[i] - sy) * (hp[i] - sy);
      for (int j = 0; j < nv; j++)
        dconv[size_t(i) * nv + j] = float(std::sqrt(xy2 + (vp[j] - sz) * (vp[j] - sz)));
    }
    for (int i = 0; i < nv; i++) {
      dz[i] = float(vp[i] - sz);
      iz[i] = float(1.0 / double(dz[i]));
    }
    for (int i = 0; i <= nz; i++)
      vz[i] = float(g.origin[2] + double(i) * g.size[2] - sz);
    g.dconv = upload(p, dconv);
    g.dz = upload(p, dz);
    g.iz = upload(p, iz);
    g.vz = upload(p, vz);
    g.inv_dz = float(1.0 / g.size[2]);
    g.pzbz = float((sz - g.origin[2]) / g.size[2]);
    g.pzbz1 = float(double(g.pzbz) + 1.0);
    const double v_step = vp[1] - vp[0];
    g.pzdv = float((sz - vp[0]) / v_step);
    g.z1 = float((g.origin[2] + g.size[2] - sz) / v_step);
    g.znm = float((g.origin[2] + double(nz - 1) * g.size[2] - sz) / v_step);
    g.pzdeps = float(double(g.pzdv) * (1.0 + double(kEps)));
    // c2D.cpp:558-600: detector columns that can see the whole volume
    std::vector<int2> hr(na);
    const double x0 = g.origin[0], xn = g.origin[0] + double(g.nx) * g.size[0];
    const double y0 = g.origin[1], yn = g.origin[1] + double(g.ny) * g.size[1];
    for (int a = 0; a < na; a++) {
      const double c = ca[a], s = sa[a];
      const double dx0 = x0 - p1x[a], dy0 = y0 - p1y[a], dxn = xn - p1x[a], dyn = yn - p1y[a];
      const double cx0 = c * x0 - sx, cxn = c * xn - sx, sy0 = s * y0, syn = s * yn;
      double y00, y01, y10, y11;
      if (std::abs(s) > std::abs(c)) {
        const double il = g.cl / s;
        y00 = (c - dx0 / (sy0 + cx0)) * il;
        y01 = (c - dx0 / (syn + cx0)) * il;
        y10 = (c - dxn / (sy0 + cxn)) * il;
        y11 = (c - dxn / (syn + cxn)) * il;
      } else {
        const double il = g.cl / c;
        y00 = (-s + dy0 / (cx0 + sy0)) * il;
        y01 = (-s + dyn / (cx0 + syn)) * il;
        y10 = (-s + dy0 / (cxn + sy0)) * il;
        y11 = (-s + dyn / (cxn + syn)) * il;
      }
      const int h00 = int(std::floor(y00 * g.cipix + g.chpix0));
      const int h01 = int(std::floor(y01 * g.cipix + g.chpix0));
      const int h10 = int(std::floor(y10 * g.cipix + g.chpix0));
      const int h11 = int(std::floor(y11 * g.cipix + g.chpix0));
      hr[a].x = std::max(std::min(std::min(h00, h01), std::min(h10, h11)), 0);
      hr[a].y = std::min(std::max(std::max(h00, h01), std::max(h10, h11)), nh - 1);
    }
    p->hrange = upload(p, hr);
    ok = ok && g.p1x && g.p1y && g.cdx && g.sdx && g.dconv && g.dz && g.iz && g.vz &&
         p->hrange;
    if (cb_fp_smem(g) > 200 * 1024 || cb_bp_smem(g) > 200 * 1024) {
      set_error("ccpi_plan_create: volume too large for the cone kernels' shared memory");
      delete p;
      return 1;
    }
    ok = ok && cb_prepare(g) == 0;
    if (ok) {
      const std::vector<int2> none(size_t(g.nx) * g.ny, make_int2(0, 0));
      int2 *band = upload(p, none);
      ok = band && cb_column_bands(g, band, 0) == 0;
      g.colband = band;
    }
    // one CTA per four rays (a warp each) for the forward projector and the
    // scatter: with 8 CTAs per SM looping over the rays, SMs sat idle at the
    // end of a launch (512^3: forward 334 -> 306 ms, scatter 629 -> 518 ms);
    // capped so that the FP64 partial sums stay few on huge ray counts
    p->fp_grid = int(std::min<i64>((i64(na) * nh + 3) / 4, i64(sm_count()) * 1024));
    p->bp_parts = g.nx * g.ny;
  }
  void *err = nullptr;
  ok = ok && cudaMalloc(&err, sizeof(int)) == cudaSuccess;
  if (err) {
    p->bufs.push_back(err);
    p->err = static_cast<int *>(err);
    cudaMemset(err, 0, sizeof(int));
  }
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
    set_error(std::string("ccpi_plan_create: device allocation or copy failed: ") +
              cudaGetErrorString(cudaGetLastError()));
    delete p;
    return 2;
  }
  *out = p;
  return 0;
}

int forward(const ccpi_plan *p, const float *vol, float *pix, int mode, const Epi &e,
            cudaStream_t st) {
  if (p->g.kind == CCPI_PARALLEL)
    return pb_forward(p->g, vol, pix, mode, e, p->fp_grid, p->err, st);
  return cb_forward(p->g, vol, pix, mode, e, p->hrange, p->fp_grid, st);
}

int backward(const ccpi_plan *p, const float *pix, float *vol, int mode, const Epi &e,
             cudaStream_t st) {
  if (p->g.kind == CCPI_PARALLEL)
    return pb_backward(p->g, pix, vol, mode, e, p->err, st);
  // the ray-driven scatter serves the plain and the norm forms (the CGLS
  // family); the SIRT / MLEM epilogues need a voxel's finished sum and stay
  // with the gather
  if (p->g.tune_scatter && (mode == EPI_STORE || mode == EPI_NORM)) {
    const int rc = cb_backward_scatter(p->g, pix, vol, e.pre, p->hrange, p->fp_grid, st);
    if (mode == EPI_NORM)
      k_sumsq_partials(vol, p->nvox, e.partials, sumsq_blocks(), st);
    return rc;
  }
  return cb_backward(p->g, pix, vol, mode, e, p->err, st);
}

int set_cone_backprojector(ccpi_plan *p, int scatter) {
  if (p->g.kind != CCPI_CONE) {
    set_error("ccpi_plan_set_cone_backprojector: not a cone-beam plan");
    return 1;
  }
  p->g.tune_scatter = scatter ? 1 : 0;
  // one FP64 partial sum per back-projector CTA (gather: one per column),
  // or per block of the sum-of-squares pass after the scatter
  p->bp_parts = scatter ? sumsq_blocks() : p->g.nx * p->g.ny;
  return 0;
}

// ------------------------------------------------------------------ solvers
namespace {

struct Work {
  float *r = nullptr, *d = nullptr, *q = nullptr, *s = nullptr, *t = nullptr, *u = nullptr;
  double *part1 = nullptr, *part2 = nullptr, *scal = nullptr, *norms = nullptr;
};

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Workspace layout per algorithm (floats V = volume, P = sinogram):
//  CGLS      r:P  d:V  q(Ad):P  s:V
//  SIRT      r:P  d(C):V  q(R):P
//  MLEM      r:P  d(N):V
//  CGLS-reg  r:P  d:V  q(Adp):P  s:V  t(Adv):V  u:V
size_t layout(const ccpi_plan *p, int alg, int niter, char *base, Work *w) {
  const size_t V = size_t(p->nvox) * 4, P = size_t(p->npix) * 4;
  size_t off = 0;
  auto take = [&](size_t bytes) -> char * {
    char *q = base ? base + off : nullptr;
    off += align_up(bytes);
    return q;
  };
  Work tmp;
  Work &W = w ? *w : tmp;
  W.r = (float *)take(P);
  W.d = (float *)take(V);
  if (alg == CCPI_CGLS || alg == CCPI_SIRT || alg >= CCPI_CGLS_TIKHONOV)
    W.q = (float *)take(P);
  if (alg == CCPI_CGLS || alg >= CCPI_CGLS_TIKHONOV)
    W.s = (float *)take(V);
  if (alg >= CCPI_CGLS_TIKHONOV) {
    W.t = (float *)take(V);
    W.u = (float *)take(V);
  }
  const int nparts = std::max(std::max(p->fp_grid, p->bp_parts), sumsq_blocks());
  W.part1 = (double *)take(sizeof(double) * nparts);
  W.part2 = (double *)take(sizeof(double) * nparts);
  W.scal = (double *)take(sizeof(double) * 8);
  W.norms = (double *)take(sizeof(double) * std::max(niter, 1));
  return off;
}

// The back projection of the CGLS residual r.  Cone beam: the residual is
// first scaled by d_conv into q (free once r is updated), the reference's
// dpixels, and the back projector reads the scaled copy.
int backward_residual(const ccpi_plan *p, const Work &W, Epi e, cudaStream_t st) {
  if (p->g.kind == CCPI_CONE && cb_bp_takes_prescaled(p->g)) {
    cb_prescale(p->g, W.r, W.q, st);
    e.pre = 1;
    return backward(p, W.q, W.s, EPI_NORM, e, st);
  }
  return backward(p, W.r, W.s, EPI_NORM, e, st);
}

// One iteration of `alg` (kernels only; capturable).
int iterate(const ccpi_plan *p, int alg, const float *sino, float *x, const Work &W,
            float lambda, cudaStream_t st) {
  const i64 V = p->nvox, P = p->npix;
  Epi e{};
  // cone SIRT / MLEM: the forward projector stores its residual scaled by
  // d_conv, which the back projector then reads as is
  const int pre = (p->g.kind == CCPI_CONE && cb_bp_takes_prescaled(p->g)) ? 1 : 0;
  int rc = 0;
  switch (alg) {
  case CCPI_CGLS:
    e.partials = W.part1;
    rc |= forward(p, W.d, W.q, EPI_NORM, e, st);
    k_cgls_scalars(S_ALPHA, W.part1, p->fp_grid, nullptr, 0, W.scal, nullptr, st);
    k_axpy_scalar(W.r, W.q, P, W.scal, 1, -1.0f, st);
    e.partials = W.part2;
    rc |= backward_residual(p, W, e, st);
    k_cgls_scalars(S_BETA, W.part2, p->bp_parts, nullptr, 0, W.scal, W.norms, st);
    k_cgls_xd(x, W.d, W.s, V, W.scal, st);
    break;
  case CCPI_SIRT:
    e.b = sino;
    e.w = W.q; // R
    e.pre = pre;
    rc |= forward(p, x, W.r, EPI_SIRT, e, st);
    e.w = W.d; // C
    e.x = x;
    rc |= backward(p, W.r, x, EPI_SIRT, e, st);
    break;
  case CCPI_MLEM:
    e.b = sino;
    e.pre = pre;
    rc |= forward(p, x, W.r, EPI_MLEM, e, st);
    e.w = W.d; // N
    e.x = x;
    rc |= backward(p, W.r, x, EPI_MLEM, e, st);
    break;
  case CCPI_CGLS_TIKHONOV:
  case CCPI_CGLS_TV:
    e.partials = W.part1;
    rc |= forward(p, W.d, W.q, EPI_NORM, e, st);
    k_reg_accumulate(alg, W.d, W.t, p->g.nx, p->g.ny, p->g.nz, lambda, W.part2,
                     sumsq_blocks(), st);
    k_cgls_scalars(S_ALPHA2, W.part1, p->fp_grid, W.part2, sumsq_blocks(), W.scal, nullptr,
                   st);
    k_axpy_scalar(W.r, W.q, P, W.scal, 1, -1.0f, st);
    k_add_scaled(W.u, x, W.d, V, W.scal, st);
    k_reg_step(alg, W.u, x, p->g.nx, p->g.ny, p->g.nz, lambda, st);
    e.partials = W.part2;
    rc |= backward_residual(p, W, e, st);
    k_cgls_scalars(S_BETA, W.part2, p->bp_parts, nullptr, 0, W.scal, W.norms, st);
    k_cgls_d(W.d, W.s, V, W.scal, st);
    break;
  default:
    return 1;
  }
  return rc;
}

// pix = A 1 and vol = A^T 1.  The parallel projectors have a form that reads
// no input (EPI_ONES); elsewhere a ones array is written into the scratch
// buffer and projected.
int forward_ones(const ccpi_plan *p, float *scratch_vol, float *pix, cudaStream_t st) {
  const Epi e{};
  if (p->g.kind == CCPI_PARALLEL) {
    const int rc = forward(p, nullptr, pix, EPI_ONES, e, st);
    if (rc != 3)
      return rc;
  }
  k_fill(scratch_vol, p->nvox, 1.0f, st);
  return forward(p, scratch_vol, pix, EPI_STORE, e, st);
}

int backward_ones(const ccpi_plan *p, float *scratch_pix, float *vol, cudaStream_t st) {
  const Epi e{};
  if (p->g.kind == CCPI_PARALLEL) {
    const int rc = backward(p, nullptr, vol, EPI_ONES, e, st);
    if (rc != 3)
      return rc;
  }
  k_fill(scratch_pix, p->npix, 1.0f, st);
  // cone: the SIRT / MLEM weights come from the deterministic gather
  // whichever back projector the iterations use, so they equal the
  // reference's bit for bit
  if (p->g.kind == CCPI_CONE)
    return cb_backward(p->g, scratch_pix, vol, EPI_STORE, e, p->err, st);
  return backward(p, scratch_pix, vol, EPI_STORE, e, st);
}

// Set-up before the first iteration (kernels only).
int prepare(const ccpi_plan *p, int alg, const float *sino, float *x, const Work &W,
            cudaStream_t st) {
  const i64 V = p->nvox, P = p->npix;
  Epi e{};
  int rc = 0;
  cudaMemsetAsync(W.scal, 0, sizeof(double) * 8, st);
  switch (alg) {
  case CCPI_CGLS:
  case CCPI_CGLS_TIKHONOV:
  case CCPI_CGLS_TV:
    // the residual starts at b even for a warm start (cgls.cpp:33-46)
    cudaMemcpyAsync(W.r, sino, size_t(P) * 4, cudaMemcpyDeviceToDevice, st);
    e.partials = W.part2;
    rc |= backward(p, W.r, W.d, EPI_NORM, e, st);
    k_cgls_scalars(S_INIT, W.part2, p->bp_parts, nullptr, 0, W.scal, nullptr, st);
    if (alg != CCPI_CGLS)
      cudaMemsetAsync(W.t, 0, size_t(V) * 4, st);
    break;
  case CCPI_SIRT:
    // R = 1 / (A 1), C = 1 / (A^T 1), non-positive -> 0 (sirt.cpp:31-48)
    rc |= forward_ones(p, W.d, W.q, st);
    k_invert_pos(W.q, P, st);
    rc |= backward_ones(p, W.r, W.d, st);
    k_invert_pos(W.d, V, st);
    break;
  case CCPI_MLEM:
    // x = 1; N = 1 / (A^T 1), zeros kept (mlem.cpp:30-41)
    k_fill(x, V, 1.0f, st);
    rc |= backward_ones(p, W.r, W.d, st);
    k_invert_nonzero(W.d, V, st);
    break;
  default:
    return 1;
  }
  return rc;
}

bool check_err(const ccpi_plan *p) {
  int h = 0;
  cudaMemcpy(&h, p->err, sizeof(int), cudaMemcpyDeviceToHost);
  if (h) {
    cudaMemset(p->err, 0, sizeof(int));
    set_error(h == 1   ? "projector: more detector columns per voxel than the back "
                         "projector stages (voxel much larger than a pixel)"
              : h == 2 ? "projector: cone back projector ray list overflow (voxel "
                         "shadow wider than 24 detector columns)"
                       : "projector: a ray's staged xy blocks or cells overflowed the "
                         "forward projector's shared-memory staging");
    return false;
  }
  return true;
}

// Capture one iteration into an executable graph.  Capture runs on a
// private stream ordered after `st` (the caller's stream may be the legacy
// default stream, which cannot be captured); the graph is launched on `st`.
bool capture_iteration(const ccpi_plan *p, int alg, const float *sino, float *x, const Work &W,
                       float lambda, cudaStream_t st, cudaGraph_t *graph, cudaGraphExec_t *exec,
                       int *rc) {
  cudaStream_t cap = nullptr;
  cudaEvent_t ev = nullptr;
  bool ok = cuda_ok(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream") &&
            cuda_ok(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "capture event");
  ok = ok && cuda_ok(cudaEventRecord(ev, st), "capture event record") &&
       cuda_ok(cudaStreamWaitEvent(cap, ev, 0), "capture stream wait");
  ok = ok && cuda_ok(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal),
                     "begin capture");
  if (ok) {
    *rc |= iterate(p, alg, sino, x, W, lambda, cap);
    ok = cuda_ok(cudaStreamEndCapture(cap, graph), "end capture");
  }
  ok = ok && cuda_ok(cudaGraphInstantiate(exec, *graph, 0), "graph instantiate");
  if (ev)
    cudaEventDestroy(ev);
  if (cap)
    cudaStreamDestroy(cap);
  return ok;
}

} // namespace

size_t solve_workspace_bytes(const ccpi_plan *p, int alg, int niter) {
  return layout(p, alg, niter, nullptr, nullptr);
}

// ---- sessions: one prepared solver whose iteration is a captured graph
struct Session {
  const ccpi_plan *plan = nullptr;
  int alg = 0;
  const float *sino = nullptr;
  float *x = nullptr;
  float lambda = 0.0f;
  int flags = 0;
  int max_iter = 0, done = 0;
  cudaStream_t st = nullptr;
  void *ws = nullptr;
  Work W;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~Session() {
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
    if (ws)
      cudaFree(ws);
  }
};

void *session_create(const ccpi_plan *p, int alg, const float *sino, float *x, double lambda,
                     int max_iter, int flags, cudaStream_t st, int *rc) {
  *rc = 0;
  if (alg < CCPI_CGLS || alg > CCPI_CGLS_TV || max_iter < 0) {
    set_error("ccpi_session_create: unknown algorithm or negative iteration budget");
    *rc = 1;
    return nullptr;
  }
  Session *S = new Session();
  S->plan = p;
  S->alg = alg;
  S->sino = sino;
  S->x = x;
  S->lambda = float(lambda);
  S->flags = flags;
  S->max_iter = max_iter;
  S->st = st;
  const size_t need = layout(p, alg, max_iter, nullptr, nullptr);
  if (!cuda_ok(cudaMalloc(&S->ws, need), "ccpi_session_create: workspace")) {
    delete S;
    *rc = 2;
    return nullptr;
  }
  layout(p, alg, max_iter, static_cast<char *>(S->ws), &S->W);
  *rc = prepare(p, alg, sino, x, S->W, st);
  if (*rc == 0 && !(flags & CCPI_SOLVE_PLAIN)) {
    if (!capture_iteration(p, alg, sino, x, S->W, S->lambda, st, &S->graph, &S->exec, rc))
      *rc |= 4;
  }
  if (*rc) {
    delete S;
    return nullptr;
  }
  return S;
}

int session_run(void *h, int n) {
  Session *S = static_cast<Session *>(h);
  if (n < 0 || S->done + n > S->max_iter) {
    set_error("ccpi_session_run: iteration budget of the session exceeded");
    return 1;
  }
  int rc = 0;
  for (int it = 0; it < n && rc == 0; it++) {
    if (S->flags & CCPI_SOLVE_PLAIN) {
      double scal[8];
      rc |= iterate(S->plan, S->alg, S->sino, S->x, S->W, S->lambda, S->st);
      cudaMemcpyAsync(scal, S->W.scal, sizeof(scal), cudaMemcpyDeviceToHost, S->st);
      cudaStreamSynchronize(S->st);
    } else if (!cuda_ok(cudaGraphLaunch(S->exec, S->st), "ccpi_session_run: graph launch")) {
      rc = 4;
    }
  }
  S->done += n;
  return rc;
}

int session_finish(void *h, double *h_norms) {
  Session *S = static_cast<Session *>(h);
  k_clamp0(S->x, S->plan->nvox, S->st);
  if (!cuda_ok(cudaStreamSynchronize(S->st), "ccpi_session_finish: execution"))
    return 8;
  if (!check_err(S->plan))
    return 16;
  if (h_norms && S->done > 0 && (S->alg == CCPI_CGLS || S->alg >= CCPI_CGLS_TIKHONOV))
    cudaMemcpy(h_norms, S->W.norms, sizeof(double) * S->done, cudaMemcpyDeviceToHost);
  return 0;
}

void session_destroy(void *h) { delete static_cast<Session *>(h); }

// ---- z-sharded CGLS family: one slab of a parallel-beam volume per rank
//
// A parallel-beam volume cut along z into slabs (rows map to their own
// slices, so each rank projects its slab alone; the reference's MPI split,
// voxels.cpp:27-45) needs, per CGLS iteration, the two step-scalar sums over
// all ranks and, for TV, the z planes next to each cut.  The iteration of
// iterate() is split at those points into stages; between stages the caller
// all-reduces one double (sum) and, for TV, swaps edge planes into the
// neighbours' halo buffers.  With one rank and no halos the stages give the
// unsharded solve bit for bit.
struct Shard {
  const ccpi_plan *plan = nullptr;
  int alg = 0;
  const float *sino = nullptr;
  float *x = nullptr;
  float lambda = 0.0f;
  int max_iter = 0, done = 0;
  int next = SHARD_SETUP; // the stage the protocol expects next
  cudaStream_t st = nullptr;
  void *ws = nullptr;
  Work W;
  double *sum = nullptr;              // caller-owned, 1 double
  float *edge_lo = nullptr, *edge_hi = nullptr;   // caller-owned, nx * ny each
  const float *halo_lo = nullptr, *halo_hi = nullptr; // caller-owned or NULL
  ~Shard() {
    if (ws)
      cudaFree(ws);
  }
};

void *shard_create(const ccpi_plan *p, int alg, const float *sino, float *x, double lambda,
                   int max_iter, double *sum, float *edges, const float *halo_lo,
                   const float *halo_hi, cudaStream_t st, int *rc) {
  *rc = 0;
  if (alg != CCPI_CGLS && alg != CCPI_CGLS_TIKHONOV && alg != CCPI_CGLS_TV) {
    set_error("ccpi_shard_create: sharded solves are the CGLS family (SIRT and MLEM need no "
              "exchange: solve each slab alone)");
    *rc = 1;
    return nullptr;
  }
  if (p->g.kind != CCPI_PARALLEL || max_iter < 0 || !sum || !edges) {
    set_error("ccpi_shard_create: needs a parallel-beam plan, an iteration budget, a sum and "
              "an edge buffer");
    *rc = 1;
    return nullptr;
  }
  Shard *S = new Shard();
  S->plan = p;
  S->alg = alg;
  S->sino = sino;
  S->x = x;
  S->lambda = float(lambda);
  S->max_iter = max_iter;
  S->st = st;
  S->sum = sum;
  const i64 nxy = i64(p->g.nx) * p->g.ny;
  S->edge_lo = edges;
  S->edge_hi = edges + nxy;
  S->halo_lo = halo_lo;
  S->halo_hi = halo_hi;
  const size_t need = layout(p, alg, max_iter, nullptr, nullptr);
  if (!cuda_ok(cudaMalloc(&S->ws, need), "ccpi_shard_create: workspace")) {
    delete S;
    *rc = 2;
    return nullptr;
  }
  layout(p, alg, max_iter, static_cast<char *>(S->ws), &S->W);
  return S;
}

int shard_stage(void *h, int stage) {
  Shard *S = static_cast<Shard *>(h);
  if (stage != S->next) {
    set_error("ccpi_shard_stage: stage " + std::to_string(stage) + " out of order (expected " +
              std::to_string(S->next) + ")");
    return 1;
  }
  if (stage == SHARD_FORWARD && S->done >= S->max_iter) {
    set_error("ccpi_shard_stage: iteration budget of the shard exceeded");
    return 1;
  }
  const ccpi_plan *p = S->plan;
  const Work &W = S->W;
  const cudaStream_t st = S->st;
  const i64 V = p->nvox, P = p->npix;
  const int nx = p->g.nx, ny = p->g.ny, nz = p->g.nz, nb = sumsq_blocks();
  const bool reg = S->alg != CCPI_CGLS;
  Epi e{};
  int rc = 0;
  switch (stage) {
  case SHARD_SETUP:
    // the residual starts at b (cgls.cpp:33-46); d = A^T r
    cudaMemsetAsync(W.scal, 0, sizeof(double) * 8, st);
    cudaMemcpyAsync(W.r, S->sino, size_t(P) * 4, cudaMemcpyDeviceToDevice, st);
    e.partials = W.part2;
    rc |= backward(p, W.r, W.d, EPI_NORM, e, st);
    k_shard_scalars(SH_LOCAL, W.part2, p->bp_parts, nullptr, 0, S->sum, W.scal, nullptr, st);
    if (reg)
      cudaMemsetAsync(W.t, 0, size_t(V) * 4, st);
    k_pack_edges(W.d, nx, ny, nz, S->edge_lo, S->edge_hi, st);
    S->next = SHARD_FORWARD;
    break;
  case SHARD_FORWARD:
    if (S->done == 0)
      k_shard_scalars(SH_INIT, nullptr, 0, nullptr, 0, S->sum, W.scal, nullptr, st);
    e.partials = W.part1;
    rc |= forward(p, W.d, W.q, EPI_NORM, e, st);
    if (reg)
      k_reg_accumulate(S->alg, W.d, W.t, nx, ny, nz, S->lambda, W.part2, nb, st, S->halo_lo,
                       S->halo_hi);
    k_shard_scalars(SH_LOCAL, W.part1, p->fp_grid, reg ? W.part2 : nullptr, nb, S->sum, W.scal,
                    nullptr, st);
    S->next = SHARD_UPDATE;
    break;
  case SHARD_UPDATE:
    k_shard_scalars(SH_ALPHA, nullptr, 0, nullptr, 0, S->sum, W.scal, nullptr, st);
    k_axpy_scalar(W.r, W.q, P, W.scal, 1, -1.0f, st);
    if (reg) {
      k_add_scaled(W.u, S->x, W.d, V, W.scal, st);
      k_pack_edges(W.u, nx, ny, nz, S->edge_lo, S->edge_hi, st);
    }
    S->next = SHARD_BACKWARD;
    break;
  case SHARD_BACKWARD:
    if (reg)
      k_reg_step(S->alg, W.u, S->x, nx, ny, nz, S->lambda, st, S->halo_lo, S->halo_hi);
    e.partials = W.part2;
    rc |= backward(p, W.r, W.s, EPI_NORM, e, st);
    k_shard_scalars(SH_LOCAL, W.part2, p->bp_parts, nullptr, 0, S->sum, W.scal, nullptr, st);
    S->next = SHARD_NEXT;
    break;
  case SHARD_NEXT:
    k_shard_scalars(SH_BETA, nullptr, 0, nullptr, 0, S->sum, W.scal, W.norms, st);
    if (reg) {
      k_cgls_d(W.d, W.s, V, W.scal, st);
      k_pack_edges(W.d, nx, ny, nz, S->edge_lo, S->edge_hi, st);
    } else {
      k_cgls_xd(S->x, W.d, W.s, V, W.scal, st);
    }
    S->done++;
    S->next = SHARD_FORWARD;
    break;
  default:
    set_error("ccpi_shard_stage: unknown stage");
    return 1;
  }
  if (!cuda_ok(cudaGetLastError(), "ccpi_shard_stage: launch"))
    rc |= 4;
  return rc;
}

int shard_finish(void *h, double *h_norms) {
  Shard *S = static_cast<Shard *>(h);
  if (S->next != SHARD_FORWARD) {
    set_error("ccpi_shard_finish: the last iteration is incomplete (finish after "
              "CCPI_SHARD_NEXT or CCPI_SHARD_SETUP)");
    return 1;
  }
  k_clamp0(S->x, S->plan->nvox, S->st);
  if (!cuda_ok(cudaStreamSynchronize(S->st), "ccpi_shard_finish: execution"))
    return 8;
  if (!check_err(S->plan))
    return 16;
  if (h_norms && S->done > 0)
    cudaMemcpy(h_norms, S->W.norms, sizeof(double) * S->done, cudaMemcpyDeviceToHost);
  return 0;
}

void shard_destroy(void *h) { delete static_cast<Shard *>(h); }

int solve(const ccpi_plan *p, int alg, const float *sino, float *x, int niter, double lambda,
          double *h_norms, int flags, void *ws, size_t ws_bytes, cudaStream_t st) {
  if (alg < CCPI_CGLS || alg > CCPI_CGLS_TV) {
    set_error("ccpi_solve: unknown algorithm");
    return 1;
  }
  if (niter < 0) {
    set_error("ccpi_solve: negative iteration count");
    return 1;
  }
  const size_t need = layout(p, alg, niter, nullptr, nullptr);
  void *owned = nullptr;
  if (!ws) {
    if (!cuda_ok(cudaMalloc(&owned, need), "ccpi_solve: workspace allocation"))
      return 2;
    ws = owned;
  } else if (ws_bytes < need) {
    set_error("ccpi_solve: workspace too small");
    return 1;
  }
  Work W;
  layout(p, alg, niter, static_cast<char *>(ws), &W);
  int rc = prepare(p, alg, sino, x, W, st);
  const float lam = float(lambda);
  if (flags & CCPI_SOLVE_PLAIN) {
    double scal[8];
    for (int it = 0; it < niter && rc == 0; it++) {
      rc |= iterate(p, alg, sino, x, W, lam, st);
      cudaMemcpyAsync(scal, W.scal, sizeof(scal), cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
    }
  } else if (niter > 0 && rc == 0) {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ok = capture_iteration(p, alg, sino, x, W, lam, st, &graph, &exec, &rc);
    for (int it = 0; ok && it < niter; it++)
      ok = cuda_ok(cudaGraphLaunch(exec, st), "ccpi_solve: graph launch");
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
    if (!ok)
      rc |= 4;
  }
  // every reconstruction is clamped at zero (voxels.cpp:187, :272, :352)
  k_clamp0(x, p->nvox, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "ccpi_solve: execution"))
    rc |= 8;
  if (rc == 0 && !check_err(p))
    rc = 16;
  if (rc == 0 && h_norms && niter > 0 && (alg == CCPI_CGLS || alg >= CCPI_CGLS_TIKHONOV))
    cudaMemcpy(h_norms, W.norms, sizeof(double) * niter, cudaMemcpyDeviceToHost);
  if (owned)
    cudaFree(owned);
  if (rc && g_last_error.empty())
    set_error("ccpi_solve: kernel launch failed");
  return rc;
}

int solve_batched(int n, const ccpi_plan *const *plans, int alg, const float *const *sino,
                  float *const *x, int niter, const double *lambda, cudaStream_t st) {
  if (n <= 0)
    return 0;
  std::vector<void *> ws(n, nullptr);
  std::vector<Work> W(n);
  int rc = 0;
  for (int i = 0; i < n && rc == 0; i++) {
    const size_t need = layout(plans[i], alg, niter, nullptr, nullptr);
    if (!cuda_ok(cudaMalloc(&ws[i], need), "ccpi_solve_batched: workspace"))
      rc = 2;
    else
      layout(plans[i], alg, niter, static_cast<char *>(ws[i]), &W[i]);
  }
  // branches: problem i runs on stream i % kStreams inside the graph
  const int kStreams = std::min(n, 16);
  std::vector<cudaStream_t> br(kStreams, nullptr);
  std::vector<cudaEvent_t> ev(kStreams + 1, nullptr);
  for (int k = 0; k < kStreams && rc == 0; k++)
    if (cudaStreamCreateWithFlags(&br[k], cudaStreamNonBlocking) != cudaSuccess)
      rc = 2;
  for (int k = 0; k <= kStreams && rc == 0; k++)
    if (cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming) != cudaSuccess)
      rc = 2;
  auto fork_join = [&](cudaStream_t root, auto &&body) {
    cudaEventRecord(ev[kStreams], root);
    for (int k = 0; k < kStreams; k++)
      cudaStreamWaitEvent(br[k], ev[kStreams], 0);
    for (int i = 0; i < n; i++)
      rc |= body(i, br[i % kStreams]);
    for (int k = 0; k < kStreams; k++) {
      cudaEventRecord(ev[k], br[k]);
      cudaStreamWaitEvent(root, ev[k], 0);
    }
  };
  cudaStream_t root = nullptr;
  if (rc == 0 && !cuda_ok(cudaStreamCreateWithFlags(&root, cudaStreamNonBlocking),
                          "ccpi_solve_batched: capture stream"))
    rc = 2;
  if (rc == 0) {
    fork_join(st, [&](int i, cudaStream_t s) { return prepare(plans[i], alg, sino[i], x[i], W[i], s); });
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    // capture on a private stream ordered after st (st may be the legacy
    // default stream, which cannot be captured)
    cudaEventRecord(ev[kStreams], st);
    cudaStreamWaitEvent(root, ev[kStreams], 0);
    bool ok = cuda_ok(cudaStreamBeginCapture(root, cudaStreamCaptureModeThreadLocal),
                      "ccpi_solve_batched: begin capture");
    if (ok) {
      fork_join(root, [&](int i, cudaStream_t s) {
        return iterate(plans[i], alg, sino[i], x[i], W[i], float(lambda ? lambda[i] : 0.0), s);
      });
      ok = cuda_ok(cudaStreamEndCapture(root, &graph), "ccpi_solve_batched: end capture");
    }
    ok = ok && cuda_ok(cudaGraphInstantiate(&exec, graph, 0), "ccpi_solve_batched: instantiate");
    for (int it = 0; ok && it < niter; it++)
      ok = cuda_ok(cudaGraphLaunch(exec, st), "ccpi_solve_batched: graph launch");
    if (exec)
      cudaGraphExecDestroy(exec);
    if (graph)
      cudaGraphDestroy(graph);
    if (!ok)
      rc |= 4;
    for (int i = 0; i < n; i++)
      k_clamp0(x[i], plans[i]->nvox, st);
    if (!cuda_ok(cudaStreamSynchronize(st), "ccpi_solve_batched: execution"))
      rc |= 8;
    for (int i = 0; i < n && rc == 0; i++)
      if (!check_err(plans[i]))
        rc = 16;
  }
  for (auto s : br)
    if (s)
      cudaStreamDestroy(s);
  if (root)
    cudaStreamDestroy(root);
  for (auto e : ev)
    if (e)
      cudaEventDestroy(e);
  for (auto w : ws)
    if (w)
      cudaFree(w);
  return rc;
}

// Time the launch-shape candidates of this plan's projectors on scratch data
// and keep the fastest (CUDA events on st; a warm-up launch, then the mean of
// two).  Every candidate forms each ray's and each voxel's sum in the same
// order, so projections do not depend on the choice; only the number of
// per-CTA partial sums of squares (and so the FP64 summation order of the
// CGLS step scalars) follows the forward projector's grid.
int plan_autotune(ccpi_plan *p, cudaStream_t st, int *chosen) {
  float *vol = nullptr, *pix = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  if (!cuda_ok(cudaMalloc(&vol, size_t(p->nvox) * 4), "autotune: volume") ||
      !cuda_ok(cudaMalloc(&pix, size_t(p->npix) * 4), "autotune: sinogram") ||
      !cuda_ok(cudaEventCreate(&e0), "autotune: event") ||
      !cuda_ok(cudaEventCreate(&e1), "autotune: event"))
    rc = 2;
  if (rc == 0) {
    k_fill(vol, p->nvox, 1.0f, st);
    k_fill(pix, p->npix, 1.0f, st);
  }
  auto timed = [&](auto &&launch) -> float {
    launch();
    cudaEventRecord(e0, st);
    launch();
    launch();
    cudaEventRecord(e1, st);
    float ms = 0.0f;
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return 1e30f;
    return ms / 2.0f;
  };
  const Epi none{};
  int best_fp = 0, best_bp = 0;
  if (rc == 0 && p->g.kind == CCPI_PARALLEL) {
    float t_best = 1e30f;
    const int defgrid = p->fp_grid;
    for (int per_sm : {3, 4, 5}) {
      // defgrid is min(work tiles, 5 CTAs per SM)
      const int gcand = std::max(1, std::min(defgrid, 148 * per_sm));
      p->fp_grid = gcand;
      const float t = timed([&] { pb_forward(p->g, vol, pix, EPI_STORE, none, p->fp_grid, p->err, st); });
      if (t < t_best) {
        t_best = t;
        best_fp = gcand;
      }
    }
    p->fp_grid = best_fp;
    t_best = 1e30f;
    for (int vw : {16, 8, 4}) {
      if (p->g.map_type != 1 || p->g.nv != p->g.nz || p->g.nz % vw != 0)
        continue;
      p->g.tune_vw = vw;
      const float t = timed([&] { pb_backward(p->g, pix, vol, EPI_STORE, none, p->err, st); });
      if (t < t_best) {
        t_best = t;
        best_bp = vw;
      }
    }
    p->g.tune_vw = best_bp;
    p->bp_parts = pb_bp_tiles(p->g);
  } else if (rc == 0) {
    float t_best = 1e30f;
    for (int rpl : {4, 8, 12}) {
      p->g.tune_rpl = rpl;
      const float t = timed([&] {
        cb_forward(p->g, vol, pix, EPI_STORE, none, p->hrange, p->fp_grid, st);
      });
      if (t < t_best) {
        t_best = t;
        best_fp = rpl;
      }
    }
    p->g.tune_rpl = best_fp;
    // back projector: the deterministic voxel gather or the ray-driven
    // scatter, whichever is faster on this geometry, each timed in the
    // form the CGLS iterations run (on a sinogram pre-scaled by d_conv
    // where the gather takes one; the scratch values do not matter)
    Epi pre{};
    pre.pre = cb_bp_takes_prescaled(p->g) ? 1 : 0;
    const float t_gather = timed([&] {
      cb_backward(p->g, pix, vol, EPI_STORE, pre, p->err, st);
    });
    const float t_scatter = timed([&] {
      cb_backward_scatter(p->g, pix, vol, pre.pre, p->hrange, p->fp_grid, st);
    });
    set_cone_backprojector(p, t_scatter < t_gather ? 1 : 0);
    best_bp = p->g.tune_scatter;
  }
  if (rc == 0 && !cuda_ok(cudaStreamSynchronize(st), "autotune"))
    rc = 2;
  if (rc == 0 && !check_err(p))
    rc = 16;
  if (chosen) {
    chosen[0] = p->g.kind == CCPI_PARALLEL ? p->fp_grid : p->g.tune_rpl;
    chosen[1] = p->g.kind == CCPI_PARALLEL ? p->g.tune_vw : p->g.tune_scatter;
  }
  if (e0)
    cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
  cudaFree(vol);
  cudaFree(pix);
  return rc;
}

} // namespace ccpi
