// CPU restatement of CCPi-Reconstruction's iterative hot path: the parallel-
// and cone-beam Siddon projectors of Core/src/p2D.cpp and Core/src/c2D.cpp,
// the CGLS / SIRT / MLEM / CGLS-Tikhonov / CGLS-TV solvers of
// Core/src/Algorithms/*.cpp with the vector kernels of Core/src/blas.hpp,
// and the regularisers of Core/src/tikhonov.cpp and Core/src/total_v.cpp.
//
// TEST INFRASTRUCTURE ONLY (the oracle).  Only tests/, the smoke check and
// bench.py's CPU-baseline leg call it; no product code links it.
//
// It is written from the reference's algorithm, not copied: one walk routine
// per geometry handles the four direction octants with step signs, and the
// routines are templated on the arithmetic type.  The float instantiation
// keeps the reference's types (double geometry, float "recon_type"
// intermediates, float data) and its operation order and evaluation rules
// (exact-equality entry faces, FLT_EPSILON tie tolerance, int() truncation
// vs floor), so it reproduces the reference bit for bit; the double
// instantiation is the FP64 oracle.  Compiled with -ffp-contract=off so no
// multiply-add is fused (the reference's x86-64 build has no FMA).
//
// Where the reference reads outside an array (noted per routine) this
// restatement skips the access; those paths only occur in geometries the
// reference itself cannot handle (rays missing the volume vertically at
// entry, detector rows outside the volume in pb_forward_project).
#include "restate.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

typedef long long i64;
const float kEps = FLT_EPSILON; // p2D.cpp:20, c2D.cpp:15

// T = data type, R = the reference's recon_type (float) or double.
template <class T> struct types {
  typedef T R;
};

inline i64 vox_index(int x, int y, int ny, int nz) {
  return (i64(x) * ny + y) * nz;
}

// ------------------------------------------------------------ parallel beam

// p2D.cpp:22-61: detector row -> voxel slice, and the special cases
// 1 (one row per slice), 2 and 4 (rows per slice) the loops exploit.
void gen_mapping(const rs_geometry *g, std::vector<int> &map, int &type) {
  map.assign(g->nv, 0);
  for (int v = 0; v < g->nv; v++)
    map[v] = int(std::floor((g->v_pixels[v] - g->origin[2]) / g->size[2]));
  type = 0;
  for (int per : {1, 2, 4}) {
    bool ok = true;
    for (int v = 0; v < g->nv && ok; v++)
      ok = map[v] == v / per;
    if (ok) {
      type = per;
      return;
    }
  }
}

// Accumulate sum_m len[m] * column_m(z) into one detector column
// (p2D.cpp:63-213, scalar paths; the GCC build uses these).
template <class T, class R>
void pb_add_columns(T *pix, const T *vol, const std::vector<i64> &cells,
                    const std::vector<R> &len, int nv, int nz,
                    const std::vector<int> &map, int map_type) {
  for (size_t m = 0; m < cells.size(); m++) {
    const T *col = vol + cells[m];
    const T w = T(len[m]);
    switch (map_type) {
    case 1:
      for (int v = 0; v < nv; v++)
        pix[v] += col[v] * w;
      break;
    case 2:
    case 4:
      // the reference runs z over all nz slices; rows past nv do not exist
      for (int z = 0, v = 0; z < nz; z++)
        for (int r = 0; r < map_type; r++, v++)
          if (v < nv)
            pix[v] += col[z] * w;
      break;
    default:
      // the reference reads col[map[v]] without a range check
      for (int v = 0; v < nv; v++)
        if (map[v] >= 0 && map[v] < nz)
          pix[v] += col[map[v]] * w;
      break;
    }
  }
}

// One ray through one 32x32 xy block (p2D.cpp:215-466).  The ray is
// p2 + alpha (c, s), alpha in [-d_conv, 0]; lengths are alpha differences.
// Appends visited columns (volume offsets) and chord lengths.
template <class R>
void pb_block_walk(double p2x, double p2y, double bx, double by, double dx,
                   double dy, int nxb, int nyb, int bx0, int by0, int ny,
                   int nz, R d_conv, double c, double s,
                   std::vector<i64> &cells, std::vector<R> &len) {
  cells.clear();
  len.clear();
  if (std::abs(c) < kEps) {
    if (std::abs(s) < kEps)
      return;
    // parallel to y: one column of cells, walked in the ray direction
    int i = int(std::floor((p2x - bx) / dx));
    if (i < 0 || i >= nxb)
      return;
    for (int t = 0; t < nyb; t++) {
      int j = s < 0.0 ? nyb - 1 - t : t;
      cells.push_back(vox_index(bx0 + i, by0 + j, ny, nz));
      len.push_back(R(dy));
    }
    return;
  }
  if (std::abs(s) < kEps) {
    int j = int(std::floor((p2y - by) / dy));
    if (j < 0 || j >= nyb)
      return;
    for (int t = 0; t < nxb; t++) {
      int i = c < 0.0 ? nxb - 1 - t : t;
      cells.push_back(vox_index(bx0 + i, by0 + j, ny, nz));
      len.push_back(R(dx));
    }
    return;
  }
  const double x0 = bx, y0 = by;
  const double xn = bx + double(nxb) * dx, yn = by + double(nyb) * dy;
  const double inv_c = 1.0 / c, inv_s = 1.0 / s;
  const double ax0 = (x0 - p2x) * inv_c, ay0 = (y0 - p2y) * inv_s;
  const double axn = (xn - p2x) * inv_c, ayn = (yn - p2y) * inv_s;
  const double amin = std::max(std::max(std::min(ax0, axn), std::min(ay0, ayn)),
                               double(-d_conv));
  const double amax =
      std::min(std::min(std::max(ax0, axn), std::max(ay0, ayn)), 0.0);
  if (!(amin < amax - kEps))
    return;
  const int sx = c > 0.0 ? 1 : -1, sy = s > 0.0 ? 1 : -1;
  auto alpha_x = [&](int i) { return (bx + double(i) * dx - p2x) * inv_c; };
  auto alpha_y = [&](int j) { return (by + double(j) * dy - p2y) * inv_s; };
  auto cell_x = [&]() { return int(std::floor((p2x + amin * c - bx) / dx)); };
  auto cell_y = [&]() { return int(std::floor((p2y + amin * s - by) / dy)); };
  // entry cell: the face tested first differs per octant in the reference
  int x = 0, y = 0;
  if (sx > 0 && sy > 0) {
    if (amin == ax0) {
      x = 0;
      y = cell_y();
    } else if (amin == ay0) {
      x = cell_x();
      y = 0;
    }
  } else if (sx > 0) {
    if (amin == ayn) {
      x = cell_x();
      y = nyb - 1;
    } else if (amin == ax0) {
      x = 0;
      y = cell_y();
    }
  } else if (sy > 0) {
    if (amin == axn) {
      x = nxb - 1;
      y = cell_y();
    } else if (amin == ay0) {
      x = cell_x();
      y = 0;
    }
  } else {
    if (amin == axn) {
      x = nxb - 1;
      y = (amin == ayn) ? nyb - 1 : cell_y();
    } else if (amin == ayn) {
      x = cell_x();
      y = nyb - 1;
    }
  }
  double ap = amin;
  // the reference's loop only tests the bound in the direction of travel
  while ((sx > 0 ? x < nxb : x >= 0) && (sy > 0 ? y < nyb : y >= 0)) {
    const double nx_a = alpha_x(sx > 0 ? x + 1 : x);
    const double ny_a = alpha_y(sy > 0 ? y + 1 : y);
    const int gx = bx0 + x, gy = by0 + y;
    cells.push_back(vox_index(gx, gy, ny, nz));
    if (nx_a < ny_a - kEps) {
      len.push_back(R(nx_a - ap));
      ap = nx_a;
      x += sx;
    } else if (ny_a < nx_a - kEps) {
      len.push_back(R(ny_a - ap));
      ap = ny_a;
      y += sy;
    } else {
      const double mx = std::max(nx_a, ny_a);
      len.push_back(R(mx - ap));
      ap = mx;
      x += sx;
      y += sy;
    }
  }
}

struct pb_hrange {
  int hmin, hmax;
};

// Detector columns that can see the xy box [vx,wx) x [vy,wy) at angle
// (c, s) (p2D.cpp:527-595; the same rule is used per voxel column by the
// back projector, p2D.cpp:808-915).
pb_hrange pb_block_hrange(double vx, double wx, double vy, double wy, double c,
                          double s, double ihp, double hp0, double h0,
                          int nh) {
  int hmin = 0, hmax = nh - 1;
  if (std::abs(c) < kEps) {
    if (s < 0.0) {
      hmin = int(std::floor(vx * ihp - hp0));
      hmax = int(std::floor((wx - kEps) * ihp - hp0));
    } else {
      hmin = int(std::ceil((-wx + kEps) * ihp - hp0));
      hmax = int(std::ceil((-vx) * ihp - hp0));
    }
    hmin = std::max(hmin, 0);
    hmax = std::min(hmax, nh - 1);
  } else if (std::abs(s) < kEps) {
    if (c < 0.0) {
      hmin = int(std::ceil((-wy + kEps) * ihp - hp0));
      hmax = int(std::ceil((-vy) * ihp - hp0));
    } else {
      hmin = int(std::floor(vy * ihp - hp0));
      hmax = int(std::floor((wy - kEps) * ihp - hp0));
    }
    hmin = std::max(hmin, 0);
    hmax = std::min(hmax, nh - 1);
  } else {
    double ymin, ymax;
    if (c > 0.0) {
      if (s > 0.0) {
        ymin = vy * c - wx * s;
        ymax = wy * c - vx * s;
      } else {
        ymin = vy * c - vx * s;
        ymax = wy * c - wx * s;
      }
    } else {
      if (s > 0.0) {
        ymin = wy * c - wx * s;
        ymax = vy * c - vx * s;
      } else {
        ymin = wy * c - vx * s;
        ymax = vy * c - wx * s;
      }
    }
    hmin = (ymin < h0) ? 0 : int(std::floor(ymin * ihp - hp0));
    hmax = std::min(int(std::floor(ymax * ihp - hp0)), nh - 1);
  }
  return {hmin, hmax};
}

// parallel_beam::f2D (p2D.cpp:468-611).
template <class T> void pb_forward(const rs_geometry *g, const T *vol, T *pix) {
  typedef typename types<T>::R R;
  const int nx = g->nx, ny = g->ny, nz = g->nz, nh = g->nh, nv = g->nv;
  const double det_x =
      2.0 * std::max(std::abs(g->origin[0]),
                     std::max(std::abs(g->origin[1]), std::abs(g->origin[2])));
  const R d_conv = R(3.0 * det_x);
  std::vector<int> map;
  int map_type = 0;
  gen_mapping(g, map, map_type);
  const double *hp = g->h_pixels;
  const double ihp = 1.0 / (hp[1] - hp[0]);
  const double hp0 = hp[0] / (hp[1] - hp[0]);
  const int B = 32;
#pragma omp parallel for schedule(dynamic)
  for (int a = 0; a < g->na; a++) {
    std::vector<i64> cells;
    std::vector<R> len;
    const double c = std::cos(g->angles[a]), s = std::sin(g->angles[a]);
    for (int bx0 = 0; bx0 < nx; bx0 += B) {
      const int nxb = std::min(B, nx - bx0);
      const double vx = g->origin[0] + double(bx0) * g->size[0];
      const double wx = g->origin[0] + double(bx0 + nxb) * g->size[0];
      for (int by0 = 0; by0 < ny; by0 += B) {
        const int nyb = std::min(B, ny - by0);
        const double vy = g->origin[1] + double(by0) * g->size[1];
        const double wy = g->origin[1] + double(by0 + nyb) * g->size[1];
        pb_hrange r = pb_block_hrange(vx, wx, vy, wy, c, s, ihp, hp0, hp[0], nh);
        for (int h = r.hmin; h <= r.hmax; h++) {
          const double p2x = c * det_x - s * hp[h];
          const double p2y = s * det_x + c * hp[h];
          pb_block_walk<R>(p2x, p2y, vx, vy, g->size[0], g->size[1], nxb, nyb,
                           bx0, by0, ny, nz, d_conv, c, s, cells, len);
          // entry rounding can put the first cell one step outside the
          // block; the reference then reads a neighbour (or outside the
          // volume): only in-volume cells are kept here.
          for (size_t m = 0; m < cells.size(); m++)
            if (cells[m] < 0 || cells[m] >= i64(nx) * ny * nz)
              len[m] = R(0), cells[m] = 0;
          pb_add_columns<T, R>(pix + (i64(a) * nh + h) * nv, vol, cells, len,
                               nv, nz, map, map_type);
        }
      }
    }
  }
}

// parallel_beam::b2D (p2D.cpp:950-1087) with bproject_ah (:775-948) and
// calc_ah_z (:613-773): a voxel-column gather of trapezoid chord weights.
template <class T> void pb_backward(const rs_geometry *g, const T *pix, T *vol) {
  typedef typename types<T>::R R;
  const int nx = g->nx, ny = g->ny, nz = g->nz, nh = g->nh, nv = g->nv,
            na = g->na;
  std::vector<double> ca(na), sa(na), yoff(na), ioff(na), length(na);
  const double o0 = g->origin[0], o1 = g->origin[1];
  const double d0 = g->size[0], d1 = g->size[1];
  for (int a = 0; a < na; a++) {
    const double c = std::cos(g->angles[a]), s = std::sin(g->angles[a]);
    ca[a] = c;
    sa[a] = s;
    // footprint corners of the (0,0) voxel (p2D.cpp:999-1049)
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
    length[a] = (std::abs(c) > std::abs(s)) ? d0 / std::abs(c) : d1 / std::abs(s);
  }
  std::vector<int> map;
  int map_type = 0;
  gen_mapping(g, map, map_type);
  const double *hp = g->h_pixels;
  const double ihp = 1.0 / (hp[1] - hp[0]);
  const double hp0 = hp[0] / (hp[1] - hp[0]);
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nx; i++) {
    std::vector<i64> rows;
    std::vector<R> w;
    const double x0 = o0 + double(i) * d0, xn = o0 + double(i + 1) * d0;
    for (int j = 0; j < ny; j++) {
      const double y0 = o1 + double(j) * d1, yn = o1 + double(j + 1) * d1;
      rows.clear();
      w.clear();
      for (int a = 0; a < na; a++) {
        const double c = ca[a], s = sa[a];
        const i64 abase = i64(a) * nh;
        if (std::abs(c) < kEps || std::abs(s) < kEps) {
          pb_hrange r = pb_block_hrange(x0, xn, y0, yn, c, s, ihp, hp0, hp[0], nh);
          const bool par_y = std::abs(c) < kEps;
          const double lo = par_y ? x0 : y0, hi = par_y ? xn : yn;
          // sign of the detector axis along the box axis for this direction
          const bool neg = par_y ? !(s < 0.0) : (c < 0.0);
          const R wt = R(par_y ? g->size[1] : g->size[0]);
          for (int h = r.hmin; h <= r.hmax; h++) {
            const double u = neg ? -hp[h] : hp[h];
            if (u >= lo && u < hi) {
              rows.push_back((abase + h) * nv);
              w.push_back(wt);
            }
          }
          continue;
        }
        double ymin, ymax;
        if (c > 0.0) {
          if (s > 0.0) {
            ymin = y0 * c - xn * s;
            ymax = yn * c - x0 * s;
          } else {
            ymin = y0 * c - x0 * s;
            ymax = yn * c - xn * s;
          }
        } else {
          if (s > 0.0) {
            ymin = yn * c - xn * s;
            ymax = y0 * c - x0 * s;
          } else {
            ymin = yn * c - x0 * s;
            ymax = y0 * c - xn * s;
          }
        }
        const int hmin = (ymin < hp[0]) ? 0 : int(std::floor(ymin * ihp - hp0));
        const int hmax = std::min(int(std::floor(ymax * ihp - hp0)), nh - 1);
        const double ybot = ymin + yoff[a], ytop = ymax - yoff[a];
        const double l = length[a];
        for (int h = hmin; h <= hmax; h++) {
          if (h < 0)
            continue; // the reference would read h_pixels[-1]
          const double hv = hp[h];
          if (!(hv > ymin + kEps))
            continue;
          R wt;
          if (hv < ybot)
            wt = R(l * (hv - ymin) * ioff[a]);
          else if (hv <= ytop)
            wt = R(l);
          else if (hv < ymax - kEps)
            wt = R(l * (ymax - hv) * ioff[a]);
          else
            break;
          rows.push_back((abase + h) * nv);
          w.push_back(wt);
        }
      }
      T *col = vol + vox_index(i, j, ny, nz);
      for (size_t m = 0; m < rows.size(); m++) {
        const T *p = pix + rows[m];
        const T wt = T(w[m]);
        switch (map_type) {
        case 1:
          for (int v = 0; v < nv; v++)
            col[v] += p[v] * wt;
          break;
        case 2:
          for (int z = 0; z < nz && 2 * z + 1 < nv; z++)
            col[z] += (p[2 * z] + p[2 * z + 1]) * wt;
          break;
        case 4:
          for (int z = 0; z < nz && 4 * z + 3 < nv; z++)
            col[z] += (p[4 * z] + p[4 * z + 1] + p[4 * z + 2] + p[4 * z + 3]) * wt;
          break;
        default:
          for (int v = 0; v < nv; v++)
            if (map[v] >= 0 && map[v] < nz)
              col[map[v]] += p[v] * wt;
          break;
        }
      }
    }
  }
}

// ---------------------------------------------------------------- cone beam

// Per-row and per-slice tables shared by the cone projectors
// (c2D.cpp:480-516 and :959-1010).
template <class R> struct cone_tables {
  int mid;
  R inv_dz, pzbz, pzdv, z_1, z_nm;
  std::vector<R> delta_z, inv_delz, vox_z, d_conv; // d_conv (nh, nv)
};

template <class R>
bool make_cone_tables(const rs_geometry *g, cone_tables<R> &t) {
  const double sx = g->source[0], sy = g->source[1], sz = g->source[2];
  const int nv = g->nv, nh = g->nh, nz = g->nz;
  t.mid = -1;
  for (int i = 0; i < nv; i++)
    if (g->v_pixels[i] > sz) {
      t.mid = i;
      break;
    }
  if (t.mid <= 0)
    return false; // the reference indexes v_pixels[mid - 1] unchecked
  t.d_conv.resize(size_t(nh) * nv);
  const double x2 = (g->detector_x - sx) * (g->detector_x - sx);
  for (int i = 0; i < nh; i++) {
    const double xy2 = x2 + (g->h_pixels[i] - sy) * (g->h_pixels[i] - sy);
    for (int j = 0; j < nv; j++)
      t.d_conv[size_t(i) * nv + j] =
          R(std::sqrt(xy2 + (g->v_pixels[j] - sz) * (g->v_pixels[j] - sz)));
  }
  t.inv_dz = R(1.0 / g->size[2]);
  t.pzbz = R((sz - g->origin[2]) / g->size[2]);
  const double v_step = g->v_pixels[1] - g->v_pixels[0];
  t.pzdv = R((sz - g->v_pixels[0]) / v_step);
  t.z_1 = R((g->origin[2] + g->size[2] - sz) / v_step);
  t.z_nm = R((g->origin[2] + double(nz - 1) * g->size[2] - sz) / v_step);
  t.delta_z.resize(nv);
  t.inv_delz.resize(nv);
  for (int i = 0; i < nv; i++) {
    t.delta_z[i] = R(g->v_pixels[i] - sz);
    t.inv_delz[i] = R(1.0 / double(t.delta_z[i]));
  }
  t.vox_z.resize(nz + 1);
  for (int i = 0; i <= nz; i++)
    t.vox_z[i] = R(g->origin[2] + double(i) * g->size[2] - sz);
  return true;
}

// Detector-column range that can see the xy box [x0,xn) x [y0,yn) from the
// source at angle a (c2D.cpp:558-600 and :831-901).
void cone_hrange(const rs_geometry *g, double c, double s, double p1x,
                 double p1y, double x0, double xn, double y0, double yn,
                 int &hmin, int &hmax) {
  const double sx = g->source[0];
  const double l = g->detector_x - sx;
  const double step = g->h_pixels[1] - g->h_pixels[0];
  const double ipix = 1.0 / step;
  const double hpix0 = (g->source[1] - g->h_pixels[0]) / step;
  const double dx0 = x0 - p1x, dy0 = y0 - p1y, dxn = xn - p1x, dyn = yn - p1y;
  const double cx0 = c * x0 - sx, cxn = c * xn - sx;
  const double sy0 = s * y0, syn = s * yn;
  double y00, y01, y10, y11;
  if (std::abs(s) > std::abs(c)) {
    const double il = l / s;
    y00 = (c - dx0 / (sy0 + cx0)) * il;
    y01 = (c - dx0 / (syn + cx0)) * il;
    y10 = (c - dxn / (sy0 + cxn)) * il;
    y11 = (c - dxn / (syn + cxn)) * il;
  } else {
    const double il = l / c;
    y00 = (-s + dy0 / (cx0 + sy0)) * il;
    y01 = (-s + dyn / (cx0 + syn)) * il;
    y10 = (-s + dy0 / (cxn + sy0)) * il;
    y11 = (-s + dyn / (cxn + syn)) * il;
  }
  const int h00 = int(std::floor(y00 * ipix + hpix0));
  const int h01 = int(std::floor(y01 * ipix + hpix0));
  const int h10 = int(std::floor(y10 * ipix + hpix0));
  const int h11 = int(std::floor(y11 * ipix + hpix0));
  hmin = std::max(std::min(std::min(h00, h01), std::min(h10, h11)), 0);
  hmax = std::min(std::max(std::max(h00, h01), std::max(h10, h11)), g->nh - 1);
}

// xy Siddon walk of one cone ray in voxel-normalised coordinates
// (c2D.cpp:193-467).  alpha is the fraction of source->pixel; alphas[0] is
// the entry and cells[m-1] spans [alphas[m-1], alphas[m]].
template <class R>
void cone_walk(const rs_geometry *g, double p1x, double p1y, double p2x,
               double p2y, std::vector<i64> &cells, std::vector<R> &alphas) {
  cells.clear();
  alphas.clear();
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const double q1x = (p1x - g->origin[0]) / g->size[0];
  const double q1y = (p1y - g->origin[1]) / g->size[1];
  const double q2x = (p2x - g->origin[0]) / g->size[0];
  const double q2y = (p2y - g->origin[1]) / g->size[1];
  const double ddx = q2x - q1x, ddy = q2y - q1y;
  const double inv_dx = 1.0 / ddx, inv_dy = 1.0 / ddy;
  if (std::abs(ddx) < kEps) {
    if (std::abs(ddy) < kEps)
      return;
    const int i = int(std::floor(q1x));
    if (i < 0 || i >= nx)
      return;
    if (ddy < 0.0) {
      alphas.push_back(R((double(ny) - q1y) * inv_dy));
      for (int j = ny - 1; j >= 0; j--) {
        alphas.push_back(R((double(j) - q1y) * inv_dy));
        cells.push_back(vox_index(i, j, ny, nz));
      }
    } else {
      alphas.push_back(R((0.0 - q1y) * inv_dy));
      for (int j = 0; j < ny; j++) {
        alphas.push_back(R((double(j + 1) - q1y) * inv_dy));
        cells.push_back(vox_index(i, j, ny, nz));
      }
    }
    return;
  }
  if (std::abs(ddy) < kEps) {
    const int j = int(std::floor(q1y));
    if (j < 0 || j >= ny)
      return;
    if (ddx < 0.0) {
      alphas.push_back(R((double(nx) - q1x) * inv_dx));
      for (int i = nx - 1; i >= 0; i--) {
        alphas.push_back(R((double(i) - q1x) * inv_dx));
        cells.push_back(vox_index(i, j, ny, nz));
      }
    } else {
      alphas.push_back(R((0.0 - q1x) * inv_dx));
      for (int i = 0; i < nx; i++) {
        alphas.push_back(R((double(i + 1) - q1x) * inv_dx));
        cells.push_back(vox_index(i, j, ny, nz));
      }
    }
    return;
  }
  const double ax0 = (0.0 - q1x) * inv_dx, ay0 = (0.0 - q1y) * inv_dy;
  const double axn = (double(nx) - q1x) * inv_dx;
  const double ayn = (double(ny) - q1y) * inv_dy;
  const double amin =
      std::max(std::max(std::min(ax0, axn), std::min(ay0, ayn)), 0.0);
  const double amax =
      std::min(std::min(std::max(ax0, axn), std::max(ay0, ayn)), 1.0);
  if (!(amin < amax - kEps))
    return;
  const int sx = ddx > 0.0 ? 1 : -1, sy = ddy > 0.0 ? 1 : -1;
  auto ax = [&](int i) { return (double(i) - q1x) * inv_dx; };
  auto ay = [&](int j) { return (double(j) - q1y) * inv_dy; };
  auto cx = [&]() { return int(std::floor(q1x + amin * ddx)); };
  auto cy = [&]() { return int(std::floor(q1y + amin * ddy)); };
  int x = 0, y = 0;
  if (sx > 0 && sy > 0) {
    if (amin == ax0) {
      x = 0;
      y = cy();
    } else if (amin == ay0) {
      x = cx();
      y = 0;
    }
  } else if (sx > 0) {
    if (amin == ayn) {
      x = cx();
      y = ny - 1;
    } else if (amin == ax0) {
      x = 0;
      y = cy();
    }
  } else if (sy > 0) {
    if (amin == axn) {
      x = nx - 1;
      y = cy();
    } else if (amin == ay0) {
      x = cx();
      y = 0;
    }
  } else {
    if (amin == axn) {
      x = nx - 1;
      y = (amin == ayn) ? ny - 1 : cy();
    } else if (amin == ayn) {
      x = cx();
      y = ny - 1;
    }
  }
  alphas.push_back(R(amin));
  while ((sx > 0 ? x < nx : x >= 0) && (sy > 0 ? y < ny : y >= 0)) {
    const double nxa = ax(sx > 0 ? x + 1 : x);
    const double nya = ay(sy > 0 ? y + 1 : y);
    // a cell outside the volume (entry rounding) contributes nothing
    cells.push_back((x >= 0 && x < nx && y >= 0 && y < ny)
                        ? vox_index(x, y, ny, nz)
                        : -1);
    if (nxa < nya - kEps) {
      alphas.push_back(R(nxa));
      x += sx;
    } else if (nya < nxa - kEps) {
      alphas.push_back(R(nya));
      y += sy;
    } else {
      alphas.push_back(R(std::max(nxa, nya)));
      x += sx;
      y += sy;
    }
  }
}

// z split of one cone ray over its xy cells (c2D.cpp:17-191): rows below
// the source (v < mid) descend and may spill into k-1, rows above into k+1.
template <class T, class R>
void cone_add_cells(T *pix, const T *vol, const std::vector<i64> &cells,
                    const std::vector<R> &alphas, const cone_tables<R> &t,
                    int nv, int nz) {
  const int n = int(alphas.size());
  if (n < 2)
    return;
  const int nzm1 = nz - 1, midp = t.mid;
  const R *dz = t.delta_z.data(), *iz = t.inv_delz.data(), *vz = t.vox_z.data();
  std::vector<R> ainv(n);
  for (int m = 0; m < n; m++)
    ainv[m] = alphas[m] * t.inv_dz;
  auto col = [&](int m) -> const T * {
    const i64 c = cells[m - 1];
    return c < 0 ? nullptr : vol + c;
  };
  // first segment at which the lowest / highest row leaves the volume
  int min_xy_all = n;
  for (int m = 1; m < n; m++) {
    const int k = int(std::floor(t.pzbz + ainv[m - 1] * dz[0]));
    if (k <= 0) {
      min_xy_all = (k == 0) ? m : 0;
      break;
    }
  }
  int max_xy_all = n;
  for (int m = 1; m < n; m++) {
    const int k = int(std::floor(t.pzbz + ainv[m - 1] * dz[nv - 1]));
    if (k >= nzm1) {
      max_xy_all = (k == nzm1) ? m : 0;
      break;
    }
  }
  // rows whose whole path stays inside
  int min_v_all = midp;
  for (int v = 0; v < midp; v++)
    if (int(std::floor(t.pzbz + ainv[n - 2] * dz[v])) > 0) {
      min_v_all = v;
      break;
    }
  int max_v_all = midp - 1;
  for (int v = nv - 1; v >= midp; v--)
    if (int(std::floor(t.pzbz + ainv[n - 2] * dz[v])) < nzm1) {
      max_v_all = v;
      break;
    }
  const int ncom = std::min(min_xy_all, max_xy_all);
  auto seg = [&](int m, int v0, int v1, R a0) {
    // rows [v0, v1) of cell m, all known to stay inside the volume
    const T *c = col(m);
    const R a1 = alphas[m];
    const R av = ainv[m - 1];
    if (!c)
      return;
    for (int v = v0; v < v1; v++) {
      const int k = int(t.pzbz + av * dz[v]);
      const int kn = v < midp ? k - 1 : k + 1;
      const R az = vz[v < midp ? k : k + 1] * iz[v];
      const R mz = std::min(az, a1);
      pix[v] += T(c[k] * T(mz - a0) + c[kn] * T(a1 - mz));
    }
  };
  R a0 = alphas[0];
  for (int m = 1; m < ncom; m++) {
    seg(m, 0, nv, a0);
    a0 = alphas[m];
  }
  // the reference starts this loop at m = ncom, reading ainv[-1] when
  // ncom == 0 (a row missing the volume at entry); that case is skipped.
  for (int m = std::max(ncom, 1); m < n; m++) {
    seg(m, min_v_all, max_v_all + 1, a0);
    a0 = alphas[m];
  }
  if (ncom < 1)
    return;
  const R pzbz1 = R(t.pzbz + 1.0);
  a0 = alphas[ncom - 1];
  for (int m = ncom; m < n; m++) {
    const T *c = col(m);
    const R av = ainv[m - 1], a1 = alphas[m];
    for (int v = min_v_all - 1; v >= 0 && c; v--) {
      const int k = int(pzbz1 + av * dz[v]) - 1;
      if (k > 0) {
        const R mz = std::min(R(vz[k] * iz[v]), a1);
        pix[v] += T(c[k] * T(mz - a0) + c[k - 1] * T(a1 - mz));
      } else if (k == 0) {
        const R mz = std::min(R(vz[0] * iz[v]), a1);
        pix[v] += T(c[0] * T(mz - a0));
      } else
        break;
    }
    a0 = a1;
  }
  a0 = alphas[ncom - 1];
  for (int m = ncom; m < n; m++) {
    const T *c = col(m);
    const R av = ainv[m - 1], a1 = alphas[m];
    for (int v = max_v_all + 1; v < nv && c; v++) {
      const int k = int(t.pzbz + av * dz[v]);
      if (k < nzm1) {
        const R mz = std::min(R(vz[k + 1] * iz[v]), a1);
        pix[v] += T(c[k] * T(mz - a0) + c[k + 1] * T(a1 - mz));
      } else if (k == nzm1) {
        const R mz = std::min(R(vz[nz] * iz[v]), a1);
        pix[v] += T(c[nzm1] * T(mz - a0));
      } else
        break;
    }
    a0 = a1;
  }
}

// cone_beam::f2D (c2D.cpp:469-625): whole volume as one block.
template <class T> void cb_forward(const rs_geometry *g, const T *vol, T *pix) {
  typedef typename types<T>::R R;
  cone_tables<R> t;
  if (!make_cone_tables(g, t))
    return;
  const int nh = g->nh, nv = g->nv;
  const double x0 = g->origin[0], xn = g->origin[0] + g->nx * g->size[0];
  const double y0 = g->origin[1], yn = g->origin[1] + g->ny * g->size[1];
#pragma omp parallel for schedule(dynamic)
  for (int a = 0; a < g->na; a++) {
    std::vector<i64> cells;
    std::vector<R> alphas;
    const double c = std::cos(g->angles[a]), s = std::sin(g->angles[a]);
    const double p1x = c * g->source[0] - s * g->source[1];
    const double p1y = s * g->source[0] + c * g->source[1];
    int hmin, hmax;
    cone_hrange(g, c, s, p1x, p1y, x0, xn, y0, yn, hmin, hmax);
    for (int h = hmin; h <= hmax; h++) {
      const double p2x = c * g->detector_x - s * g->h_pixels[h];
      const double p2y = s * g->detector_x + c * g->h_pixels[h];
      cone_walk<R>(g, p1x, p1y, p2x, p2y, cells, alphas);
      cone_add_cells<T, R>(pix + (i64(a) * nh + h) * nv, vol, cells, alphas, t,
                           nv, g->nz);
    }
    T *row = pix + i64(a) * nh * nv;
    for (i64 hv = 0; hv < i64(nh) * nv; hv++)
      row[hv] *= T(t.d_conv[hv]);
  }
}

// cone_beam::b2D (c2D.cpp:1052-1119 -> :948-1050) with bproject_ah
// (:788-946) and calc_ah_z (:640-751).  The sinogram is first scaled by the
// source-pixel distance into a copy, then gathered per voxel column.
template <class T> void cb_backward(const rs_geometry *g, const T *pix, T *vol) {
  typedef typename types<T>::R R;
  cone_tables<R> t;
  if (!make_cone_tables(g, t))
    return;
  const int na = g->na, nh = g->nh, nv = g->nv, nx = g->nx, ny = g->ny,
            nz = g->nz, nzm1 = nz - 1, midp = t.mid;
  std::vector<T> dpix(size_t(na) * nh * nv);
  for (int a = 0; a < na; a++)
    for (i64 hv = 0; hv < i64(nh) * nv; hv++)
      dpix[i64(a) * nh * nv + hv] = pix[i64(a) * nh * nv + hv] * T(t.d_conv[hv]);
  const double sx = g->source[0], sy = g->source[1];
  std::vector<double> ca(na), sa(na), p1x(na), p1y(na), cdx(na), sdx(na);
  for (int a = 0; a < na; a++) {
    ca[a] = std::cos(g->angles[a]);
    sa[a] = std::sin(g->angles[a]);
    p1x[a] = ca[a] * sx - sa[a] * sy;
    p1y[a] = sa[a] * sx + ca[a] * sy;
    cdx[a] = ca[a] * g->detector_x;
    sdx[a] = sa[a] * g->detector_x;
  }
  const R *dz = t.delta_z.data(), *iz = t.inv_delz.data(), *vz = t.vox_z.data();
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nx; i++) {
    std::vector<i64> rows;
    std::vector<R> a0s, a1s;
    std::vector<int> kv(nv);
    const double x0 = g->origin[0] + double(i) * g->size[0];
    const double xn = g->origin[0] + double(i + 1) * g->size[0];
    for (int j = 0; j < ny; j++) {
      const double y0 = g->origin[1] + double(j) * g->size[1];
      const double yn = g->origin[1] + double(j + 1) * g->size[1];
      rows.clear();
      a0s.clear();
      a1s.clear();
      for (int a = 0; a < na; a++) {
        int hmin, hmax;
        cone_hrange(g, ca[a], sa[a], p1x[a], p1y[a], x0, xn, y0, yn, hmin, hmax);
        const double dx0 = x0 - p1x[a], dy0 = y0 - p1y[a];
        const double dxn = xn - p1x[a], dyn = yn - p1y[a];
        for (int h = hmin; h <= hmax; h++) {
          const double p2x = cdx[a] - sa[a] * g->h_pixels[h];
          const double p2y = sdx[a] + ca[a] * g->h_pixels[h];
          const double ddx = p2x - p1x[a], ddy = p2y - p1y[a];
          if (std::abs(ddx) < kEps || std::abs(ddy) < kEps)
            continue; // rejected by the reference ("Ooops")
          const double idx = 1.0 / ddx, idy = 1.0 / ddy;
          const double ax0 = dx0 * idx, ay0 = dy0 * idy;
          const double axn = dxn * idx, ayn = dyn * idy;
          const double amin =
              std::max(std::max(std::min(ax0, axn), std::min(ay0, ayn)), 0.0);
          const double amax =
              std::min(std::min(std::max(ax0, axn), std::max(ay0, ayn)), 1.0);
          if (amin < amax - kEps) {
            rows.push_back((i64(a) * nh + h) * nv);
            a0s.push_back(R(amin));
            a1s.push_back(R(amax));
          }
        }
      }
      const int n = int(rows.size());
      if (!n)
        continue;
      T *col = vol + vox_index(i, j, ny, nz);
      // rows [min_v, max_v) stay inside the column for every segment
      const R pzdeps = R(double(t.pzdv) * (1.0 + double(kEps)));
      int min_v = 0;
      for (int m = 0; m < n; m++)
        min_v = std::max(min_v, int(std::ceil(R(pzdeps + R(t.z_1 / a0s[m])))));
      int max_v = nv;
      for (int m = 0; m < n; m++)
        max_v = std::min(max_v, int(std::floor(R(t.pzdv + R(t.z_nm / a0s[m])))));
      const R pzbz1 = R(double(t.pzbz) + 1.0);
      std::fill(kv.begin(), kv.end(), 0);
      for (int m = 0; m < n; m++) {
        const T *p = dpix.data() + rows[m];
        const R a0 = a0s[m], a1 = a1s[m], av = a0 * t.inv_dz;
        for (int v = min_v; v < max_v; v++)
          kv[v] = int(t.pzbz + av * dz[v]);
        for (int v = min_v; v < midp; v++) {
          // k below 1 here is the reference's unchecked edge (see header)
          const int k = kv[v];
          if (k < 1 || k > nzm1)
            continue;
          const R mz = std::min(R(vz[k] * iz[v]), a1);
          col[k] += p[v] * T(mz - a0);
          col[k - 1] += p[v] * T(a1 - mz);
        }
        for (int v = midp; v < max_v; v++) {
          const int k = kv[v];
          if (k < 0 || k >= nzm1)
            continue;
          const R mz = std::min(R(vz[k + 1] * iz[v]), a1);
          col[k] += p[v] * T(mz - a0);
          col[k + 1] += p[v] * T(a1 - mz);
        }
      }
      for (int m = 0; m < n; m++) {
        const T *p = dpix.data() + rows[m];
        const R a0 = a0s[m], a1 = a1s[m], av = a0 * t.inv_dz;
        for (int v = min_v - 1; v >= 0; v--) {
          const int k = int(pzbz1 + av * dz[v]) - 1;
          if (k > 0) {
            if (k > nzm1)
              continue;
            const R mz = std::min(R(vz[k] * iz[v]), a1);
            col[k] += p[v] * T(mz - a0);
            col[k - 1] += p[v] * T(a1 - mz);
          } else if (k == 0) {
            const R mz = std::min(R(vz[0] * iz[v]), a1);
            col[0] += p[v] * T(mz - a0);
          } else
            break;
        }
        for (int v = std::max(max_v, 0); v < nv; v++) {
          const int k = int(t.pzbz + av * dz[v]);
          if (k < nzm1) {
            if (k < 0)
              continue;
            const R mz = std::min(R(vz[k + 1] * iz[v]), a1);
            col[k] += p[v] * T(mz - a0);
            col[k + 1] += p[v] * T(a1 - mz);
          } else if (k == nzm1) {
            const R mz = std::min(R(vz[k + 1] * iz[v]), a1);
            col[k] += p[v] * T(mz - a0);
          } else
            break;
        }
      }
    }
  }
}

// ---------------------------------------------------------------- vectors
// blas.hpp:204-284 summation order with one thread: per slowest index a
// partial of partials, then a running total.
template <class T> T norm3(const T *v, i64 n0, i64 n1, i64 n2) {
  T norm = 0;
  for (i64 i = 0; i < n0; i++) {
    T n1s = 0;
    for (i64 j = 0; j < n1; j++) {
      T n2s = 0;
      const T *p = v + (i * n1 + j) * n2;
      for (i64 k = 0; k < n2; k++)
        n2s += p[k] * p[k];
      n1s += n2s;
    }
    norm += n1s;
  }
  return norm;
}

// ------------------------------------------------------------ regularisers

// tikhonov.cpp:5-33: 0.25 * (four xy neighbours) - centre, mirrored edges.
template <class T> void tikhonov(int nx, int ny, int nz, const T *a, T *b) {
  for (int i = 0; i < nx; i++) {
    const int i1 = (i + 1 >= nx) ? i - 1 : i + 1;
    const int i2 = (i - 1 < 0) ? i + 1 : i - 1;
    for (int j = 0; j < ny; j++) {
      const int j1 = (j + 1 >= ny) ? j - 1 : j + 1;
      const int j2 = (j - 1 < 0) ? j + 1 : j - 1;
      const T *p1 = a + vox_index(i1, j, ny, nz), *p2 = a + vox_index(i2, j, ny, nz);
      const T *p3 = a + vox_index(i, j1, ny, nz), *p4 = a + vox_index(i, j2, ny, nz);
      const T *pc = a + vox_index(i, j, ny, nz);
      T *q = b + vox_index(i, j, ny, nz);
      for (int k = 0; k < nz; k++)
        q[k] = T(0.25 * double(p1[k] + p2[k] + p3[k] + p4[k]) - double(pc[k]));
    }
  }
}

inline int sgn(double x) { return (x > 0) - (x < 0); }

// total_v.cpp:21-195: divergence of a gradient normalised by a minmod
// estimate of the cross terms; Neumann (mirror) boundaries.  Note the
// reference reuses cross terms (T2 takes denom3x, T3 takes denom2y and
// denom2x), reproduced as is.
template <class T> void total_variation(int nx, int ny, int nz, const T *A, T *B) {
  const i64 n = i64(nx) * ny * nz;
  std::vector<T> D1(n), D2(n), D3(n);
  const T eps = T(FLT_EPSILON);
  auto at = [&](int i, int j, int k) { return A[vox_index(i, j, ny, nz) + k]; };
  for (int i = 0; i < nx; i++) {
    const int i1 = (i + 1 >= nx) ? i - 1 : i + 1;
    const int i2 = (i - 1 < 0) ? i + 1 : i - 1;
    for (int j = 0; j < ny; j++) {
      const int j1 = (j + 1 >= ny) ? j - 1 : j + 1;
      const int j2 = (j - 1 < 0) ? j + 1 : j - 1;
      for (int k = 0; k < nz; k++) {
        const int k1 = (k + 1 >= nz) ? k - 1 : k + 1;
        const int k2 = (k - 1 < 0) ? k + 1 : k - 1;
        const T c = at(i, j, k);
        const T x1 = at(i1, j, k) - c, y1 = at(i, j1, k) - c;
        const T y0 = c - at(i, j2, k), x0 = c - at(i2, j, k);
        const T z1 = at(i, j, k1) - c, z0 = c - at(i, j, k2);
        const T d1x = x1 * x1, d1y = y1 * y1, d1z = z1 * z1;
        T d2x = T(0.5 * (sgn(y1) + sgn(y0)) * std::min(std::abs(y1), std::abs(y0)));
        T d2y = T(0.5 * (sgn(x1) + sgn(x0)) * std::min(std::abs(x1), std::abs(x0)));
        d2x = d2x * d2x;
        d2y = d2y * d2y;
        T d3x = T(0.5 * (sgn(z1) + sgn(z0)) * std::min(std::abs(z1), std::abs(z0)));
        d3x = d3x * d3x;
        const T t1 = std::sqrt(d1x + d2x + d3x + eps);
        const T t2 = std::sqrt(d1y + d2y + d3x + eps);
        const T t3 = std::sqrt(d1z + d2y + d2x + eps);
        const i64 o = vox_index(i, j, ny, nz) + k;
        D1[o] = x1 / t1;
        D2[o] = y1 / t2;
        D3[o] = z1 / t3;
      }
    }
  }
  for (int i = 0; i < nx; i++) {
    const int i2 = (i - 1 < 0) ? i + 1 : i - 1;
    for (int j = 0; j < ny; j++) {
      const int j2 = (j - 1 < 0) ? j + 1 : j - 1;
      for (int k = 0; k < nz; k++) {
        const int k2 = (k - 1 < 0) ? k + 1 : k - 1;
        const i64 o = vox_index(i, j, ny, nz) + k;
        const T dv1 = D1[o] - D1[vox_index(i2, j, ny, nz) + k];
        const T dv2 = D2[o] - D2[vox_index(i, j2, ny, nz) + k];
        const T dv3 = D3[o] - D3[vox_index(i, j, ny, nz) + k2];
        B[o] = dv1 + dv2 + dv3;
      }
    }
  }
}

template <class T> void regularize(int alg, int nx, int ny, int nz, const T *a, T *b) {
  if (alg == RS_TIKHONOV)
    tikhonov(nx, ny, nz, a, b);
  else
    total_variation(nx, ny, nz, a, b);
}

// ------------------------------------------------------------------ solvers
template <class T> struct problem {
  const rs_geometry *g;
  i64 nvox, npix;
  void fp(const T *x, T *p) const {
    std::fill(p, p + npix, T(0));
    if (g->kind == 0)
      pb_forward(g, x, p);
    else
      cb_forward(g, x, p);
  }
  void bp(const T *p, T *x) const {
    std::fill(x, x + nvox, T(0));
    if (g->kind == 0)
      pb_backward(g, p, x);
    else
      cb_backward(g, p, x);
  }
  T vnorm(const T *x) const { return norm3(x, g->nx, g->ny, g->nz); }
  T pnorm(const T *p) const { return norm3(p, g->na, g->nh, g->nv); }
};

// cgls_base::reconstruct with cgls_3d (Algorithms/cgls.cpp:26-157).  The
// residual starts at b even for a warm start (the reference's behaviour).
template <class T>
void cgls(const problem<T> &P, const T *sino, T *x, int niter, double *norms) {
  std::vector<T> b(sino, sino + P.npix), d(P.nvox), Ad(P.npix), s(P.nvox);
  P.bp(b.data(), d.data());
  T normr2 = P.vnorm(d.data());
  for (int it = 0; it < niter; it++) {
    P.fp(d.data(), Ad.data());
    T alpha = P.pnorm(Ad.data());
    alpha = normr2 / alpha;
    for (i64 i = 0; i < P.nvox; i++)
      x[i] += alpha * d[i];
    const T malpha = -alpha;
    for (i64 i = 0; i < P.npix; i++)
      b[i] += malpha * Ad[i];
    P.bp(b.data(), s.data());
    const double nnew = double(P.vnorm(s.data()));
    const T beta = T(nnew / double(normr2));
    normr2 = T(nnew);
    for (i64 i = 0; i < P.nvox; i++)
      d[i] = beta * d[i] + s[i];
    if (norms)
      norms[it] = std::sqrt(double(normr2));
  }
}

// sirt::reconstruct (Algorithms/sirt.cpp:15-80).
template <class T> void sirt(const problem<T> &P, const T *sino, T *x, int niter) {
  std::vector<T> R(P.npix), C(P.nvox), ones_v(P.nvox, T(1)), ones_p(P.npix, T(1));
  P.fp(ones_v.data(), R.data());
  for (auto &r : R)
    r = (r > T(0)) ? T(1.0 / double(r)) : T(0);
  P.bp(ones_p.data(), C.data());
  for (auto &c : C)
    c = (c > T(0)) ? T(1.0 / double(c)) : T(0);
  std::vector<T> r(P.npix), bpv(P.nvox);
  for (int it = 0; it < niter; it++) {
    P.fp(x, r.data());
    for (i64 i = 0; i < P.npix; i++)
      r[i] = (T(-1) * r[i] + sino[i]) * R[i];
    P.bp(r.data(), bpv.data());
    for (i64 i = 0; i < P.nvox; i++) {
      const T v = x[i] + T(1) * (bpv[i] * C[i]);
      x[i] = std::max(v, T(0));
    }
  }
}

// mlem::reconstruct (Algorithms/mlem.cpp:15-80).
template <class T> void mlem(const problem<T> &P, const T *sino, T *x, int niter) {
  std::fill(x, x + P.nvox, T(1));
  std::vector<T> N(P.nvox), ones_p(P.npix, T(1));
  P.bp(ones_p.data(), N.data());
  for (auto &v : N)
    if (v != T(0))
      v = T(1.0 / double(v));
  std::vector<T> est(P.npix), ratio(P.npix), bpr(P.nvox);
  for (int it = 0; it < niter; it++) {
    P.fp(x, est.data());
    for (i64 i = 0; i < P.npix; i++) {
      const T q = (est[i] != T(0)) ? sino[i] / est[i] : T(0);
      ratio[i] = std::max(q, T(0));
    }
    P.bp(ratio.data(), bpr.data());
    for (i64 i = 0; i < P.nvox; i++) {
      const T v = x[i] * (N[i] * bpr[i]);
      x[i] = std::max(v, T(0));
    }
  }
}

// cgls_regularize::reconstruct (Algorithms/cgls.cpp:343-411).  Ad_vox is
// allocated once and accumulated, never reset; the r_vox update of the
// reference only touches memory that is never read and is omitted.
template <class T>
void cgls_reg(const problem<T> &P, int alg, const T *sino, T *x, int niter,
              double lambda, double *norms) {
  const rs_geometry *g = P.g;
  std::vector<T> r(sino, sino + P.npix), d(P.nvox), Adv(P.nvox, T(0)),
      Adp(P.npix), L(P.nvox), s(P.nvox);
  P.bp(r.data(), d.data());
  T normr2 = P.vnorm(d.data());
  const T lam = T(lambda);
  for (int it = 0; it < niter; it++) {
    P.fp(d.data(), Adp.data());
    regularize(alg, g->nx, g->ny, g->nz, d.data(), L.data());
    for (i64 i = 0; i < P.nvox; i++)
      Adv[i] += lam * L[i];
    T alpha = T(P.pnorm(Adp.data()) + P.vnorm(Adv.data()));
    alpha = normr2 / alpha;
    for (i64 i = 0; i < P.nvox; i++)
      x[i] += alpha * d[i];
    const T malpha = -alpha;
    for (i64 i = 0; i < P.npix; i++)
      r[i] += malpha * Adp[i];
    regularize(alg, g->nx, g->ny, g->nz, x, L.data());
    for (i64 i = 0; i < P.nvox; i++)
      x[i] += lam * L[i];
    P.bp(r.data(), s.data());
    const double nnew = double(P.vnorm(s.data()));
    const T beta = T(nnew / double(normr2));
    normr2 = T(nnew);
    for (i64 i = 0; i < P.nvox; i++)
      d[i] = beta * d[i] + s[i];
    if (norms)
      norms[it] = std::sqrt(double(normr2));
  }
}

template <class T>
int solve(const rs_geometry *g, int alg, const T *sino, T *x, int niter,
          double lambda, double *norms) {
  problem<T> P{g, i64(g->nx) * g->ny * g->nz, i64(g->na) * g->nh * g->nv};
  switch (alg) {
  case RS_CGLS:
    cgls(P, sino, x, niter, norms);
    break;
  case RS_SIRT:
    sirt(P, sino, x, niter);
    break;
  case RS_MLEM:
    mlem(P, sino, x, niter);
    break;
  case RS_TIKHONOV:
  case RS_TV:
    cgls_reg(P, alg, sino, x, niter, lambda, norms);
    break;
  default:
    return 1;
  }
  // every reconstruction is clamped at zero (voxels.cpp:187, :272, :352)
  for (i64 i = 0; i < P.nvox; i++)
    x[i] = std::max(x[i], T(0));
  return 0;
}

} // namespace

extern "C" {

void rs_fp_f32(const rs_geometry *g, const float *vol, float *pix) {
  if (g->kind == 0)
    pb_forward(g, vol, pix);
  else
    cb_forward(g, vol, pix);
}
void rs_bp_f32(const rs_geometry *g, const float *pix, float *vol) {
  if (g->kind == 0)
    pb_backward(g, pix, vol);
  else
    cb_backward(g, pix, vol);
}
void rs_fp_f64(const rs_geometry *g, const double *vol, double *pix) {
  if (g->kind == 0)
    pb_forward(g, vol, pix);
  else
    cb_forward(g, vol, pix);
}
void rs_bp_f64(const rs_geometry *g, const double *pix, double *vol) {
  if (g->kind == 0)
    pb_backward(g, pix, vol);
  else
    cb_backward(g, pix, vol);
}
int rs_solve_f32(const rs_geometry *g, int alg, const float *sino, float *x,
                 int niter, double lambda, double *norms) {
  return solve(g, alg, sino, x, niter, lambda, norms);
}
int rs_solve_f64(const rs_geometry *g, int alg, const double *sino, double *x,
                 int niter, double lambda, double *norms) {
  return solve(g, alg, sino, x, niter, lambda, norms);
}
void rs_regularize_f32(int alg, int nx, int ny, int nz, const float *a, float *b) {
  regularize(alg, nx, ny, nz, a, b);
}
void rs_regularize_f64(int alg, int nx, int ny, int nz, const double *a, double *b) {
  regularize(alg, nx, ny, nz, a, b);
}

} // extern "C"

extern "C" {
// -log(p) with the C library's float logarithm, as Diamond::read_scans and
// Nikon_XTek::read_scans apply it to transmission data
// (diamond.cpp:442, Readers/xtek.cpp:556).
void rs_neglog_f32(const float *in, float *out, long long n) {
  for (long long i = 0; i < n; i++)
    out[i] = -std::log(in[i]);
}

void rs_expneg_f32(const float *in, float *out, long long n) {
  for (long long i = 0; i < n; i++)
    out[i] = std::exp(-in[i]);
}
}

// ---------------------------------------------------------------------------
// High-peaks filter (Core/src/diamond.cpp:513-617).  Per detector row v, and
// num_pix times: first every angle a < na-1 becomes p[a+1] + d with
// d = p[a] - p[a+1] raised to -jump when below it (the comparison is FP64,
// the float difference against the real jump); then, on that result, every
// angle a+1 > 0 becomes p[a] + d with d = p[a+1] - p[a] limited the same
// way.  Each pass forms all its differences before it writes (the
// reference's temp1 plane), which this restatement keeps as written.
extern "C" int rs_high_peaks_f32(float *p, int na, int nh, int nv, double jump, int num_pix) {
  if (jump < 0.0 || num_pix < 1 || num_pix >= na)
    return 1;
  auto at = [&](int a, int h, int v) -> float & {
    return p[(size_t(a) * nh + h) * nv + v];
  };
  std::vector<float> d(size_t(na - 1) * nh);
  for (int v = 0; v < nv; v++)
    for (int k = 0; k < num_pix; k++) {
      for (int a = 0; a + 1 < na; a++)
        for (int h = 0; h < nh; h++) {
          float t = at(a, h, v) - at(a + 1, h, v);
          if (double(t) < -jump)
            t = float(-jump);
          d[size_t(a) * nh + h] = t;
        }
      for (int a = 0; a + 1 < na; a++)
        for (int h = 0; h < nh; h++)
          at(a, h, v) = at(a + 1, h, v) + d[size_t(a) * nh + h];
      for (int a = 0; a + 1 < na; a++)
        for (int h = 0; h < nh; h++) {
          float t = at(a + 1, h, v) - at(a, h, v);
          if (double(t) < -jump)
            t = float(-jump);
          d[size_t(a) * nh + h] = t;
        }
      for (int a = na - 2; a >= 0; a--)
        for (int h = 0; h < nh; h++)
          at(a + 1, h, v) = at(a, h, v) + d[size_t(a) * nh + h];
    }
  return 0;
}

// ---------------------------------------------------------------------------
// Column ring-artefact filter (Core/src/diamond.cpp:619-658): per (h, v),
// the FP64 sum over angles in order, divided by na, rounded to float once
// and subtracted from every angle.
extern "C" void rs_column_ring_f32(float *p, int na, int nh, int nv) {
  for (int v = 0; v < nv; v++)
    for (int h = 0; h < nh; h++) {
      double s = 0.0;
      for (int a = 0; a < na; a++)
        s += double(p[(size_t(a) * nh + h) * nv + v]);
      s /= double(na);
      const float m = float(s);
      for (int a = 0; a < na; a++)
        p[(size_t(a) * nh + h) * nv + v] -= m;
    }
}

// ---------------------------------------------------------------------------
// AML ring-artefact filter (Core/src/diamond.cpp:660-808; Applied
// Mathematics Letters 23, p1489).  For every detector row v and every term
// s of the angular series (1, sqrt2 sin(k pi a / na), sqrt2 cos(k pi a / na)
// for k < num_series): project the sinogram onto the term (FP64 sum over
// angles in order), form the regularised second difference of that profile
// along h, smooth it with the fixed matrix of the first series order
// (diamond.cpp:775-781 uses that one matrix for every term), and subtract
// the term back from every angle in float.  Series terms apply one after
// another to the updated sinogram.
extern "C" int rs_aml_ring_f32(float *p, int na, int nh, int nv, double param_n,
                               double param_r, int num_series) {
  if (param_n < -1e-10 || param_r < 1e-8 || num_series < 1 || num_series > 100)
    return 1;
  const int nx = nh;
  const int nterms = 2 * num_series - 1;
  // series table: term 0 is 1, terms 2k-1 / 2k are sqrt2 sin / sqrt2 cos
  std::vector<double> term(size_t(nterms) * na, 1.0);
  const double r2 = std::sqrt(2.0);
  for (int k = 1; k < num_series; k++) {
    const double slope = double(k) * M_PI / double(na);
    for (int a = 0; a < na; a++) {
      const double x = double(a) * slope;
      double sv = std::sin(x), cv = std::cos(x);
      sv *= r2;
      cv *= r2;
      term[size_t(2 * k - 1) * na + a] = sv;
      term[size_t(2 * k) * na + a] = cv;
    }
  }
  // smoothing matrix of order 1
  const double alpha = (param_n + param_r) * 1.0;
  const double mdiv = std::sqrt(alpha * (alpha + 4.0));
  const double tau = 2.0 * std::asinh(std::sqrt(alpha) / 2.0);
  std::vector<double> ex(size_t(2 * nx + 2));
  for (int i = 0; i < 2 * nx + 2; i++)
    ex[i] = std::exp(-tau * double(i));
  const double dv = mdiv * (1.0 - ex[2 * nx]);
  std::vector<double> mat(size_t(nx) * nx);
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < nx; j++) {
      const int lo = std::min(i, j) + 1, hi = std::max(i, j) + 1;
      double m = ex[hi - lo] * (1.0 + ex[2 * nx - 2 * hi + 1]) * (1.0 + ex[2 * lo - 1]);
      m /= dv;
      mat[size_t(i) * nx + j] = m;
    }
  std::vector<double> prof(nx), diff(nx);
  std::vector<float> corr(nx);
  for (int v = 0; v < nv; v++) {
    for (int t = 0; t < nterms; t++) {
      const double *w = term.data() + size_t(t) * na;
      const int order = (t + 2) / 2;
      for (int h = 0; h < nx; h++) {
        double acc = 0.0;
        for (int a = 0; a < na; a++)
          acc += double(p[(size_t(a) * nh + h) * nv + v]) * w[a];
        prof[h] = acc / double(na);
      }
      const double coef = param_n * double(order * order);
      for (int h = 0; h < nx; h++) {
        double d = coef * prof[h];
        if (h < nx - 1) {
          d += prof[h];
          d -= prof[h + 1];
        }
        if (h >= 1) {
          d += prof[h];
          d -= prof[h - 1];
        }
        diff[h] = d;
      }
      for (int i = 0; i < nx; i++) {
        double dp = 0.0;
        for (int h = 0; h < nx; h++)
          dp += diff[h] * mat[size_t(i) * nx + h];
        corr[i] = float(dp);
      }
      for (int a = 0; a < na; a++) {
        const float wf = float(w[a]);
        for (int h = 0; h < nx; h++)
          p[(size_t(a) * nh + h) * nv + v] -= wf * corr[h];
      }
    }
  }
  return 0;
}
