// AML ring-artefact filter for parallel-beam sinograms on the GPU
// (CCPi::remove_aml_ring_artefacts, Core/src/diamond.cpp:660-808, after
// Applied Mathematics Letters 23, p1489; exposed by the reference as
// parallelbeam.filters.aml_ring_artefacts, Wrappers/Python/src/
// diamond_wrapper.cpp:18-51).
//
// For every detector row v and every term t of the angular series (1, then
// sqrt2 sin and sqrt2 cos of k pi a / n_angles for k < num_series) the
// filter projects the sinogram onto the term (an FP64 sum over angles, in
// angle order), forms the regularised second difference of that profile
// along h, multiplies it by a fixed smoothing matrix (the reference uses the
// matrix of series order 1 for every term, diamond.cpp:775-781) and
// subtracts term x profile from every angle in float.  Terms apply one after
// another.
//
// The GPU does one sweep over the sinogram per term (subtract the previous
// term's correction and, in the same pass, sum the next term's projection)
// and one matrix-vector product per term for all rows at once.  Every FP64
// and float operation is the reference's, unfused and in its order (this
// file is compiled with --fmad=false), so the result is the reference's bit
// for bit.  The series table and the matrix depend only on the sizes and the
// two parameters; they are built on the host with the C library's sin, cos,
// exp, sqrt and asinh, as the reference builds them.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/ccpi_b200.h"
#include "engine.h"
#include "kernels.h"

namespace ccpi {
namespace {

constexpr int kAmlThreads = 256;

// One pass over the sinogram [a][h][v] for the (h, v) columns: first
// p -= float(w_prev[a]) * corr[h][v] (if w_prev), then
// res[h][v] = (sum_a double(p) * w_next[a]) / na (if w_next).
__global__ void __launch_bounds__(kAmlThreads)
    aml_sweep(float *__restrict__ px, int na, int nh, int nv, const double *__restrict__ w_prev,
              const float *__restrict__ corr, const double *__restrict__ w_next,
              double *__restrict__ res) {
  const i64 ncol = i64(nh) * nv;
  for (i64 c = blockIdx.x * i64(blockDim.x) + threadIdx.x; c < ncol;
       c += i64(gridDim.x) * blockDim.x) {
    const float cc = w_prev ? corr[c] : 0.0f;
    double acc = 0.0;
    float *col = px + c;
    for (int a = 0; a < na; a++) {
      float p = col[i64(a) * ncol];
      if (w_prev) {
        p = __fsub_rn(p, __fmul_rn(__double2float_rn(w_prev[a]), cc));
        col[i64(a) * ncol] = p;
      }
      if (w_next)
        acc = __dadd_rn(acc, __dmul_rn(double(p), w_next[a]));
    }
    if (w_next)
      res[c] = __ddiv_rn(acc, double(na));
  }
}

// corr[i][v] = float(sum_h d[h][v] * mat[i][h]) with the second difference
// d formed on the fly from the profile res (diamond.cpp:767-774):
// d[h] = coef res[h] (+ res[h] - res[h+1] if h < nh-1) (+ res[h] - res[h-1] if h > 0).
__global__ void __launch_bounds__(kAmlThreads)
    aml_smooth(const double *__restrict__ res, const double *__restrict__ mat, int nh, int nv,
               double coef, float *__restrict__ corr) {
  const i64 n = i64(nh) * nv;
  for (i64 t = blockIdx.x * i64(blockDim.x) + threadIdx.x; t < n;
       t += i64(gridDim.x) * blockDim.x) {
    const int i = int(t / nv), v = int(t - i64(i) * nv);
    const double *mrow = mat + i64(i) * nh;
    double prev = 0.0, cur = res[v];
    double dp = 0.0;
    for (int h = 0; h < nh; h++) {
      const double next = (h + 1 < nh) ? res[i64(h + 1) * nv + v] : 0.0;
      double d = __dmul_rn(coef, cur);
      if (h < nh - 1) {
        d = __dadd_rn(d, cur);
        d = __dsub_rn(d, next);
      }
      if (h >= 1) {
        d = __dadd_rn(d, cur);
        d = __dsub_rn(d, prev);
      }
      dp = __dadd_rn(dp, __dmul_rn(d, mrow[h]));
      prev = cur;
      cur = next;
    }
    corr[t] = __double2float_rn(dp);
  }
}

int grid_of(i64 n) {
  const i64 b = (n + kAmlThreads - 1) / kAmlThreads;
  return int(std::min<i64>(std::max<i64>(b, 1), 148 * 16));
}

} // namespace

int aml_ring_filter(float *d_sino, int na, int nh, int nv, double param_n, double param_r,
                    int num_series, cudaStream_t st) {
  if (!d_sino || na < 1 || nh < 2 || nv < 1) {
    set_error("aml ring filter: need a sinogram of >= 1 angle, >= 2 columns, >= 1 row");
    return 1;
  }
  if (param_n < -1e-10) {
    set_error("aml ring filter: param_n must be >= 0");
    return 1;
  }
  if (param_r < 1e-8) {
    set_error("aml ring filter: param_r must be > 0");
    return 1;
  }
  if (num_series < 1 || num_series > 100) {
    set_error("aml ring filter: num_series must be in [1, 100]");
    return 1;
  }
  const int nx = nh, nterms = 2 * num_series - 1;
  // series table (diamond.cpp:690-711)
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
  // smoothing matrix of series order 1 (diamond.cpp:712-746)
  const double alpha = (param_n + param_r) * 1.0;
  const double mdiv = std::sqrt(alpha * (alpha + 4.0));
  const double tau = 2.0 * std::asinh(std::sqrt(alpha) / 2.0);
  std::vector<double> ex(size_t(2 * nx + 2));
  for (int i = 0; i < 2 * nx + 2; i++)
    ex[i] = std::exp(-tau * double(i));
  const double dv = mdiv * (1.0 - ex[2 * nx]);
  std::vector<double> mat(size_t(nx) * nx);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < nx; j++) {
      const int lo = std::min(i, j) + 1, hi = std::max(i, j) + 1;
      double m = ex[hi - lo] * (1.0 + ex[2 * nx - 2 * hi + 1]) * (1.0 + ex[2 * lo - 1]);
      m /= dv;
      mat[size_t(i) * nx + j] = m;
    }
  const i64 ncol = i64(nh) * nv;
  double *d_term = nullptr, *d_mat = nullptr, *d_res = nullptr;
  float *d_corr = nullptr;
  int rc = 0;
  if (!cuda_ok(cudaMalloc(&d_term, term.size() * sizeof(double)), "aml: table") ||
      !cuda_ok(cudaMalloc(&d_mat, mat.size() * sizeof(double)), "aml: matrix") ||
      !cuda_ok(cudaMalloc(&d_res, size_t(ncol) * sizeof(double)), "aml: profile") ||
      !cuda_ok(cudaMalloc(&d_corr, size_t(ncol) * sizeof(float)), "aml: correction"))
    rc = 2;
  if (rc == 0 &&
      (!cuda_ok(cudaMemcpyAsync(d_term, term.data(), term.size() * sizeof(double),
                                cudaMemcpyHostToDevice, st),
                "aml: upload table") ||
       !cuda_ok(cudaMemcpyAsync(d_mat, mat.data(), mat.size() * sizeof(double),
                                cudaMemcpyHostToDevice, st),
                "aml: upload matrix")))
    rc = 2;
  for (int t = 0; rc == 0 && t < nterms; t++) {
    const double *w_prev = t > 0 ? d_term + size_t(t - 1) * na : nullptr;
    aml_sweep<<<grid_of(ncol), kAmlThreads, 0, st>>>(d_sino, na, nh, nv, w_prev, d_corr,
                                                     d_term + size_t(t) * na, d_res);
    const int order = (t + 2) / 2;
    const double coef = param_n * double(order * order);
    aml_smooth<<<grid_of(ncol), kAmlThreads, 0, st>>>(d_res, d_mat, nh, nv, coef, d_corr);
  }
  if (rc == 0)
    aml_sweep<<<grid_of(ncol), kAmlThreads, 0, st>>>(
        d_sino, na, nh, nv, d_term + size_t(nterms - 1) * na, d_corr, nullptr, nullptr);
  if (rc == 0 && !cuda_ok(cudaStreamSynchronize(st), "aml ring filter"))
    rc = 2;
  cudaFree(d_term);
  cudaFree(d_mat);
  cudaFree(d_res);
  cudaFree(d_corr);
  return rc;
}

} // namespace ccpi
