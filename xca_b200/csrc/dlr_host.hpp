// Host-side construction of the DLR basis (the third-party cppdlr's build_dlr_rf / imtime_ops, whose
// published algorithm is restated here; TRIQS/xca call sites hyb.cpp:158-159,
// block_sparse_backbone.cpp:68-70, python/triqs_xca/block_sparse_solver.py:134).
//
// Set-up code: it runs once per (Lambda, eps) on the host, as in the reference.
//  1. composite Chebyshev fine grids: t in [0, 1/2] with npt = max(ceil(log2 Lambda) - 2, 1) dyadic
//     panels refined toward 0 (p = 24 first-kind Chebyshev nodes per panel), mirrored to (1/2, 1] in
//     relative format; omega in [-Lambda, Lambda] with npo = max(ceil(log2 Lambda), 1) dyadic panels
//     per sign refined toward 0;
//  2. pivoted, twice-orthogonalised Gram-Schmidt on the frequency columns of K(t, omega) selects the
//     real frequencies, stopping when the largest residual column has RMS entry below eps (this gives
//     the rank r = 36 at Lambda = 200, eps = 1e-10 that test_block_sparse_backbone_eval.cpp:47-50 pins);
//  3. the same procedure, to full rank, on the rows of K(t_fine, omega_dlr) selects the time nodes.
#pragma once
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <vector>

namespace xca {

// cppdlr's signed fermionic kernel in relative time format:
// K(t, om) = -exp(-t om) / (1 + exp(-om)) (om >= 0), -exp((1 - t) om) / (1 + exp(om)) (om < 0).
inline double k_it(double t, double om) {
  if (t < 0) { t = -t; om = -om; }
  if (om >= 0) return -std::exp(-t * om) / (1.0 + std::exp(-om));
  return -std::exp((1.0 - t) * om) / (1.0 + std::exp(om));
}
inline double k_abs(double t, double om) {
  if (om >= 0) return -std::exp(-t * om) / (1.0 + std::exp(-om));
  return -std::exp((1.0 - t) * om) / (1.0 + std::exp(om));
}

inline void dlr_fine_grids(double lam, std::vector<double> &t, std::vector<double> &om, int p = 24) {
  int nl = (int)std::ceil(std::log(lam) / std::log(2.0));
  int npo = std::max(nl, 1), npt = std::max(nl - 2, 1);
  std::vector<double> xc(p);
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < p; ++j) xc[j] = -std::cos(pi * (j + 0.5) / p);
  std::vector<double> half;
  for (int i = 0; i < npt; ++i) {
    double a = (i == 0) ? 0.0 : std::ldexp(1.0, -(npt - i + 1));
    double b = std::ldexp(1.0, -(npt - i));
    for (int j = 0; j < p; ++j) half.push_back(a + (b - a) * (xc[j] + 1) / 2);
  }
  t = half;
  for (int j = (int)half.size() - 1; j >= 0; --j) t.push_back(-half[j]);
  std::vector<double> pos;
  for (int i = 0; i < npo; ++i) {
    double a = (i == 0) ? 0.0 : lam * std::ldexp(1.0, -(npo - i));
    double b = lam * std::ldexp(1.0, -(npo - i - 1));
    for (int j = 0; j < p; ++j) pos.push_back(a + (b - a) * (xc[j] + 1) / 2);
  }
  om.clear();
  for (int j = (int)pos.size() - 1; j >= 0; --j) om.push_back(-pos[j]);
  for (double x : pos) om.push_back(x);
}

// Pivoted twice-orthogonalised Gram-Schmidt on the rows of a (m x n, row-major).
inline std::vector<int> pivoted_gs(std::vector<double> a, int m, int n, double eps_rms) {
  std::vector<double> norms(m);
  std::vector<int> piv(m);
  for (int i = 0; i < m; ++i) {
    piv[i] = i;
    double s = 0;
    for (int j = 0; j < n; ++j) s += a[(size_t)i * n + j] * a[(size_t)i * n + j];
    norms[i] = s;
  }
  double thresh = eps_rms * eps_rms * n;
  int kmax = std::min(m, n);
  for (int j = 0; j < kmax; ++j) {
    int k = j;
    for (int i = j + 1; i < m; ++i)
      if (norms[i] > norms[k]) k = i;
    if (norms[k] <= thresh || norms[k] == 0.0) return std::vector<int>(piv.begin(), piv.begin() + j);
    if (k != j) {
      for (int c = 0; c < n; ++c) std::swap(a[(size_t)j * n + c], a[(size_t)k * n + c]);
      std::swap(norms[j], norms[k]);
      std::swap(piv[j], piv[k]);
    }
    double nr = 0;
    for (int c = 0; c < n; ++c) nr += a[(size_t)j * n + c] * a[(size_t)j * n + c];
    nr = std::sqrt(nr);
    for (int c = 0; c < n; ++c) a[(size_t)j * n + c] /= nr;
    for (int pass = 0; pass < 2; ++pass)
      for (int i = j + 1; i < m; ++i) {
        double d = 0;
        for (int c = 0; c < n; ++c) d += a[(size_t)i * n + c] * a[(size_t)j * n + c];
        for (int c = 0; c < n; ++c) a[(size_t)i * n + c] -= d * a[(size_t)j * n + c];
      }
    for (int i = j + 1; i < m; ++i) {
      double s = 0;
      for (int c = 0; c < n; ++c) s += a[(size_t)i * n + c] * a[(size_t)i * n + c];
      norms[i] = s;
    }
  }
  return std::vector<int>(piv.begin(), piv.begin() + kmax);
}

inline std::vector<double> build_dlr_rf(double lam, double eps) {
  std::vector<double> t, om;
  dlr_fine_grids(lam, t, om);
  int nt = (int)t.size(), no = (int)om.size();
  std::vector<double> kt((size_t)no * nt);  // rows = frequencies
  for (int j = 0; j < no; ++j)
    for (int i = 0; i < nt; ++i) kt[(size_t)j * nt + i] = k_it(t[i], om[j]);
  auto piv = pivoted_gs(kt, no, nt, eps);
  std::vector<double> rf;
  for (int k : piv) rf.push_back(om[k]);
  std::sort(rf.begin(), rf.end());
  return rf;
}

inline std::vector<double> build_dlr_it(double lam, const std::vector<double> &rf) {
  std::vector<double> t, om;
  dlr_fine_grids(lam, t, om);
  int nt = (int)t.size(), r = (int)rf.size();
  std::vector<double> k((size_t)nt * r);
  for (int i = 0; i < nt; ++i)
    for (int l = 0; l < r; ++l) k[(size_t)i * r + l] = k_it(t[i], rf[l]);
  auto piv = pivoted_gs(k, nt, r, 0.0);
  if ((int)piv.size() != r) throw std::runtime_error("DLR time-node selection lost rank");
  std::sort(piv.begin(), piv.end());
  std::vector<double> it;
  for (int i : piv) it.push_back(t[i]);
  return it;
}

// LU with partial pivoting (LAPACK getrf: piv[k] is the row swapped with k at step k).
inline void lu_factor(std::vector<double> &a, int n, std::vector<int> &piv) {
  piv.resize(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(a[(size_t)k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(a[(size_t)i * n + k]) > best) { best = std::fabs(a[(size_t)i * n + k]); p = i; }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
    double d = a[(size_t)k * n + k];
    if (d == 0.0) throw std::runtime_error("singular DLR matrix");
    for (int i = k + 1; i < n; ++i) {
      double f = a[(size_t)i * n + k] / d;
      a[(size_t)i * n + k] = f;
      if (f == 0.0) continue;
      for (int j = k + 1; j < n; ++j) a[(size_t)i * n + j] -= f * a[(size_t)k * n + j];
    }
  }
}

// Reciprocals 1 / U_kk of the upper factor's diagonal (each one correctly rounded division).
inline std::vector<double> lu_diag_reciprocals(const std::vector<double> &lu, int n) {
  std::vector<double> d(n);
  for (int k = 0; k < n; ++k) d[k] = 1.0 / lu[(size_t)k * n + k];
  return d;
}

// Solve A X = B in place (B is n x nrhs, row-major) with the factors of lu_factor, in the column order of
// the reference BLAS dtrsm that LAPACK getrs calls: row interchanges; forward, for k ascending,
// b_i -= L_ik b_k (i > k); backward, for k descending, b_k *= 1 / U_kk (the diagonal's precomputed
// reciprocal, as BLAS triangular solves with an inverted packed diagonal do), then b_i -= U_ik b_k
// (i < k); every update one fused multiply-add.  The operation order of the device's DLR transforms.
inline void lu_solve_recip(const std::vector<double> &lu, const std::vector<double> &dinv, int n, const std::vector<int> &piv, double *b,
                           long nrhs) {
  for (int k = 0; k < n; ++k)
    if (piv[k] != k)
      for (long j = 0; j < nrhs; ++j) std::swap(b[(size_t)k * nrhs + j], b[(size_t)piv[k] * nrhs + j]);
  for (int k = 0; k < n; ++k)
    for (int i = k + 1; i < n; ++i) {
      double f = lu[(size_t)i * n + k];
      for (long j = 0; j < nrhs; ++j) b[(size_t)i * nrhs + j] = std::fma(-f, b[(size_t)k * nrhs + j], b[(size_t)i * nrhs + j]);
    }
  for (int k = n - 1; k >= 0; --k) {
    for (long j = 0; j < nrhs; ++j) b[(size_t)k * nrhs + j] *= dinv[k];
    for (int i = 0; i < k; ++i) {
      double f = lu[(size_t)i * n + k];
      for (long j = 0; j < nrhs; ++j) b[(size_t)i * nrhs + j] = std::fma(-f, b[(size_t)k * nrhs + j], b[(size_t)i * nrhs + j]);
    }
  }
}

}  // namespace xca
