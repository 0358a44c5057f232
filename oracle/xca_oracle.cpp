// Oracle (test infrastructure only): a CPU FP64 restatement of the TRIQS/xca pseudo-particle
// hot path.  Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py load it,
// always as the checker; the product never calls it.
//
// Arithmetic is complex<double> throughout, as in the reference (dcomplex everywhere,
// c++/triqs_xca/block_sparse.hpp:24).  Each routine names the reference lines it restates.
// The DLR operations restate the published algorithms of the third-party library cppdlr
// (TRIQS 4.0.x; not present here): vals2coefs is an LU solve against K(t_i, om_l); the
// time-ordered and full fermionic convolutions use the closed forms
//   int_0^t K(t-s,om_k) K(s,om_l) ds = [K(0,om_k) K(t,om_l) - K(0,om_l) K(t,om_k)] / (om_k - om_l)
//   (k != l), and t K(0,om_k) K(t,om_k) (k == l),
// and the Matsubara-space product rule for the full convolution.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using cd = std::complex<double>;

namespace {

// Fused multiply-adds of the restated arithmetic: every a * b + c below is one correctly rounded
// operation per real component, the operation model the device path reproduces bit for bit.
inline cd cfma(const cd &a, const cd &b, const cd &c) {
  return {std::fma(a.real(), b.real(), std::fma(-a.imag(), b.imag(), c.real())),
          std::fma(a.real(), b.imag(), std::fma(a.imag(), b.real(), c.imag()))};
}
inline cd dfma(double a, const cd &b, const cd &c) { return {std::fma(a, b.real(), c.real()), std::fma(a, b.imag(), c.imag())}; }
inline double dfma(double a, double b, double c) { return std::fma(a, b, c); }
inline cd dfma(const cd &a, const cd &b, const cd &c) { return cfma(a, b, c); }

// ---------------------------------------------------------------- kernel and DLR basis
// cppdlr::k_it (call sites hyb.cpp:98-103).  cppdlr's kernel carries the Green's-function sign,
// K(t, om) = -exp(-t om) / (1 + exp(-om)) (om >= 0), -exp((1 - t) om) / (1 + exp(om)) (om < 0): the
// analytic expectations of test_block_sparse_backbone_eval.cpp:142-268 hold only with this sign
// (the positive-kernel helper of test/python/pycppdlr.py:29-43 builds G = -kernel).
double k_it(double t, double om) {
  if (t < 0) { t = -t; om = -om; }  // relative format: t < 0 stands for 1 + t, K(1-s, om) = K(s, -om)
  if (om >= 0) return -std::exp(-t * om) / (1.0 + std::exp(-om));
  return -std::exp((1.0 - t) * om) / (1.0 + std::exp(om));
}
double k_abs(double t, double om) {  // absolute t in [0, 1]
  if (om >= 0) return -std::exp(-t * om) / (1.0 + std::exp(-om));
  return -std::exp((1.0 - t) * om) / (1.0 + std::exp(om));
}

// LU with partial pivoting (LAPACK getrf semantics) and the matching solve (getrs).
template <class T>
void lu_factor(std::vector<T> &a, int n, std::vector<int> &piv) {
  piv.resize(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::abs(a[(size_t)k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      double v = std::abs(a[(size_t)i * n + k]);
      if (v > best) { best = v; p = i; }
    }
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[(size_t)k * n + j], a[(size_t)p * n + j]);
    T d = a[(size_t)k * n + k];
    if (d == T(0)) throw std::runtime_error("singular matrix in LU");
    for (int i = k + 1; i < n; ++i) {
      T f = a[(size_t)i * n + k] / d;
      a[(size_t)i * n + k] = f;
      if (f == T(0)) continue;
      T *ri = &a[(size_t)i * n];
      const T *rk = &a[(size_t)k * n];
      for (int j = k + 1; j < n; ++j) ri[j] -= f * rk[j];
    }
  }
}
// Solve A X = B in place, B is n x nrhs row-major, with the LU factors of lu_factor.  The
// substitutions run in the column order of the reference BLAS dtrsm that LAPACK getrs calls: forward,
// for k ascending, b_i -= L_ik b_k (i > k); backward, for k descending, b_k /= U_kk then
// b_i -= U_ik b_k (i < k), each update one fused multiply-add.
template <class T, class U>
void lu_solve(const std::vector<T> &lu, int n, const std::vector<int> &piv, U *b, long nrhs) {
  for (int k = 0; k < n; ++k)
    if (piv[k] != k)
      for (long j = 0; j < nrhs; ++j) std::swap(b[(size_t)k * nrhs + j], b[(size_t)piv[k] * nrhs + j]);
  for (int k = 0; k < n; ++k)
    for (int i = k + 1; i < n; ++i) {
      T f = lu[(size_t)i * n + k];
      for (long j = 0; j < nrhs; ++j) b[(size_t)i * nrhs + j] = dfma(-f, b[(size_t)k * nrhs + j], b[(size_t)i * nrhs + j]);
    }
  for (int k = n - 1; k >= 0; --k) {
    T d = lu[(size_t)k * n + k];
    for (long j = 0; j < nrhs; ++j) b[(size_t)k * nrhs + j] /= d;
    for (int i = 0; i < k; ++i) {
      T f = lu[(size_t)i * n + k];
      for (long j = 0; j < nrhs; ++j) b[(size_t)i * nrhs + j] = dfma(-f, b[(size_t)k * nrhs + j], b[(size_t)i * nrhs + j]);
    }
  }
}

struct Dlr {
  int r;
  std::vector<double> rf, it, tabs, k0, k1;  // k0 = K(0, om_l), k1 = K(1, om_l) (signed kernel)
  std::vector<double> cf2it;                 // r x r : K(t_i, om_l)
  std::vector<double> lu;                    // LU of cf2it
  std::vector<int> piv;
  std::vector<double> dinv;                  // 1 / U_kk of the LU factors
  std::vector<double> refl;                  // r x r : K(t_i, -om_l)  (values of g(beta - tau))
  Dlr(int r_, const double *rf_, const double *it_) : r(r_), rf(rf_, rf_ + r_), it(it_, it_ + r_) {
    tabs.resize(r); k0.resize(r); k1.resize(r);
    cf2it.resize((size_t)r * r); refl.resize((size_t)r * r);
    for (int i = 0; i < r; ++i) tabs[i] = it[i] < 0 ? 1.0 + it[i] : it[i];
    for (int l = 0; l < r; ++l) { k0[l] = k_abs(0.0, rf[l]); k1[l] = k_abs(1.0, rf[l]); }
    for (int i = 0; i < r; ++i)
      for (int l = 0; l < r; ++l) {
        cf2it[(size_t)i * r + l] = k_it(it[i], rf[l]);
        refl[(size_t)i * r + l] = k_it(it[i], -rf[l]);
      }
    lu = cf2it;
    lu_factor(lu, r, piv);
    dinv.resize(r);
    for (int k = 0; k < r; ++k) dinv[k] = 1.0 / lu[(size_t)k * r + k];
  }
  // cppdlr imtime_ops::vals2coefs: coefficients c with sum_l K(t_i, om_l) c_l = g(t_i).
  // The substitution applies the upper factor's diagonal through its reciprocals (b_k <- b_k * (1 / U_kk)),
  // as BLAS triangular solves with an inverted packed diagonal do.
  void vals2coefs(const cd *vals, long ncol, cd *coefs) const {
    std::copy(vals, vals + (size_t)r * ncol, coefs);
    for (int k = 0; k < r; ++k)
      if (piv[k] != k)
        for (long j = 0; j < ncol; ++j) std::swap(coefs[(size_t)k * ncol + j], coefs[(size_t)piv[k] * ncol + j]);
    for (int k = 0; k < r; ++k)
      for (int i = k + 1; i < r; ++i) {
        double f = lu[(size_t)i * r + k];
        for (long j = 0; j < ncol; ++j) coefs[(size_t)i * ncol + j] = dfma(-f, coefs[(size_t)k * ncol + j], coefs[(size_t)i * ncol + j]);
      }
    for (int k = r - 1; k >= 0; --k) {
      for (long j = 0; j < ncol; ++j) coefs[(size_t)k * ncol + j] *= dinv[k];
      for (int i = 0; i < k; ++i) {
        double f = lu[(size_t)i * r + k];
        for (long j = 0; j < ncol; ++j) coefs[(size_t)i * ncol + j] = dfma(-f, coefs[(size_t)k * ncol + j], coefs[(size_t)i * ncol + j]);
      }
    }
  }
  void coefs2vals(const cd *coefs, long ncol, cd *vals) const {
    for (int i = 0; i < r; ++i)
      for (long j = 0; j < ncol; ++j) {
        cd s = 0;
        for (int l = 0; l < r; ++l) s += cf2it[(size_t)i * r + l] * coefs[(size_t)l * ncol + j];
        vals[(size_t)i * ncol + j] = s;
      }
  }
  // cppdlr imtime_ops::reflect: values of g(beta - tau) at the nodes (hyb.cpp:84, bsb.cpp:648).
  void reflect(const cd *vals, long ncol, cd *out) const {
    std::vector<cd> c((size_t)r * ncol);
    vals2coefs(vals, ncol, c.data());
    for (int i = 0; i < r; ++i)
      for (long j = 0; j < ncol; ++j) {
        cd s = 0;
        for (int l = 0; l < r; ++l) s = dfma(refl[(size_t)i * r + l], c[(size_t)l * ncol + j], s);
        out[(size_t)i * ncol + j] = s;
      }
  }
  // cppdlr imtime_ops::coefs2eval at relative time t.
  void coefs2eval(const cd *coefs, long ncol, double t, cd *out) const {
    for (long j = 0; j < ncol; ++j) out[j] = 0;
    for (int l = 0; l < r; ++l) {
      double k = k_it(t, rf[l]);
      for (long j = 0; j < ncol; ++j) out[j] += k * coefs[(size_t)l * ncol + j];
    }
  }
  // cppdlr imtime_ops::convolve(beta, fc, gc, time_order) for matrix-valued expansions:
  // fc (r, a, b), gc (r, b, c) -> values h (r, a, c) of int f(tau - tau') g(tau') dtau'.
  void convolve(double beta, int a, int b, int c, const cd *fc, const cd *gc, bool time_order, cd *h) const {
    std::vector<cd> ft((size_t)r * a * b, 0.0), gt((size_t)r * b * c, 0.0);
    for (int l = 0; l < r; ++l)
      for (int k = 0; k < r; ++k) {
        if (k == l) continue;
        double w = (time_order ? k0[k] : 1.0) / (rf[k] - rf[l]);
        for (int x = 0; x < a * b; ++x) ft[(size_t)l * a * b + x] = dfma(w, fc[(size_t)k * a * b + x], ft[(size_t)l * a * b + x]);
        for (int x = 0; x < b * c; ++x) gt[(size_t)l * b * c + x] = dfma(w, gc[(size_t)k * b * c + x], gt[(size_t)l * b * c + x]);
      }
    for (int i = 0; i < r; ++i)
      for (int x = 0; x < a * c; ++x) h[(size_t)i * a * c + x] = 0;
    std::vector<cd> Q((size_t)r * a * c, 0.0), P((size_t)r * a * c, 0.0);
    for (int l = 0; l < r; ++l) {
      const cd *f = fc + (size_t)l * a * b, *g = gc + (size_t)l * b * c;
      const cd *fh = ft.data() + (size_t)l * a * b, *gh = gt.data() + (size_t)l * b * c;
      for (int x = 0; x < a; ++x)
        for (int z = 0; z < c; ++z) {
          cd sq = 0, sp = 0;
          for (int y = 0; y < b; ++y) {
            sq = cfma(fh[x * b + y], g[y * c + z], cfma(f[x * b + y], gh[y * c + z], sq));
            sp = cfma(f[x * b + y], g[y * c + z], sp);
          }
          Q[(size_t)l * a * c + x * c + z] = sq;
          P[(size_t)l * a * c + x * c + z] = sp;
        }
    }
    if (time_order) {
      // h(t_i) = h1_i + t_i h2_i with h1_i = sum_l (beta K_il) Q_l and h2_i = sum_l (beta K_il) (K_l(0) P_l),
      // each sum from zero in ascending l: beta sum_l K_l(t_i) [Q_l + t_i K_l(0) P_l] for the signed kernel.
      for (int i = 0; i < r; ++i)
        for (int x = 0; x < a * c; ++x) {
          cd h1 = 0, h2 = 0;
          for (int l = 0; l < r; ++l) {
            double bk = beta * cf2it[(size_t)i * r + l];
            h1 = dfma(bk, Q[(size_t)l * a * c + x], h1);
            h2 = dfma(bk, k0[l] * P[(size_t)l * a * c + x], h2);
          }
          h[(size_t)i * a * c + x] = dfma(tabs[i], h2, h1);
        }
    } else {
      // full (fermionic) convolution: h = -beta sum_l K_l(t)[Q_l + (t + K_l(1)) P_l] (weights 1 / (om_k - om_l))
      for (int l = 0; l < r; ++l)
        for (int i = 0; i < r; ++i) {
          double kil = cf2it[(size_t)i * r + l];
          double wd = tabs[i] + k1[l];
          cd *hi = h + (size_t)i * a * c;
          for (int x = 0; x < a * c; ++x) hi[x] += -beta * kil * (Q[(size_t)l * a * c + x] + wd * P[(size_t)l * a * c + x]);
        }
    }
  }
  // cppdlr imtime_ops::convmat_inplace(M, beta, Fermion, fc, time_order) (dlr_dyson_ppsc.hpp:149):
  // M[(i, x), (i', y)] with h(t_i)[x, :] = sum_{i', y} M[(i,x),(i',y)] g(t_i')[y, :] for h = f * g.
  void convmat(double beta, int n, const cd *fc, bool time_order, cd *M) const {
    size_t nn = (size_t)n * n;
    std::vector<cd> ft((size_t)r * nn, 0.0);
    for (int l = 0; l < r; ++l)
      for (int k = 0; k < r; ++k) {
        if (k == l) continue;
        double w = (time_order ? k0[k] : 1.0) / (rf[k] - rf[l]);
        for (size_t x = 0; x < nn; ++x) ft[l * nn + x] += w * fc[k * nn + x];
      }
    // A[i][k] (n x n) = +-beta [K(t_i,om_k) (ft_k + wd_ik f_k) + sum_{l != k} K(t_i,om_l) w_lk f_l]
    std::vector<cd> A((size_t)r * r * nn, 0.0);
    for (int i = 0; i < r; ++i)
      for (int k = 0; k < r; ++k) {
        cd *Aik = &A[((size_t)i * r + k) * nn];
        double kik = cf2it[(size_t)i * r + k];
        double wd = time_order ? tabs[i] * k0[k] : tabs[i] + k1[k];
        double sg = time_order ? beta : -beta;
        for (size_t x = 0; x < nn; ++x) Aik[x] = sg * kik * (ft[k * nn + x] + wd * fc[k * nn + x]);
        for (int l = 0; l < r; ++l) {
          if (l == k) continue;
          double w = sg * cf2it[(size_t)i * r + l] * (time_order ? k0[k] : 1.0) / (rf[k] - rf[l]);
          for (size_t x = 0; x < nn; ++x) Aik[x] += w * fc[l * nn + x];
        }
      }
    // M[(i,x),(i',y)] = sum_k A[i][k][x][y] it2cf[k][i'] with it2cf = K^{-1}: every row vector
    // a_k = A[i][k][x][y] is right-multiplied by K^{-1} through the LU factors (K^T z = a, the transposed
    // getrs that cppdlr's vals2coefs(g, transpose = true) performs), never through an explicit inverse.
    long N = (long)r * n;
    std::vector<cd> rhs((size_t)r * N * n);  // rows k, columns (i, x, y)
    for (int i = 0; i < r; ++i)
      for (int k = 0; k < r; ++k)
        for (size_t xy = 0; xy < nn; ++xy) rhs[(size_t)k * r * nn + (size_t)i * nn + xy] = A[((size_t)i * r + k) * nn + xy];
    solve_transposed(rhs.data(), (long)r * nn);
    for (int i = 0; i < r; ++i)
      for (int ip = 0; ip < r; ++ip)
        for (int x = 0; x < n; ++x)
          for (int y = 0; y < n; ++y) M[((size_t)i * n + x) * N + (size_t)ip * n + y] = rhs[(size_t)ip * r * nn + (size_t)i * nn + x * n + y];
  }
  // Solve K^T Z = B in place (B is r x ncol): K = P L U, so K^T = U^T L^T P^T.
  void solve_transposed(cd *b, long ncol) const {
    for (int i = 0; i < r; ++i) {  // U^T y = b (forward, U^T lower)
      for (int k = 0; k < i; ++k) {
        double f = lu[(size_t)k * r + i];
        if (f == 0.0) continue;
        for (long j = 0; j < ncol; ++j) b[(size_t)i * ncol + j] -= f * b[(size_t)k * ncol + j];
      }
      double d = lu[(size_t)i * r + i];
      for (long j = 0; j < ncol; ++j) b[(size_t)i * ncol + j] /= d;
    }
    for (int i = r - 1; i >= 0; --i)  // L^T w = y (backward, unit diagonal)
      for (int k = i + 1; k < r; ++k) {
        double f = lu[(size_t)k * r + i];
        if (f == 0.0) continue;
        for (long j = 0; j < ncol; ++j) b[(size_t)i * ncol + j] -= f * b[(size_t)k * ncol + j];
      }
    for (int k = r - 1; k >= 0; --k)  // undo the row interchanges in reverse order
      if (piv[k] != k)
        for (long j = 0; j < ncol; ++j) std::swap(b[(size_t)k * ncol + j], b[(size_t)piv[k] * ncol + j]);
  }
};

// ---------------------------------------------------------------- backbone (backbone.cpp)
struct Backbone {
  int m, n, p;
  std::vector<int> topo;  // m x 2
  bool correlator;
  std::vector<int> fb, pole_inds, orb_inds, edges /*(2m-1) x (m-1)*/, pf_ksign, pf_kexp;
  std::vector<int> v_bar, v_dag, v_hyb, v_ksign, v_orb;
  int prefactor_sign;
  long fb_ix_max, o_ix_max, p_ix_max;
  Backbone(int m_, const int *t, int n_, int p_, bool corr) : m(m_), n(n_), p(p_), topo(t, t + 2 * m_), correlator(corr) {
    // Backbone ctor backbone.cpp:19-33; CorrelatorBackbone ctor :239
    fb_ix_max = 1L << (corr ? m - 1 : m);
    o_ix_max = 1;
    for (int i = 0; i < m - 1; ++i) o_ix_max *= n;
    p_ix_max = 1;
    for (int i = 0; i < m - 1; ++i) p_ix_max *= p;
    for (int i = 0; i < m; ++i)
      if (topo[2 * i] >= topo[2 * i + 1]) throw std::invalid_argument("first row of topology must contain smaller-numbered vertices");
    if (topo[0] != 0) throw std::invalid_argument("topology(0,0) must be 0");
  }
  int t(int i, int j) const { return topo[2 * i + j]; }
  long num_backbones() const { return fb_ix_max * o_ix_max * p_ix_max; }
  // set_flat_index backbone.cpp:192-208 (CorrelatorBackbone :276-292)
  void set_flat_index(long f_ix, const std::vector<double> &poles_beta) {
    long o_ix = f_ix % o_ix_max;
    f_ix /= o_ix_max;
    long p_ix = f_ix % p_ix_max;
    long fb_ix = f_ix / p_ix_max;
    int nv = 2 * m;
    v_bar.assign(nv, 0); v_dag.assign(nv, 0); v_hyb.assign(nv, 0); v_ksign.assign(nv, 0); v_orb.assign(nv, 0);
    edges.assign((size_t)(2 * m - 1) * std::max(m - 1, 0), 0);
    pf_ksign.assign(std::max(m - 1, 0), 0);
    pf_kexp.assign(std::max(m - 1, 0), 0);
    prefactor_sign = 1;
    fb.assign(m, 0);
    // set_directions backbone.cpp:35-76 / CorrelatorBackbone :241-274
    if (!correlator) {
      for (int i = 0; i < m; ++i) { fb[i] = fb_ix % 2; fb_ix /= 2; }
      v_bar[0] = 0; v_bar[t(0, 1)] = 0;
      if (fb[0] == 1) { v_dag[0] = 0; v_dag[t(0, 1)] = 1; }
      else { v_dag[0] = 1; v_dag[t(0, 1)] = 0; }
    } else {
      fb[0] = -1;
      for (int i = 1; i < m; ++i) { fb[i] = fb_ix % 2; fb_ix /= 2; }
      v_bar[t(0, 0)] = 0; v_bar[t(0, 1)] = 0;
      v_dag[t(0, 0)] = 1; v_dag[t(0, 1)] = 0;
    }
    for (int i = 1; i < m; ++i) {
      v_bar[t(i, 0)] = 0; v_bar[t(i, 1)] = 1;
      if (fb[i] == 1) { v_dag[t(i, 0)] = 0; v_dag[t(i, 1)] = 1; }
      else { v_dag[t(i, 0)] = 1; v_dag[t(i, 1)] = 0; }
    }
    // set_pole_inds backbone.cpp:86-150
    pole_inds.assign(std::max(m - 1, 0), 0);
    for (int i = 0; i < m - 1; ++i) { pole_inds[i] = (int)(p_ix % p); p_ix /= p; }
    for (int i = 1; i < m; ++i) {
      double w = poles_beta[pole_inds[i - 1]];
      int a = t(i, 0), b = t(i, 1);
      if (fb[i] == 1) {
        if (w <= 0) {  // step 4(a)
          v_hyb[a] = i - 1; v_ksign[a] = -1;
          v_hyb[b] = i - 1; v_ksign[b] = 1;
          pf_ksign[i - 1] = -1; pf_kexp[i - 1] = 1;
        } else {       // step 4(b)
          v_hyb[b] = i - 1;
          for (int j = a; j < b; ++j) edges[(size_t)j * (m - 1) + i - 1] = 1;
          pf_ksign[i - 1] = 1; pf_kexp[i - 1] = b - a - 1;
        }
      } else {
        if (w >= 0) {  // step 4(a)
          v_hyb[a] = i - 1; v_ksign[a] = 1;
          v_hyb[b] = i - 1; v_ksign[b] = -1;
          prefactor_sign *= -1;
          pf_ksign[i - 1] = 1; pf_kexp[i - 1] = 1;
        } else {       // step 4(b)
          v_hyb[b] = i - 1;
          for (int j = a; j < b; ++j) edges[(size_t)j * (m - 1) + i - 1] = -1;
          prefactor_sign *= -1;
          pf_ksign[i - 1] = -1; pf_kexp[i - 1] = b - a - 1;
        }
      }
    }
    // set_orb_inds backbone.cpp:165-186
    orb_inds.assign(nv, 0);
    orb_inds[0] = -1; orb_inds[t(0, 1)] = -1;
    for (int i = 1; i < m; ++i) {
      orb_inds[t(i, 0)] = (int)(o_ix % n);
      orb_inds[t(i, 1)] = (int)(o_ix % n);
      o_ix /= n;
    }
    for (int i = 0; i < nv; ++i)
      if (i != 0 && i != t(0, 1)) v_orb[i] = orb_inds[i];
  }
  int edge(int e, int x) const { return edges[(size_t)e * (m - 1) + x]; }
};

// ---------------------------------------------------------------- block-sparse operators
// BlockOpSymSet / BlockOpSymSetBar (block_sparse.hpp:181-243); F blocks (q, rows, cols).
struct SymSet {
  int q = 0;
  std::vector<int> index;              // per block column: target block or -1
  std::vector<std::vector<cd>> blocks; // per block column
};
struct SymSetBar {
  int q = 0, p = 0;
  std::vector<int> index;
  std::vector<std::vector<cd>> blocks; // (q, p, rows, cols)
};

struct Evaluator {
  const Dlr *dlr;
  int r, n, p, nb, nq;
  double beta;
  std::vector<int> dims;
  std::vector<long> labels, sinds, ssizes;
  std::vector<long> set_to_orb;  // nq x n
  std::vector<SymSet> Fs, Fd;
  std::vector<SymSetBar> Fdbar, Fbarr;
  // Hybridization (hyb.cpp:15-44)
  std::vector<double> poles_beta, kitp, kitm /* r x p */, k0p, k0m;
  std::vector<cd> coeffs, values, values_refl; // (p|r, n, n)
  int Nmax;

  int rows(const SymSet &S, int b) const { return dims[S.index[b]]; }
};

void check_sym_set_block_diagonal(const cd *c, int p, const std::vector<long> &labels, const char *who) {
  // block_sparse.cpp:443-492
  long n = (long)labels.size();
  double mx = 0;
  for (long z = 0; z < (long)p * n * n; ++z) mx = std::max(mx, std::abs(c[z]));
  if (!std::isfinite(mx)) throw std::invalid_argument(std::string(who) + ": hyb_coeffs contains a non-finite entry");
  double thresh = 1.0e-12 * mx;
  for (int l = 0; l < p; ++l)
    for (long i = 0; i < n; ++i)
      for (long j = 0; j < n; ++j)
        if (labels[i] != labels[j] && std::abs(c[((size_t)l * n + i) * n + j]) > thresh)
          throw std::invalid_argument(std::string(who) + ": hyb_coeffs couples different symmetry sets");
}

// ---------------------------------------------------------------- small dense helpers
// out (r, R, C) = F (R x K) * in (r, K, C) for each node
void left_mul(int r, const cd *F, int R, int K, const cd *in, int C, cd *out) {
  for (int t = 0; t < r; ++t) {
    const cd *a = in + (size_t)t * K * C;
    cd *o = out + (size_t)t * R * C;
    for (int i = 0; i < R; ++i)
      for (int j = 0; j < C; ++j) {
        cd s = 0;
        for (int k = 0; k < K; ++k) s = cfma(F[i * K + k], a[k * C + j], s);
        o[i * C + j] = s;
      }
  }
}
// out (r, R, C) = in (r, R, K) * F (K x C)
void right_mul(int r, const cd *in, int R, int K, const cd *F, int C, cd *out) {
  for (int t = 0; t < r; ++t) {
    const cd *a = in + (size_t)t * R * K;
    cd *o = out + (size_t)t * R * C;
    for (int i = 0; i < R; ++i)
      for (int j = 0; j < C; ++j) {
        cd s = 0;
        for (int k = 0; k < K; ++k) s = cfma(a[i * K + k], F[k * C + j], s);
        o[i * C + j] = s;
      }
  }
}

struct Work {
  std::vector<cd> T, T2, GK, fc, gc, tk, tm, U, U2;
  int ind_path[16], block_dims[17];
  double flops = 0;
  long items = 0;
};

struct BlockG {  // BlockDiagOpFun(block_gf) block_sparse.cpp:31-51
  std::vector<const cd *> blk;
  std::vector<int> zero;  // -1 when max|block| < 1e-16
};

// F selector of multiply_left_vertex (bsb.cpp:141-151) / multiply_right_vertex (:477-487)
const cd *select_F(const Evaluator &E, const Backbone &B, int v, int b, int &R, int &Cc) {
  int o = B.v_orb[v];
  int q = (int)E.labels[o];
  int qo = (int)E.sinds[o];
  int l = B.pole_inds.empty() ? 0 : B.pole_inds[B.v_hyb[v]];
  if (B.v_bar[v]) {
    const SymSetBar &S = B.v_dag[v] ? E.Fdbar[q] : E.Fbarr[q];
    R = E.dims[S.index[b]]; Cc = E.dims[b];
    return S.blocks[b].data() + ((size_t)qo * S.p + l) * R * Cc;
  } else {
    const SymSet &S = B.v_dag[v] ? E.Fd[q] : E.Fs[q];
    R = E.dims[S.index[b]]; Cc = E.dims[b];
    return S.blocks[b].data() + (size_t)qo * R * Cc;
  }
}

// multiply_left_vertex bsb.cpp:127-163 with Hybridization::multiply_kernel_on_vertex hyb.cpp:46-57
void multiply_left_vertex(const Evaluator &E, const Backbone &B, Work &w, int v, int ncol, double sign) {
  int vct0 = B.t(0, 1);
  (void)vct0;
  int b = w.ind_path[v - 1];
  int R, K;
  const cd *F = select_F(E, B, v, b, R, K);
  int r = E.r;
  left_mul(r, F, R, K, w.T.data(), ncol, w.T2.data());
  std::swap(w.T, w.T2);
  w.flops += 8.0 * r * R * K * ncol;
  int ks = B.v_ksign[v];
  if (ks != 0) {
    int l = B.pole_inds[B.v_hyb[v]];
    const std::vector<double> &kt = (sign * ks > 0) ? E.kitp : E.kitm;
    for (int t = 0; t < r; ++t)
      for (int x = 0; x < R * ncol; ++x) w.T[(size_t)t * R * ncol + x] *= kt[(size_t)t * E.p + l];
  }
}

// integrate_left_edge bsb.cpp:165-178 with multiply_kernels_on_edge hyb.cpp:59-73
void edge_kernels(const Evaluator &E, const Backbone &B, int e, int d, cd *GK) {
  int r = E.r;
  for (int x = 0; x < B.m - 1; ++x) {
    int ks = B.edge(e, x);
    if (ks == 0) continue;
    int l = B.pole_inds[x];
    const std::vector<double> &kt = ks > 0 ? E.kitp : E.kitm;
    for (int t = 0; t < r; ++t)
      for (int z = 0; z < d * d; ++z) GK[(size_t)t * d * d + z] *= kt[(size_t)t * E.p + l];
  }
}
void integrate_left_edge(const Evaluator &E, const Backbone &B, const BlockG &G, Work &w, int e, int ncol) {
  int b = w.ind_path[e];
  int d = w.block_dims[e + 1];
  int r = E.r;
  std::copy(G.blk[b], G.blk[b] + (size_t)r * d * d, w.GK.begin());
  edge_kernels(E, B, e, d, w.GK.data());
  E.dlr->vals2coefs(w.GK.data(), (long)d * d, w.fc.data());
  E.dlr->vals2coefs(w.T.data(), (long)d * ncol, w.gc.data());
  E.dlr->convolve(E.beta, d, d, ncol, w.fc.data(), w.gc.data(), true, w.T.data());
  w.flops += 8.0 * ((double)r * r * (d * d + d * ncol) + 2.0 * r * r * (d * d + d * ncol) + 3.0 * r * d * d * ncol + (double)r * r * d * ncol);
}

// multiply_left_vertex_and_right_zero_vertex bsb.cpp:187-227
void zero_vertex(const Evaluator &E, const Backbone &B, Work &w, bool fwd, int b0, int pk, int pm) {
  int v = B.t(0, 1);
  int b_mu = w.ind_path[v - 1];
  int r = E.r;
  int dv = w.block_dims[v], d1 = w.block_dims[1], d0 = w.block_dims[0], dvp = w.block_dims[v + 1];
  const SymSet &Sk = fwd ? E.Fs[pk] : E.Fd[pk];
  const SymSet &Sm = fwd ? E.Fd[pm] : E.Fs[pm];
  int nk = (int)E.ssizes[pk], nm = (int)E.ssizes[pm];
  size_t sz = (size_t)r * dv * d0;
  for (int k = 0; k < nk; ++k) {
    const cd *Fk = Sk.blocks[b0].data() + (size_t)k * d1 * d0;
    right_mul(r, w.T.data(), dv, d1, Fk, d0, w.tk.data() + k * sz);
  }
  std::vector<cd> out((size_t)r * dvp * d0, 0.0);
  double hs = fwd ? 1.0 : -1.0;
  for (int mu = 0; mu < nm; ++mu) {
    std::fill(w.tm.begin(), w.tm.begin() + sz, cd(0));
    long om = E.set_to_orb[(size_t)pm * E.n + mu];
    for (int k = 0; k < nk; ++k) {
      long ok = E.set_to_orb[(size_t)pk * E.n + k];
      for (int t = 0; t < r; ++t) {
        cd h = fwd ? E.values[((size_t)t * E.n + om) * E.n + ok] : E.values_refl[((size_t)t * E.n + ok) * E.n + om];
        cd f = hs * h;
        for (int x = 0; x < dv * d0; ++x) w.tm[(size_t)t * dv * d0 + x] = cfma(f, w.tk[k * sz + (size_t)t * dv * d0 + x], w.tm[(size_t)t * dv * d0 + x]);
      }
    }
    const cd *Fm = Sm.blocks[b_mu].data() + (size_t)mu * dvp * dv;
    left_mul(r, Fm, dvp, dv, w.tm.data(), d0, w.T2.data());
    for (size_t x = 0; x < out.size(); ++x) out[x] += w.T2[x];
  }
  std::copy(out.begin(), out.end(), w.T.begin());
  w.flops += 8.0 * r * (nk * dv * d1 * d0 + nk * nm * dv * d0 + nm * dvp * dv * d0);
}

// Hybridization::multiply_kernels_prefactor hyb.cpp:75-92
double prefactor(const Evaluator &E, const Backbone &B) {
  double pf = 1.0;
  for (int x = 0; x < B.m - 1; ++x) {
    int ex = B.pf_kexp[x];
    if (ex != 0) {
      int l = B.pole_inds[x];
      double k0 = B.pf_ksign[x] > 0 ? E.k0p[l] : E.k0m[l];
      pf *= std::pow(k0, -ex);
    }
  }
  return pf;
}

// eval_self_energy_fixed_indices bsb.cpp:339-367
void eval_fixed(const Evaluator &E, const Backbone &B, const BlockG &G, Work &w, int b_ix, int pk, int pm, std::vector<cd> &Sig_b) {
  int m = B.m, vct0 = B.t(0, 1), r = E.r;
  int d1 = w.block_dims[1];
  std::copy(G.blk[w.ind_path[0]], G.blk[w.ind_path[0]] + (size_t)r * d1 * d1, w.T.begin());
  for (int v = 1; v < vct0; ++v) {
    multiply_left_vertex(E, B, w, v, w.block_dims[1], 1.0);
    integrate_left_edge(E, B, G, w, v, w.block_dims[1]);
  }
  zero_vertex(E, B, w, !B.v_dag[0], b_ix, pk, pm);
  for (int v = vct0 + 1; v < 2 * m; ++v) {
    integrate_left_edge(E, B, G, w, v - 1, w.block_dims[0]);
    multiply_left_vertex(E, B, w, v, w.block_dims[0], 1.0);
  }
  double pf = prefactor(E, B);
  int sgn = (m % 2 == 0) ? -1 : 1;
  if (B.fb[0] == 0) sgn *= -1;
  double fac = pf * sgn * B.prefactor_sign;
  int R = w.block_dims[2 * m], C = w.block_dims[0];
  if (R != E.dims[b_ix] || C != E.dims[b_ix]) throw std::invalid_argument("BlockDiagOpFun::add_block: shape mismatch");
  double mx = 0;
  size_t tot = (size_t)r * R * C;
  for (size_t x = 0; x < tot; ++x) { w.T[x] *= fac; mx = std::max(mx, std::abs(w.T[x])); }
  if (mx > 1e-16)
    for (size_t x = 0; x < tot; ++x) Sig_b[x] += w.T[x];
  w.items++;
}

// find_path_self_energy bsb.cpp:229-314.  Calls visit(b_ix, p_kap, p_mu) for each complete path.
template <class F>
void find_paths(const Evaluator &E, const Backbone &B, const BlockG &G, Work &w, F visit) {
  int m = B.m, vct0 = B.t(0, 1);
  auto Fsel_p = [&](int v, int pset) -> const SymSet & { return B.v_dag[v] ? E.Fd[pset] : E.Fs[pset]; };
  auto Fsel = [&](int v) -> const SymSet & { return Fsel_p(v, (int)E.labels[B.orb_inds[v]]); };
  auto incomplete = [&](int v, int ip) { return ip == -1 || (v < 2 * m - 1 && G.zero[ip] == -1); };
  for (int b = 0; b < E.nb; ++b)
    for (int pk = 0; pk < E.nq; ++pk) {
      bool bad = false;
      int ip = -1;
      for (int v = 0; v < vct0; ++v) {
        ip = (v == 0) ? Fsel_p(0, pk).index[b] : Fsel(v).index[ip];
        bad = incomplete(v, ip);
        if (bad) break;
        w.ind_path[v] = ip;
      }
      if (bad) continue;
      w.block_dims[0] = E.dims[b];
      w.block_dims[1] = E.dims[Fsel_p(0, pk).index[b]];
      for (int v = 0; v < vct0 - 1; ++v) w.block_dims[v + 2] = E.dims[Fsel(v + 1).index[w.ind_path[v]]];
      for (int pm = 0; pm < E.nq; ++pm) {
        if (pm != pk) continue;
        ip = w.ind_path[vct0 - 1];
        bad = false;
        for (int v = vct0; v < 2 * m; ++v) {
          ip = (v == vct0) ? Fsel_p(v, pm).index[ip] : Fsel(v).index[ip];
          bad = incomplete(v, ip);
          if (bad) break;
          if (v < 2 * m - 1) w.ind_path[v] = ip;
        }
        if (bad) continue;
        w.block_dims[vct0 + 1] = E.dims[Fsel_p(vct0, pm).index[w.ind_path[vct0 - 1]]];
        for (int v = vct0; v < 2 * m - 1; ++v) w.block_dims[v + 2] = E.dims[Fsel(v + 1).index[w.ind_path[v]]];
        visit(b, pk, pm);
      }
    }
}

void alloc_work(const Evaluator &E, Work &w) {
  size_t s = (size_t)E.r * E.Nmax * E.Nmax;
  long maxset = 1;
  for (long x : E.ssizes) maxset = std::max(maxset, x);
  w.T.assign(s, 0); w.T2.assign(s, 0); w.GK.assign(s, 0); w.fc.assign(s, 0); w.gc.assign(s, 0);
  w.tk.assign(s * maxset, 0); w.tm.assign(s, 0); w.U.assign(s, 0); w.U2.assign(s, 0);
}

BlockG make_G(const Evaluator &E, const cd *G) {
  BlockG g;
  size_t off = 0;
  for (int b = 0; b < E.nb; ++b) {
    g.blk.push_back(G + off);
    size_t sz = (size_t)E.r * E.dims[b] * E.dims[b];
    double mx = 0;
    for (size_t x = 0; x < sz; ++x) mx = std::max(mx, std::abs(G[off + x]));
    g.zero.push_back(mx < 1e-16 ? -1 : 0);
    off += sz;
  }
  return g;
}

// ---------------------------------------------------------------- correlator (bsb.cpp:517-706)
struct BlockOp {  // one flavour of F or F^dag: per block column target and (rows x cols) block
  std::vector<int> index;
  std::vector<const cd *> blk;
};

// multiply_right_vertex bsb.cpp:463-498
void multiply_right_vertex(const Evaluator &E, const Backbone &B, Work &w, int v, int nrow) {
  int b = w.ind_path[v - 1];
  int R, K;
  const cd *F = select_F(E, B, v, b, R, K);  // F: (dims[target] x dims[b]) = (block_dims(v+1) x block_dims(v))
  int r = E.r;
  // U_v(t) = U_vp(t) * F : (nrow x bd(v+1)) * (bd(v+1) x bd(v))
  right_mul(r, w.U.data(), nrow, R, F, K, w.U2.data());
  std::swap(w.U, w.U2);
  w.flops += 8.0 * r * nrow * R * K;
  int ks = B.v_ksign[v];
  if (ks != 0) {
    int l = B.pole_inds[B.v_hyb[v]];
    const std::vector<double> &kt = (-1.0 * ks > 0) ? E.kitp : E.kitm;
    for (int t = 0; t < r; ++t)
      for (int x = 0; x < nrow * K; ++x) w.U[(size_t)t * nrow * K + x] *= kt[(size_t)t * E.p + l];
  }
}
// integrate_right_edge bsb.cpp:500-515
void integrate_right_edge(const Evaluator &E, const Backbone &B, const BlockG &G, Work &w, int e, int nrow) {
  int b = w.ind_path[e];
  int d = w.block_dims[e + 1];
  int r = E.r;
  std::copy(G.blk[b], G.blk[b] + (size_t)r * d * d, w.GK.begin());
  edge_kernels(E, B, e, d, w.GK.data());
  E.dlr->vals2coefs(w.U.data(), (long)nrow * d, w.fc.data());
  E.dlr->vals2coefs(w.GK.data(), (long)d * d, w.gc.data());
  E.dlr->convolve(E.beta, nrow, d, d, w.fc.data(), w.gc.data(), true, w.U.data());
  w.flops += 8.0 * (3.0 * r * r * (d * d + d * nrow) + 3.0 * r * d * d * nrow + (double)r * r * d * nrow);
}

void eval_correlator(const Evaluator &E, const Backbone &B, const BlockG &G, const std::vector<BlockOp> &mu_ops,
                     const std::vector<BlockOp> &kap_ops, long f_ix, Work &w, cd *corr /* r x nmu x nkap, accumulated */) {
  int m = B.m, vct0 = B.t(0, 1), r = E.r, nb = E.nb;
  int nmu = (int)mu_ops.size(), nka = (int)kap_ops.size();
  auto Fsel = [&](int v) -> const SymSet & { return B.v_dag[v] ? E.Fd[E.labels[B.orb_inds[v]]] : E.Fs[E.labels[B.orb_inds[v]]]; };
  auto incomplete = [&](int ip) { return ip == -1 || G.zero[ip] == -1; };
  std::vector<std::vector<cd>> right(nb), left(nb);
  std::vector<int> rR(nb, 0), rC(nb, 0), lR(nb, 0), lC(nb, 0);
  std::vector<int> right_inds(nb, -1), left_inds(nb, -1);
  double pf = prefactor(E, B);
  // right-hand side, vertices on [tau, 0]
  for (int b = 0; b < nb; ++b) {
    bool bad = false;
    int ip = b;
    w.ind_path[0] = ip;
    for (int v = 1; v < vct0; ++v) {
      ip = Fsel(v).index[ip];
      bad = incomplete(ip);
      if (bad) break;
      w.ind_path[v] = ip;
    }
    if (bad) continue;
    w.block_dims[1] = E.dims[b];
    for (int v = 1; v < vct0; ++v) w.block_dims[v + 1] = E.dims[Fsel(v).index[w.ind_path[v - 1]]];
    int d1 = w.block_dims[1];
    std::copy(G.blk[w.ind_path[0]], G.blk[w.ind_path[0]] + (size_t)r * d1 * d1, w.T.begin());
    for (int v = 1; v < vct0; ++v) {
      multiply_left_vertex(E, B, w, v, d1, 1.0);
      integrate_left_edge(E, B, G, w, v, d1);
    }
    int R = w.block_dims[vct0];
    right[b].assign(w.T.begin(), w.T.begin() + (size_t)r * R * d1);
    for (auto &x : right[b]) x *= pf * B.prefactor_sign;
    rR[b] = R; rC[b] = d1;
    right_inds[b] = w.ind_path[vct0 - 1];
  }
  // left-hand side, vertices on [beta, tau]
  for (int b = 0; b < nb; ++b) {
    bool bad = false;
    int ip = b;
    w.ind_path[vct0] = ip;
    for (int v = vct0 + 1; v < 2 * m; ++v) {
      ip = Fsel(v).index[ip];
      bad = incomplete(ip);
      if (bad) break;
      w.ind_path[v] = ip;
    }
    if (bad) continue;
    w.block_dims[vct0 + 1] = E.dims[b];
    for (int v = vct0 + 1; v < 2 * m; ++v) w.block_dims[v + 1] = E.dims[Fsel(v).index[w.ind_path[v - 1]]];
    int nrow = w.block_dims[2 * m];
    std::copy(G.blk[w.ind_path[2 * m - 1]], G.blk[w.ind_path[2 * m - 1]] + (size_t)r * nrow * nrow, w.U.begin());
    int cur = nrow;
    for (int v = 2 * m - 1; v > vct0; --v) {
      multiply_right_vertex(E, B, w, v, nrow);
      cur = w.block_dims[v];
      integrate_right_edge(E, B, G, w, v - 1, nrow);
    }
    // U = reflect(U)
    int C = w.block_dims[vct0 + 1];
    (void)cur;
    std::vector<cd> refl((size_t)r * nrow * C);
    E.dlr->reflect(w.U.data(), (long)nrow * C, refl.data());
    int tgt = w.ind_path[vct0];
    left[tgt] = refl;
    lR[tgt] = nrow; lC[tgt] = C;
    left_inds[b] = w.ind_path[2 * m - 1];
  }
  // trace contraction: correlator = Tr[left O_mu right O_kap]
  std::vector<cd> tmp, tmuop;
  for (int mu = 0; mu < nmu; ++mu)
    for (int b = 0; b < nb; ++b) {
      int ip = right_inds[b];
      if (incomplete(ip)) continue;
      int e0 = ip;
      ip = mu_ops[mu].index[ip];
      if (incomplete(ip)) continue;
      int e1 = ip;
      ip = left_inds[ip];
      if (incomplete(ip)) continue;
      int e2 = ip;
      int c0 = rC[b], c1 = rR[b];
      int c2 = E.dims[mu_ops[mu].index[e0]];
      int c3 = lR[e1];
      const cd *Omu = mu_ops[mu].blk[e0];  // (c2 x c1)
      tmp.assign((size_t)c2 * c0, 0);
      tmuop.assign((size_t)c3 * c0, 0);
      for (int t = 0; t < r; ++t) {
        const cd *Rt = right[b].data() + (size_t)t * c1 * c0;
        const cd *Lt = left[e1].data() + (size_t)t * lR[e1] * lC[e1];
        for (int i = 0; i < c2; ++i)
          for (int j = 0; j < c0; ++j) {
            cd s = 0;
            for (int k = 0; k < c1; ++k) s = cfma(Omu[i * c1 + k], Rt[k * c0 + j], s);
            tmp[i * c0 + j] = s;
          }
        for (int i = 0; i < c3; ++i)
          for (int j = 0; j < c0; ++j) {
            cd s = 0;
            for (int k = 0; k < c2; ++k) s = cfma(Lt[i * lC[e1] + k], tmp[k * c0 + j], s);
            tmuop[i * c0 + j] = s;
          }
        for (int ka = 0; ka < nka; ++ka) {
          if (kap_ops[ka].index[e2] != b) continue;
          const cd *Ok = kap_ops[ka].blk[e2];  // (c0 x c3)
          cd s = 0;
          for (int i = 0; i < c3; ++i)
            for (int j = 0; j < c0; ++j) s = cfma(tmuop[i * c0 + j], Ok[j * c3 + i], s);
          corr[((size_t)t * nmu + mu) * nka + ka] += s;
        }
      }
    }
  (void)f_ix;
}

thread_local std::string g_err;

}  // namespace

// ==================================================================== C API
extern "C" {

const char *ora_last_error() { return g_err.c_str(); }

void *ora_dlr_new(int r, const double *rf, const double *it) {
  try { return new Dlr(r, rf, it); } catch (std::exception &e) { g_err = e.what(); return nullptr; }
}
void ora_dlr_free(void *d) { delete (Dlr *)d; }

int ora_vals2coefs(void *d, long ncol, const double *vals, double *out) {
  ((Dlr *)d)->vals2coefs((const cd *)vals, ncol, (cd *)out);
  return 0;
}
int ora_coefs2vals(void *d, long ncol, const double *c, double *out) {
  ((Dlr *)d)->coefs2vals((const cd *)c, ncol, (cd *)out);
  return 0;
}
int ora_reflect(void *d, long ncol, const double *vals, double *out) {
  ((Dlr *)d)->reflect((const cd *)vals, ncol, (cd *)out);
  return 0;
}
int ora_coefs2eval(void *d, long ncol, const double *c, double t, double *out) {
  ((Dlr *)d)->coefs2eval((const cd *)c, ncol, t, (cd *)out);
  return 0;
}
int ora_convolve(void *d, double beta, int a, int b, int c, const double *fc, const double *gc, int time_order, double *h) {
  ((Dlr *)d)->convolve(beta, a, b, c, (const cd *)fc, (const cd *)gc, time_order != 0, (cd *)h);
  return 0;
}
int ora_convmat(void *d, double beta, int n, const double *fc, int time_order, double *M) {
  ((Dlr *)d)->convmat(beta, n, (const cd *)fc, time_order != 0, (cd *)M);
  return 0;
}

// dyson_it_ppsc(beta, itops, g0).solve(sig, eta)  dlr_dyson_ppsc.hpp:91-168; with op (n x n, may be null),
// solve_with_op(sig, eta, op)  dlr_dyson_ppsc.hpp:188-216: ggs += eta g0, then ggs(k) += g0(k) op, then negated
int ora_dyson_solve_op(void *dv, double beta, int n, const double *g0_, const double *sig_, double eta, const double *op_,
                       double *g_out) {
  try {
    const Dlr &D = *(Dlr *)dv;
    int r = D.r;
    size_t sz = (size_t)r * n * n;
    const cd *g0 = (const cd *)g0_, *sig = (const cd *)sig_, *op = (const cd *)op_;
    std::vector<cd> g0c(sz), sigc(sz), ggs(sz), ggsc(sz);
    D.vals2coefs(g0, (long)n * n, g0c.data());
    D.vals2coefs(sig, (long)n * n, sigc.data());
    D.convolve(beta, n, n, n, g0c.data(), sigc.data(), true, ggs.data());
    if (op == nullptr) {
      for (size_t x = 0; x < sz; ++x) ggs[x] = -(ggs[x] + eta * g0[x]);
    } else {
      for (size_t x = 0; x < sz; ++x) ggs[x] = ggs[x] + eta * g0[x];
      for (int k = 0; k < r; ++k)
        for (int a = 0; a < n; ++a)
          for (int c = 0; c < n; ++c) {
            cd s = 0.0;
            for (int b = 0; b < n; ++b) s += g0[((size_t)k * n + a) * n + b] * op[(size_t)b * n + c];
            ggs[((size_t)k * n + a) * n + c] += s;
          }
      for (size_t x = 0; x < sz; ++x) ggs[x] = -ggs[x];
    }
    D.vals2coefs(ggs.data(), (long)n * n, ggsc.data());
    long N = (long)r * n;
    std::vector<cd> M((size_t)N * N);
    D.convmat(beta, n, ggsc.data(), true, M.data());
    for (long i = 0; i < N; ++i) M[(size_t)i * N + i] += 1.0;
    std::vector<int> piv;
    lu_factor(M, (int)N, piv);
    std::vector<cd> rhs(g0, g0 + sz);  // rows (t, i), columns j
    lu_solve(M, (int)N, piv, rhs.data(), n);
    std::copy(rhs.begin(), rhs.end(), (cd *)g_out);
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

int ora_dyson_solve(void *dv, double beta, int n, const double *g0_, const double *sig_, double eta, double *g_out) {
  return ora_dyson_solve_op(dv, beta, n, g0_, sig_, eta, nullptr, g_out);
}

// DiagramEvaluator TRIQS-free constructor (bsb.cpp:63-85) plus BlockOpSymQuartet (block_sparse.cpp:496-577)
// and Hybridization (hyb.cpp:15-44).  Poles are physical (the evaluator multiplies by beta).
// F data: for set s and block column b with index != -1, a (q_s, d_target, d_b) complex slab, packed in (s, b) order.
void *ora_eval_new(void *dv, double beta, int p, const double *poles, const double *coeffs, int n, const long *labels,
                   int nb, const int *dims, const int *F_index, const double *F_data, const int *Fd_index, const double *Fd_data) {
  try {
    auto *E = new Evaluator();
    E->dlr = (Dlr *)dv;
    E->r = E->dlr->r; E->n = n; E->p = p; E->nb = nb; E->beta = beta;
    E->dims.assign(dims, dims + nb);
    E->labels.assign(labels, labels + n);
    long nq = 0;
    for (int i = 0; i < n; ++i) nq = std::max(nq, labels[i] + 1);
    E->nq = (int)nq;
    E->sinds.assign(n, 0); E->ssizes.assign(nq, 0); E->set_to_orb.assign((size_t)nq * n, -1);
    for (int i = 0; i < n; ++i) {
      E->sinds[i] = E->ssizes[labels[i]];
      E->ssizes[labels[i]]++;
      E->set_to_orb[(size_t)labels[i] * n + E->sinds[i]] = i;
    }
    const cd *C = (const cd *)coeffs;
    check_sym_set_block_diagonal(C, p, E->labels, "DiagramEvaluator");
    // operators
    auto load = [&](const int *idx, const double *data, std::vector<SymSet> &out) {
      const cd *dp = (const cd *)data;
      out.resize(nq);
      for (int s = 0; s < nq; ++s) {
        out[s].q = (int)E->ssizes[s];
        out[s].index.assign(idx + (size_t)s * nb, idx + (size_t)(s + 1) * nb);
        out[s].blocks.resize(nb);
        for (int b = 0; b < nb; ++b) {
          int tg = out[s].index[b];
          if (tg < 0) continue;
          size_t sz = (size_t)out[s].q * dims[tg] * dims[b];
          out[s].blocks[b].assign(dp, dp + sz);
          dp += sz;
        }
      }
    };
    load(F_index, F_data, E->Fs);
    load(Fd_index, Fd_data, E->Fd);
    // barred operators, block_sparse.cpp:555-576
    E->Fdbar.resize(nq); E->Fbarr.resize(nq);
    for (int s = 0; s < nq; ++s) {
      int q = (int)E->ssizes[s];
      for (int pass = 0; pass < 2; ++pass) {
        const SymSet &S = pass == 0 ? E->Fd[s] : E->Fs[s];
        SymSetBar &B = pass == 0 ? E->Fdbar[s] : E->Fbarr[s];
        B.q = q; B.p = p; B.index = S.index; B.blocks.resize(nb);
        for (int b = 0; b < nb; ++b) {
          if (S.index[b] < 0) continue;
          size_t bs = (size_t)dims[S.index[b]] * dims[b];
          B.blocks[b].assign((size_t)q * p * bs, 0.0);
        }
      }
      for (int l = 0; l < p; ++l)
        for (int lam = 0; lam < q; ++lam)
          for (int nu = 0; nu < q; ++nu) {
            long lo = E->set_to_orb[(size_t)s * n + lam], no = E->set_to_orb[(size_t)s * n + nu];
            cd c = C[((size_t)l * n + no) * n + lo];
            for (int b = 0; b < nb; ++b) {
              if (E->Fd[s].index[b] != -1) {
                size_t bs = (size_t)dims[E->Fd[s].index[b]] * dims[b];
                cd *dst = E->Fdbar[s].blocks[b].data() + ((size_t)lam * p + l) * bs;
                const cd *src = E->Fd[s].blocks[b].data() + (size_t)nu * bs;
                for (size_t x = 0; x < bs; ++x) dst[x] += c * src[x];
              }
              if (E->Fs[s].index[b] != -1) {
                size_t bs = (size_t)dims[E->Fs[s].index[b]] * dims[b];
                cd *dst = E->Fbarr[s].blocks[b].data() + ((size_t)nu * p + l) * bs;
                const cd *src = E->Fs[s].blocks[b].data() + (size_t)lam * bs;
                for (size_t x = 0; x < bs; ++x) dst[x] += -c * src[x];
              }
            }
          }
    }
    // Hybridization hyb.cpp:15-44, coefs2vals hyb.cpp:94-113
    int r = E->r;
    E->poles_beta.resize(p);
    for (int l = 0; l < p; ++l) E->poles_beta[l] = poles[l] * beta;
    E->coeffs.assign(C, C + (size_t)p * n * n);
    E->values.assign((size_t)r * n * n, 0.0);
    for (int t = 0; t < r; ++t)
      for (int l = 0; l < p; ++l) {
        double k = k_it(E->dlr->it[t], E->poles_beta[l]);
        for (int z = 0; z < n * n; ++z) E->values[(size_t)t * n * n + z] += k * C[(size_t)l * n * n + z];
      }
    E->values_refl.resize((size_t)r * n * n);
    E->dlr->reflect(E->values.data(), (long)n * n, E->values_refl.data());
    E->kitp.resize((size_t)r * p); E->kitm.resize((size_t)r * p); E->k0p.resize(p); E->k0m.resize(p);
    for (int l = 0; l < p; ++l) {
      E->k0p[l] = k_it(0.0, E->poles_beta[l]);
      E->k0m[l] = k_it(0.0, -E->poles_beta[l]);
      for (int t = 0; t < r; ++t) {
        E->kitp[(size_t)t * p + l] = k_it(E->dlr->it[t], E->poles_beta[l]);
        E->kitm[(size_t)t * p + l] = k_it(E->dlr->it[t], -E->poles_beta[l]);
      }
    }
    E->Nmax = 1;
    for (int b = 0; b < nb; ++b) E->Nmax = std::max(E->Nmax, dims[b]);
    return E;
  } catch (std::exception &e) { g_err = e.what(); return nullptr; }
}
void ora_eval_free(void *e) { delete (Evaluator *)e; }

long ora_num_sigma_backbones(void *ev, int m, const int *topo) {
  auto *E = (Evaluator *)ev;
  return Backbone(m, topo, E->n, E->p, false).num_backbones();
}
long ora_num_spgf_backbones(void *ev, int m, const int *topo) {
  auto *E = (Evaluator *)ev;
  return Backbone(m, topo, E->n, E->p, true).num_backbones();
}

// compute_self_energy(G, topology[, f_ix_vec]) bsb.cpp:369-459.  G and Sigma are packed complex slabs
// (blocks in order, each r x d x d).  fix == nullptr evaluates every flat index.
int ora_sigma(void *ev, const double *G_, int m, const int *topo, const long *fix, long nfix, int nthreads, double *Sig_out,
              long *n_items, double *flops) {
  try {
    auto *E = (Evaluator *)ev;
    const cd *G = (const cd *)G_;
    Backbone B0(m, topo, E->n, E->p, false);
    long nmax = B0.num_backbones();
    long count = fix ? nfix : nmax;
    for (long z = 0; fix && z < nfix; ++z)
      if (fix[z] < 0 || fix[z] >= nmax) throw std::runtime_error("DiagramEvaluator::eval_self_energy: f_ix out of range");
    BlockG g = make_G(*E, G);
    std::vector<size_t> off(E->nb + 1, 0);
    for (int b = 0; b < E->nb; ++b) off[b + 1] = off[b] + (size_t)E->r * E->dims[b] * E->dims[b];
    size_t total = off[E->nb];
    std::vector<cd> Sig(total, 0.0);
    long items = 0;
    double fl = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel num_threads(nthreads)
    {
      Backbone B(m, topo, E->n, E->p, false);
      Work w;
      alloc_work(*E, w);
      std::vector<std::vector<cd>> loc(E->nb);
      for (int b = 0; b < E->nb; ++b) loc[b].assign((size_t)E->r * E->dims[b] * E->dims[b], 0.0);
#pragma omp for schedule(dynamic, 16)
      for (long z = 0; z < count; ++z) {
        long f = fix ? fix[z] : z;
        B.set_flat_index(f, E->poles_beta);
        find_paths(*E, B, g, w, [&](int b, int pk, int pm) { eval_fixed(*E, B, g, w, b, pk, pm, loc[b]); });
      }
#pragma omp critical
      {
        for (int b = 0; b < E->nb; ++b)
          for (size_t x = 0; x < loc[b].size(); ++x) Sig[off[b] + x] += loc[b][x];
        items += w.items;
        fl += w.flops;
      }
    }
    // set_zero_block_indices and block_gf conversion: a block with max|.| < 1e-16 comes back as zeros
    for (int b = 0; b < E->nb; ++b) {
      double mx = 0;
      for (size_t x = off[b]; x < off[b + 1]; ++x) mx = std::max(mx, std::abs(Sig[x]));
      if (mx < 1e-16)
        for (size_t x = off[b]; x < off[b + 1]; ++x) Sig[x] = 0;
    }
    std::copy(Sig.begin(), Sig.end(), (cd *)Sig_out);
    if (n_items) *n_items = items;
    if (flops) *flops = fl;
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

// compute_self_energy(G, topology) summed in the fixed order of the device's ordered mode (the items are
// the reference's; only the order of the additions into Sigma is fixed here, so two runs, and this
// restatement and the device, agree bit for bit).  Per output block b: the path classes (fb_ix, o_ix,
// p_kap) in that order, each class's value the sum over runs of `unit` consecutive pole tuples (p_ix
// ascending), each run's value the sum of its items in p_ix order; every partial sum starts from zero.
// The runs of one (fb_ix, o_ix) group are evaluated in parallel.
int ora_sigma_ordered(void *ev, const double *G_, int m, const int *topo, long unit, int nthreads, double *Sig_out, long *n_items) {
  try {
    auto *E = (Evaluator *)ev;
    if (unit < 1) throw std::invalid_argument("unit must be positive");
    const cd *G = (const cd *)G_;
    Backbone B0(m, topo, E->n, E->p, false);
    BlockG g = make_G(*E, G);
    std::vector<size_t> off(E->nb + 1, 0);
    for (int b = 0; b < E->nb; ++b) off[b + 1] = off[b] + (size_t)E->r * E->dims[b] * E->dims[b];
    std::vector<cd> Sig(off[E->nb], 0.0);
    const long omax = B0.o_ix_max, npt = B0.p_ix_max, fbmax = B0.fb_ix_max;
    const long nruns = (npt + unit - 1) / unit;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    long items = 0;
    for (long fb = 0; fb < fbmax; ++fb)
      for (long o = 0; o < omax; ++o) {
        // the valid (b, p_kap) classes of this group do not depend on the pole tuple
        std::vector<std::pair<int, int>> cls;
        {
          Backbone B(m, topo, E->n, E->p, false);
          Work w;
          B.set_flat_index(o + omax * (npt * fb), E->poles_beta);
          find_paths(*E, B, g, w, [&](int b, int pk, int) { cls.emplace_back(b, pk); });
        }
        if (cls.empty()) continue;
        const size_t nc = cls.size();
        std::vector<std::vector<cd>> part(nruns * nc);
        long grp_items = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : grp_items)
        {
          Backbone B(m, topo, E->n, E->p, false);
          Work w;
          alloc_work(*E, w);
#pragma omp for schedule(dynamic, 1)
          for (long run = 0; run < nruns; ++run) {
            for (size_t k = 0; k < nc; ++k) part[run * nc + k].assign((size_t)E->r * E->dims[cls[k].first] * E->dims[cls[k].first], 0.0);
            for (long pix = run * unit; pix < std::min(npt, (run + 1) * unit); ++pix) {
              B.set_flat_index(o + omax * (pix + npt * fb), E->poles_beta);
              size_t k = 0;
              find_paths(*E, B, g, w, [&](int b, int pk, int pm) {
                while (k < nc && !(cls[k].first == b && cls[k].second == pk)) ++k;
                if (k == nc) throw std::logic_error("class set changed with the pole tuple");
                eval_fixed(*E, B, g, w, b, pk, pm, part[run * nc + k]);
              });
            }
            grp_items += w.items;
            w.items = 0;
          }
        }
        items += grp_items;
        for (size_t k = 0; k < nc; ++k) {
          const int b = cls[k].first;
          std::vector<cd> cp((size_t)E->r * E->dims[b] * E->dims[b], 0.0);
          for (long run = 0; run < nruns; ++run)
            for (size_t x = 0; x < cp.size(); ++x) cp[x] += part[run * nc + k][x];
          for (size_t x = 0; x < cp.size(); ++x) Sig[off[b] + x] += cp[x];
        }
      }
    for (int b = 0; b < E->nb; ++b) {
      double mx = 0;
      for (size_t x = off[b]; x < off[b + 1]; ++x) mx = std::max(mx, std::abs(Sig[x]));
      if (mx < 1e-16)
        for (size_t x = off[b]; x < off[b + 1]; ++x) Sig[x] = 0;
    }
    std::copy(Sig.begin(), Sig.end(), (cd *)Sig_out);
    if (n_items) *n_items = items;
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

// compute_self_energy(G, topology, f_ix_vec) with the additions into Sigma in list order (for each listed
// flat index its items in (b_ix, p_kap) order, each block's sum from zero), the order of the device's
// ordered mode for a flat-index list.  The items are evaluated in parallel and summed afterwards.
int ora_sigma_list_ordered(void *ev, const double *G_, int m, const int *topo, const long *fix, long nfix, int nthreads, double *Sig_out) {
  try {
    auto *E = (Evaluator *)ev;
    Backbone B0(m, topo, E->n, E->p, false);
    const long nmax = B0.num_backbones();
    for (long z = 0; z < nfix; ++z)
      if (fix[z] < 0 || fix[z] >= nmax) throw std::runtime_error("DiagramEvaluator::eval_self_energy: f_ix out of range");
    BlockG g = make_G(*E, (const cd *)G_);
    std::vector<size_t> off(E->nb + 1, 0);
    for (int b = 0; b < E->nb; ++b) off[b + 1] = off[b] + (size_t)E->r * E->dims[b] * E->dims[b];
    // per listed index: its contributions (block, slab) in visit order
    std::vector<std::vector<std::pair<int, std::vector<cd>>>> parts(nfix);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel num_threads(nthreads)
    {
      Backbone B(m, topo, E->n, E->p, false);
      Work w;
      alloc_work(*E, w);
#pragma omp for schedule(dynamic, 1)
      for (long z = 0; z < nfix; ++z) {
        B.set_flat_index(fix[z], E->poles_beta);
        find_paths(*E, B, g, w, [&](int b, int pk, int pm) {
          std::vector<cd> one((size_t)E->r * E->dims[b] * E->dims[b], 0.0);
          eval_fixed(*E, B, g, w, b, pk, pm, one);
          parts[z].emplace_back(b, std::move(one));
        });
      }
    }
    std::vector<cd> Sig(off[E->nb], 0.0);
    for (long z = 0; z < nfix; ++z)
      for (auto &pr : parts[z])
        for (size_t x = 0; x < pr.second.size(); ++x) Sig[off[pr.first] + x] += pr.second[x];
    for (int b = 0; b < E->nb; ++b) {
      double mx = 0;
      for (size_t x = off[b]; x < off[b + 1]; ++x) mx = std::max(mx, std::abs(Sig[x]));
      if (mx < 1e-16)
        for (size_t x = off[b]; x < off[b + 1]; ++x) Sig[x] = 0;
    }
    std::copy(Sig.begin(), Sig.end(), (cd *)Sig_out);
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

// Valid item list of find_path_self_energy for flat indices [f0, f1): rows (f_ix, b_ix, p_kap, ind_path[0..2m-2]).
long ora_items(void *ev, const double *G_, int m, const int *topo, long f0, long f1, long *out, long max_rows) {
  auto *E = (Evaluator *)ev;
  Backbone B(m, topo, E->n, E->p, false);
  BlockG g = make_G(*E, (const cd *)G_);
  Work w;
  long rows = 0;
  int width = 3 + 2 * m - 1;
  for (long f = f0; f < f1; ++f) {
    B.set_flat_index(f, E->poles_beta);
    find_paths(*E, B, g, w, [&](int b, int pk, int) {
      if (rows < max_rows) {
        long *o = out + rows * width;
        o[0] = f; o[1] = b; o[2] = pk;
        for (int i = 0; i < 2 * m - 1; ++i) o[3 + i] = w.ind_path[i];
      }
      rows++;
    });
  }
  return rows;
}

// compute_single_ptcle_gf(G, topology[, f_ix_vec]) bsb.cpp:779-821 with the mu/kap operators of
// setup_mu_ops_for_single_ptcle_gf / setup_kap_ops_for_single_ptcle_gf (:739-777).  g_out is (r, n, n) complex.
int ora_spgf(void *ev, const double *G_, int m, const int *topo, const long *fix, long nfix, int nthreads, double *g_out) {
  try {
    auto *E = (Evaluator *)ev;
    Backbone B0(m, topo, E->n, E->p, true);
    long nmax = B0.num_backbones();
    long count = fix ? nfix : nmax;
    BlockG g = make_G(*E, (const cd *)G_);
    std::vector<BlockOp> mu(E->n), ka(E->n);
    for (int o = 0; o < E->n; ++o) {
      int s = (int)E->labels[o], i = (int)E->sinds[o];
      mu[o].index = E->Fs[s].index;
      ka[o].index = E->Fd[s].index;
      mu[o].blk.assign(E->nb, nullptr);
      ka[o].blk.assign(E->nb, nullptr);
      for (int b = 0; b < E->nb; ++b) {
        if (E->Fs[s].index[b] >= 0) mu[o].blk[b] = E->Fs[s].blocks[b].data() + (size_t)i * E->dims[E->Fs[s].index[b]] * E->dims[b];
        if (E->Fd[s].index[b] >= 0) ka[o].blk[b] = E->Fd[s].blocks[b].data() + (size_t)i * E->dims[E->Fd[s].index[b]] * E->dims[b];
      }
    }
    size_t tot = (size_t)E->r * E->n * E->n;
    std::vector<cd> acc(tot, 0.0);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel num_threads(nthreads)
    {
      Backbone B(m, topo, E->n, E->p, true);
      Work w;
      alloc_work(*E, w);
      std::vector<cd> loc(tot, 0.0);
#pragma omp for schedule(dynamic, 4)
      for (long z = 0; z < count; ++z) {
        long f = fix ? fix[z] : z;
        B.set_flat_index(f, E->poles_beta);
        eval_correlator(*E, B, g, mu, ka, f, w, loc.data());
      }
#pragma omp critical
      for (size_t x = 0; x < tot; ++x) acc[x] += loc[x];
    }
    (void)nmax;
    std::copy(acc.begin(), acc.end(), (cd *)g_out);
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

// compute_one_time_correlator(G, ops_tau, ops_0, ad, topology, f_ix_vec) bsb.cpp:843-866: eval_correlator with
// the given block operators (setup_ops_from_triqs_2nd_quant_ops, :810-840) in place of F_mu and F^dag_ka.
// mu_index[mu * nb + b] (-1: none) and mu_data packing the (d_target x d_b) blocks in (mu, b) order; likewise
// ka.  out is (r, nmu, nka) complex.
int ora_correlator(void *ev, const double *G_, int m, const int *topo, const long *fix, long nfix, int nthreads, int nmu,
                   const int *mu_index, const double *mu_data, int nka, const int *ka_index, const double *ka_data, double *out) {
  try {
    auto *E = (Evaluator *)ev;
    Backbone B0(m, topo, E->n, E->p, true);
    long nmax = B0.num_backbones();
    long count = fix ? nfix : nmax;
    for (long z = 0; fix && z < nfix; ++z)
      if (fix[z] < 0 || fix[z] >= nmax) throw std::runtime_error("DiagramEvaluator::compute_one_time_correlator: f_ix out of range");
    BlockG g = make_G(*E, (const cd *)G_);
    auto build = [&](int nops, const int *index, const double *data, std::vector<BlockOp> &ops) {
      const cd *dp = (const cd *)data;
      ops.resize(nops);
      for (int o = 0; o < nops; ++o) {
        ops[o].index.assign(index + (size_t)o * E->nb, index + (size_t)(o + 1) * E->nb);
        ops[o].blk.assign(E->nb, nullptr);
        for (int b = 0; b < E->nb; ++b) {
          const int t = ops[o].index[b];
          if (t < 0) continue;
          ops[o].blk[b] = dp;
          dp += (size_t)E->dims[t] * E->dims[b];
        }
      }
    };
    std::vector<BlockOp> mu, ka;
    build(nmu, mu_index, mu_data, mu);
    build(nka, ka_index, ka_data, ka);
    size_t tot = (size_t)E->r * nmu * nka;
    std::vector<cd> acc(tot, 0.0);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
#pragma omp parallel num_threads(nthreads)
    {
      Backbone B(m, topo, E->n, E->p, true);
      Work w;
      alloc_work(*E, w);
      std::vector<cd> loc(tot, 0.0);
#pragma omp for schedule(dynamic, 4)
      for (long z = 0; z < count; ++z) {
        long f = fix ? fix[z] : z;
        B.set_flat_index(f, E->poles_beta);
        eval_correlator(*E, B, g, mu, ka, f, w, loc.data());
      }
#pragma omp critical
      for (size_t x = 0; x < tot; ++x) acc[x] += loc[x];
    }
    std::copy(acc.begin(), acc.end(), (cd *)out);
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

// expectation_value(op, ad, G) block_sparse.cpp:797-818: sum += -trace(O_b G_b(beta)) over the blocks with an
// operator block (op_index[b] == b), G_b(beta) by DLR evaluation; the trace entries (O G)_xx as fused
// multiply-adds over the inner index, the diagonal and the blocks summed in order.
int ora_expectation(void *dv, int nb, const int *dims, const double *G_, const int *op_index, const double *op_data, double *out) {
  try {
    const Dlr &D = *(Dlr *)dv;
    const int r = D.r;
    const cd *G = (const cd *)G_, *op = (const cd *)op_data;
    cd sum = 0;
    size_t goff = 0;
    for (int b = 0; b < nb; ++b) {
      const int d = dims[b];
      const size_t sz = (size_t)r * d * d;
      if (op_index[b] != -1 && op_index[b] != b) throw std::invalid_argument("expectation_value: operator must be block diagonal");
      if (op_index[b] == b) {
        std::vector<cd> c(sz), gb((size_t)d * d);
        D.vals2coefs(G + goff, (long)d * d, c.data());
        D.coefs2eval(c.data(), (long)d * d, 1.0, gb.data());
        cd tr = 0;
        for (int x = 0; x < d; ++x) {
          cd s = 0;
          for (int y = 0; y < d; ++y) s = cfma(op[x * d + y], gb[y * d + x], s);
          tr += s;
        }
        sum += -tr;
        op += (size_t)d * d;
      }
      goff += sz;
    }
    out[0] = sum.real();
    out[1] = sum.imag();
    return 0;
  } catch (std::exception &e) { g_err = e.what(); return 1; }
}

// Hybridization values / reflected values and kernel tables (for cross-checks)
int ora_hyb_values(void *ev, double *vals, double *vals_refl) {
  auto *E = (Evaluator *)ev;
  std::copy(E->values.begin(), E->values.end(), (cd *)vals);
  std::copy(E->values_refl.begin(), E->values_refl.end(), (cd *)vals_refl);
  return 0;
}

}  // extern "C"
