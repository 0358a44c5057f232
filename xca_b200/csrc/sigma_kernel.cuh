// Sigma backbone evaluation on the device: one warp per (path class, pole tuple) item, all of the
// item's chain resident in shared memory, one work unit (a run of pole tuples of one path class) per
// scheduling step.
//
// The arithmetic of one item follows the reference's eval_self_energy_fixed_indices
// (c++/triqs_xca/block_sparse_backbone.cpp:339-367): vertex multiplies (:127-163 with
// hyb.cpp:46-57), edge convolutions (:165-178 with hyb.cpp:59-73 and the cppdlr time-ordered
// convolution), the zero-vertex hybridization contraction (:187-227), the K(0) prefactor
// (hyb.cpp:75-92), the order / direction sign and the 1e-16 contribution guard (:359-366).
// The backbone decode of a pole tuple restates Backbone::set_pole_inds (backbone.cpp:86-150).
#pragma once
#include <cstdint>

namespace xca {

constexpr int MAXM = 3;             // orders 1..3 (NCA, OCA, TCA)
constexpr int MAXV = 2 * MAXM;      // vertices
constexpr int NBUF = 6;             // per-warp slabs: A, B, C, D, E, ACC
constexpr int MAXE = 2 * MAXM;      // largest K(0) exponent of a prefactor, plus one

struct DevBasis {
  int r, p, n, nb, nq, nmax;
  double beta;
  const double *LU;     // r x r packed LU of K(t_i, om_l) (unit lower L below the diagonal)
  const int *piv;       // r, LAPACK row-swap sequence
  const double *W;      // r x r: W[l][k] = K(0, om_k) / (om_k - om_l), 0 on the diagonal
  const double *Kit;    // r x r: K(t_i, om_l)
  const double *tabs;   // r: absolute t_i
  const double *k0;     // r: K(0, om_l)
  const double *kitp;   // r x p: K(t_i, +beta w_l)
  const double *kitm;   // r x p: K(t_i, -beta w_l)
  const double *k0p;    // p
  const double *k0m;    // p
  const double *kpow;   // [2][p][MAXE+1]: pow(k0p[l], -e) (row 0) and pow(k0m[l], -e) (row 1)
  const double *polesb; // p: beta w_l
  const double *hval;   // r x n x n: Delta(tau_i)
  const double *hrefl;  // r x n x n: Delta(beta - tau_i)
  const long *goff;     // nb: offsets of the blocks in a packed slab
  const int *dims;      // nb
  const double *ops;    // all operator slabs
  const long *F_off, *Fd_off, *Fb_off, *Fdb_off;  // [s * nb + b] -> offset into ops, -1 when absent
  const int *set_to_orb;                          // [s * n + i]
};

struct ClassRec {
  int m, vct0, fbmask, b_out, pk;
  int npt;                 // pole tuples p^(m-1)
  int la[MAXM], lb[MAXM];  // line endpoints
  int ind_path[2 * MAXM - 1];
  int bdims[2 * MAXM + 1];
  int vkind[MAXV];         // 0: F, 1: F^dag, 2: F^bar (reflected), 3: F^dag bar
  int vset[MAXV], vqo[MAXV], vline[MAXV];
};

struct WorkUnit {
  int cls;
  int first;
  int count;
};

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Arithmetic of the plain FP64 path: every product and sum rounded on its own (no contraction), in the
// operation order of the reference's CPU arithmetic, so that one item's result is bit-identical to it.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// X (r x ncol, row-major) <- K^{-1} X by the stored LU (LAPACK getrs order): row swaps, unit-lower then
// upper substitution, one column per lane.
__device__ __forceinline__ void lu_solve_cols(const double *__restrict__ LU, const int *__restrict__ piv, int r, double *X, int ncol,
                                              int lane) {
  for (int c = lane; c < ncol; c += 32) {
    for (int k = 0; k < r; ++k) {
      int pk = piv[k];
      if (pk != k) {
        double a = X[k * ncol + c];
        X[k * ncol + c] = X[pk * ncol + c];
        X[pk * ncol + c] = a;
      }
    }
    for (int i = 1; i < r; ++i) {
      double s = X[i * ncol + c];
      for (int k = 0; k < i; ++k) s = sub(s, mul(LU[i * r + k], X[k * ncol + c]));
      X[i * ncol + c] = s;
    }
    for (int i = r - 1; i >= 0; --i) {
      double s = X[i * ncol + c];
      for (int k = i + 1; k < r; ++k) s = sub(s, mul(LU[i * r + k], X[k * ncol + c]));
      X[i * ncol + c] = __ddiv_rn(s, LU[i * r + i]);
    }
  }
}

// Y (r x ncol) = M (r x r) X (r x ncol), each dot product summed from zero in ascending order.
__device__ __forceinline__ void matvec_cols(const double *__restrict__ M, int r, const double *X, double *Y, int ncol, int lane) {
  int tot = r * ncol;
  for (int idx = lane; idx < tot; idx += 32) {
    int l = idx / ncol, c = idx - l * ncol;
    const double *mr = M + l * r;
    double s = 0.0;
    for (int k = 0; k < r; ++k) s = add(s, mul(mr[k], X[k * ncol + c]));
    Y[idx] = s;
  }
}

}  // namespace xca
