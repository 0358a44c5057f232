// Sigma backbone evaluation on the device (plain FP64 path).
//
// Work decomposition: a path class (topology, directions, orbital tuple, output block, symmetry set:
// everything but the pole tuple) fixes the block chain, so its p^(m-1) items share every shape.  A
// warp takes a work unit (a run of pole tuples of one class) and evaluates `batch` of them in
// lockstep: for column-wise steps (LU substitution, Hilbert sums, the K(t_i, om_l) contraction) each
// lane owns one (item, column) of the T slab and keeps that column in registers; for row-mixing steps
// (vertex and small block products) the lanes stride over (item, node, row, column) outputs.
//
// The arithmetic of one item follows the reference's eval_self_energy_fixed_indices
// (c++/triqs_xca/block_sparse_backbone.cpp:339-367): vertex multiplies (:127-163 with
// hyb.cpp:46-57), edge convolutions (:165-178 with hyb.cpp:59-73 and the time-ordered DLR
// convolution), the zero-vertex hybridization contraction (:187-227), the K(0) prefactor
// (hyb.cpp:75-92), the order / direction sign and the 1e-16 contribution guard (:359-366).  Every
// product and sum is rounded exactly as in the operation order of the CPU
// restatement (one fused multiply-add wherever it fuses one), so each item's contribution is
// bit-identical to it.  The G-side coefficients of an
// edge (fc = K^-1 (G_b * prod K) and W fc) depend only on the block and the edge's K factors; they are
// tabulated once per G by edge_table_kernel.
#pragma once
#include <cstdint>

namespace xca {

constexpr int MAXM = 3;             // orders 1..3 (NCA, OCA, TCA)
constexpr int MAXV = 2 * MAXM;      // vertices
constexpr int MAXE = 2 * MAXM;      // largest K(0) exponent of a prefactor, plus one
constexpr int NSLAB = 3;            // per-item slabs: T, X, Y
constexpr int WARPS_MAX = 8;
constexpr int PANEL_BMAX = 128;    // items per panel batch at most

struct DevBasis {
  int r, p, n, nb, nq;
  double beta;
  const double *LUp;    // RP x RP padded LU of K(t_i, om_l), column-major: unit L below the diagonal, U on and above
                        // (pad: U_kk = 1), followed by the RP reciprocals 1 / U_kk
  const int *perm;      // RP: row gathered into position i by the pivoting (-1 beyond r)
  const int *pinv;      // RP: position of row t after the pivoting (-1 beyond r)
  const double *Wp;     // RP x RP column-major: W[l][k] = K(0, om_k) / (om_k - om_l), 0 on the diagonal and in the pad
  const double *BKp;    // RP x RP column-major: beta * K(t_i, om_l), 0 in the pad
  const double *tabs;   // r: absolute t_i
  const double *k0;     // r: K(0, om_l)
  const double *kitp;   // r x p: K(t_i, +beta w_l)
  const double *kitm;   // r x p: K(t_i, -beta w_l)
  const double *kpow;   // [2][p][MAXE+1]: pow(K(0, +beta w_l), -e) (row 0) and pow(K(0, -beta w_l), -e) (row 1)
  const double *polesb; // p: beta w_l
  const double *hval;   // r x n x n: Delta(tau_i)
  const double *hrefl;  // r x n x n: Delta(beta - tau_i)
  const long *goff;     // nb: offsets of the blocks in a packed slab
  const int *dims;      // nb
  const double *ops;    // all operator slabs
  const long *F_off, *Fd_off, *Fb_off, *Fdb_off;  // [s * nb + b] -> offset into ops, -1 when absent
  const int *set_to_orb;                          // [s * n + i]
  const double *tab;    // edge tables: per block b at tab_off[b], per signature [fc (r d^2) | W fc (r d^2)]
  const long *tab_off;
  int nsig;             // signatures per block: 1 + 2p (+ 4p^2 when two K factors can meet on an edge)
  const double *gmax;   // nullptr, or per block max |G_b| of this call's G: the kernels then drop the work units
                        // whose block path meets a block below 1e-16 (the work list was built without that test)
};

// Does the block path of a class meet a zero block of G (max |G_b| < 1e-16, find_path_self_energy,
// c++/triqs_xca/block_sparse_backbone.cpp:248-262)?  Only when the work list was built without the test.
__device__ __forceinline__ bool path_meets_zero_block(const DevBasis &B, const int *ind_path, int m) {
  if (B.gmax == nullptr) return false;
  bool z = false;
  for (int v = 0; v < 2 * m - 1; ++v) z |= B.gmax[ind_path[v]] < 1e-16;
  return z;
}

struct ClassRec {
  int m, vct0, fbmask, b_out, pk;
  int npt;                 // pole tuples p^(m-1)
  int batch;               // items a CTA evaluates together as panel columns: batch * dcmax <= panel width
  int dcmax;               // panel columns of one item at the widest point of the chain
  int wide;                // 1: dcmax exceeds the panel width, evaluated by sigma_wide_kernel
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
  int job = 0;  // job index of a job-batched launch (0 otherwise)
};

// Where a Sigma launch puts its result.  Fast mode (slots == nullptr): every batch adds scale * (its sum)
// into Sigma with atomics, so the order in which items reach Sigma varies from run to run.  Ordered
// mode: work unit u keeps the running sum of its items, in pole-tuple order, in slots + slot_off[u]
// (r d_out d_0 doubles); a reduction kernel then sums the units in a fixed order into Sigma.
struct SigmaOut {
  double *Sigma;
  double scale;
  double *slots;
  const long *slot_off;
};

// One job of a job-batched Sigma launch: a solve's basis, model and edge tables (B), the path classes of
// one topology, the solve's G and where the topology's Sigma goes (fast summation: Sigma += scale * ...).
struct SigmaJob {
  DevBasis B;
  const ClassRec *classes;
  const double *G;
  SigmaOut out;
};

// Per-item state of a batch, kept in shared memory.
struct ItemState {
  double scale;          // prefactor * prefactor sign * order / direction sign
  int lpole[MAXM];       // pole index of line i (i >= 1)
  int caseA[MAXM];       // line i in case 4(a): K on its end vertices; else 4(b): K on the edges it spans
  long taboff;           // per-step: edge-table offset of this item
  int keep;              // 1e-16 guard outcome
};

// Device state of the Dyson solve, trace and normalisation kernels (dyson_kernel.cuh).
struct DysonBasis {
  int r, nb;
  double beta;
  const double *LUp, *Wp, *BKp;  // RP x RP column-major (as DevBasis)
  const int *perm;
  const double *tabs, *k0, *k1;  // r: absolute t_i, K(0, om_l), K(1, om_l)
  const double *rf;              // r: DLR frequencies om_l
  const long *goff;              // nb: block offsets in a packed slab
  const int *dims;               // nb
  const long *woff;              // nb: per-block work offsets (6 r d^2 doubles each)
  const long *moff;              // nb: per-block system matrix offsets ((r d)^2 doubles each)
  const double *g0, *g0c, *g0t;  // packed slabs: G0 values, K^-1 G0, W K^-1 G0
  double *work;
  double *mats;
  const double *convw;           // RP^3: ((beta K_il) K_k(0)) / (om_k - om_l) at (k RP + l) RP + i
};

// D = A B + C on one 8 x 8 x 4 tile (a: A[g][q], b: B[q][g], c/d: C[g][2q], C[g][2q + 1], g = lane / 4, q = lane % 4).
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};" : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

// Batched small matrix products on the FP64 tensor cores, shared by the warps of a CTA:
// for every batch entry e < nbatch, C_e[m][n] = sum_{k < K} A_e(m, k) B_e(k, n) for m < M, n < N, each entry
// one chain of fused multiply-adds over k ascending from zero (an m8n8k4 MMA computes its tile as four
// correctly rounded fused multiply-adds in ascending k), handed to epi(e, m, n, value).  Warps take 8 x 8
// output tiles in turn (a warp index `warp` of `nwarps`); out-of-range rows, columns and k read as zero,
// which adds exactly zero to the chain.  The accessors a(e, m, k) and b(e, k, n) read the operands.
template <class FA, class FB, class FE>
__device__ __forceinline__ void warp_gemm_dmma(int nbatch, int M, int N, int K, FA a, FB b, FE epi, int warp, int nwarps) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int mt = (M + 7) >> 3, nt = (N + 7) >> 3;
  const long ntiles = (long)nbatch * mt * nt;
  for (long tile = warp; tile < ntiles; tile += nwarps) {
    const int e = (int)(tile / (mt * nt));
    const int rem = (int)(tile - (long)e * mt * nt);
    const int m0 = (rem / nt) * 8, n0 = (rem - (rem / nt) * nt) * 8;
    const int ma = m0 + g, nb = n0 + g;
    double c0 = 0.0, c1 = 0.0;
    // the next k-group's fragments are loaded before the current MMA issues
    double an = (ma < M && q < K) ? a(e, ma, q) : 0.0;
    double bn = (q < K && nb < N) ? b(e, q, nb) : 0.0;
    for (int k0 = 0; k0 < K; k0 += 4) {
      const double av = an, bv = bn;
      const int k = k0 + 4 + q;
      if (k0 + 4 < K) {
        an = (ma < M && k < K) ? a(e, ma, k) : 0.0;
        bn = (k < K && nb < N) ? b(e, k, nb) : 0.0;
      }
      dmma(c0, c1, av, bv);
    }
    const int nc = n0 + 2 * q;
    if (ma < M) {
      if (nc < N) epi(e, ma, nc, c0);
      if (nc + 1 < N) epi(e, ma, nc + 1, c1);
    }
  }
}

// Arithmetic of the plain FP64 path: the fused multiply-adds and the separately rounded products and
// sums of the CPU restatement, at the same places and in the same order.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double fmad(double a, double b, double c) { return __fma_rn(a, b, c); }

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// x <- K^{-1} x for one register-resident column (already gathered through the pivoting): forward
// unit-lower then backward upper substitution in dtrsm column order, the upper factor's diagonal applied
// as a multiplication by its precomputed reciprocal (x_k <- x_k * (1 / U_kk), as BLAS triangular solves
// with an inverted packed diagonal do).  LUT is the LU factor stored column-major (LUT[k * RP + i] =
// LU[i][k]) followed by the RP reciprocals (LUT[RP * RP + k] = 1 / U_kk; 1 in the pad).  Operand pairs
// at even offsets are loaded together.  Padding rows stay zero.
template <int RP>
__device__ __forceinline__ void lu_solve_reg(const double *__restrict__ LUT, double (&x)[RP]) {
#pragma unroll
  for (int k = 0; k < RP; ++k) {
    const double xk = x[k];
    const double *col = LUT + k * RP;
    if ((k + 1) < RP && ((k + 1) & 1)) x[k + 1] = fmad(-col[k + 1], xk, x[k + 1]);
#pragma unroll
    for (int i = (k + 2) & ~1; i + 1 < RP; i += 2) {
      const double2 l = *reinterpret_cast<const double2 *>(col + i);
      x[i] = fmad(-l.x, xk, x[i]);
      x[i + 1] = fmad(-l.y, xk, x[i + 1]);
    }
  }
#pragma unroll
  for (int k = RP - 1; k >= 0; --k) {
    x[k] = mul(x[k], LUT[RP * RP + k]);
    const double xk = x[k];
    const double *col = LUT + k * RP;
#pragma unroll
    for (int i = 0; i + 1 < k; i += 2) {
      const double2 l = *reinterpret_cast<const double2 *>(col + i);
      x[i] = fmad(-l.x, xk, x[i]);
      x[i + 1] = fmad(-l.y, xk, x[i + 1]);
    }
    if (k & 1) x[k - 1] = fmad(-col[k - 1], xk, x[k - 1]);
  }
}

// y_l = sum_k M[l][k] x_k for l < r (fused multiply-adds from zero, k ascending), with MT = M stored
// column-major (MT[k * RP + l]); y written with stride `ld`.
template <int RP>
__device__ __forceinline__ void matvec_reg(const double *__restrict__ MT, const double (&x)[RP], int r, double *y, int ld) {
  constexpr int CH = 8;
#pragma unroll 1
  for (int l0 = 0; l0 < RP; l0 += CH) {
    if (l0 >= r) break;
    double acc[CH];
#pragma unroll
    for (int j = 0; j < CH; ++j) acc[j] = 0.0;
#pragma unroll
    for (int k = 0; k < RP; ++k) {
#pragma unroll
      for (int j = 0; j < CH; ++j) acc[j] = fmad(MT[k * RP + l0 + j], x[k], acc[j]);
    }
#pragma unroll
    for (int j = 0; j < CH; ++j)
      if (l0 + j < r) y[(l0 + j) * ld] = acc[j];
  }
}

}  // namespace xca
