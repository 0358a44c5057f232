// Single-particle Green's function backbones on the device (plain FP64 path).
//
// DiagramEvaluator::compute_single_ptcle_gf (c++/triqs_xca/block_sparse_backbone.cpp:779-821) sums, over
// the flat indices of a CorrelatorBackbone (c++/triqs_xca/backbone.cpp:239-292), eval_correlator
// (block_sparse_backbone.cpp:528-706):
//   right chains  (vertices 1 .. vct0-1 on [0, tau]): T = G_b, then vertex, edge, ... (multiply_left_vertex,
//                 integrate_left_edge), scaled by the prefactor and its sign;
//   left chains   (vertices 2m-1 .. vct0+1 on [tau, beta]): U = G, then vertex, edge, ... from the right
//                 (multiply_right_vertex, integrate_right_edge, :463-515), then U <- reflect(U) (:648);
//   contraction   g(t)[mu][ka] += Tr[L(t) F_mu R(t) F^dag_ka] over the blocks that close the trace.
// Everything that does not depend on the pole tuple (directions, orbitals, block paths, which chains
// close a trace) is a correlator class built on the host; a warp evaluates the pole tuples of a class
// one at a time, its lanes striding over matrix entries and register-resident columns, with per-warp
// scratch in global memory.  Every product and sum is rounded as in the CPU restatement.
#pragma once
#include "sigma_kernel.cuh"

namespace xca {

struct CorrChain {
  int gblock;               // block of G the chain starts from
  int start;                // right: ind_path[0]; left: ind_path[vct0]
  int path[MAXV];           // ind_path entries of the chain's segment (-1 elsewhere)
  int bd[MAXV + 1];         // block_dims entries of the chain's segment
  int rows, cols;           // result per tau: right R x d1, left nrow x C
};

struct CorrTerm {
  int mu, ka;               // orbitals of F_mu (at vct0) and F^dag_ka (at 0)
  int rchain, lchain;       // chain indices within the class (right, left)
  int e0, e2;               // column blocks of F_mu and F^dag_ka
  int c0, c1, c2, c3;       // dims: right cols, right rows, F_mu rows, left rows
};

struct CorrClass {
  int m, vct0, fbmask;      // fbmask bit i (i >= 1): line i forward
  int la[MAXM], lb[MAXM];
  int vkind[MAXV], vset[MAXV], vqo[MAXV], vline[MAXV];
  int chain0, n_right, n_left;  // chains [chain0, chain0 + n_right) right, then n_left left
  int term0, n_terms;
};

struct CorrBasis {
  const double *RFp;        // RP x RP column-major: K(t_i, -om_l) (reflect), 0 in the pad
  const double *ops;        // slabs of the external operators (the evaluator's F / F^dag slabs for g(tau))
  const long *mu_off;       // [mu * nb + b]: offset of O_mu's (d_target x d_b) slab in ops (-1: none)
  const long *ka_off;       // [ka * nb + b]: offset of O'_ka's slab in ops (-1: none)
  int nmu, nka;             // operators at tau and at 0 (the result is r x nmu x nka)
};

// Per-item pole data, decoded as Backbone::set_pole_inds (c++/triqs_xca/backbone.cpp:86-150).
struct CorrItem {
  int lpole[MAXM];
  int caseA[MAXM];
  double scale;             // prefactor * prefactor sign
};

__device__ __forceinline__ CorrItem corr_decode(const DevBasis &B, const CorrClass &C, int q) {
  CorrItem S;
  const int m = C.m, p = B.p;
  for (int i = 0; i < MAXM; ++i) { S.lpole[i] = 0; S.caseA[i] = 0; }
  for (int i = 1; i < m; ++i) {
    S.lpole[i] = q % p;
    q /= p;
  }
  double pf = 1.0;
  int psign = 1;
  for (int i = 1; i < m; ++i) {
    const int fwd = (C.fbmask >> i) & 1;
    const double w = B.polesb[S.lpole[i]];
    S.caseA[i] = fwd ? (w <= 0.0) : (w >= 0.0);
    if (!fwd) psign = -psign;
    const int row = S.caseA[i] ? (fwd ? 1 : 0) : (fwd ? 0 : 1);
    const int ex = S.caseA[i] ? 1 : C.lb[i] - C.la[i] - 1;
    if (ex != 0) pf = mul(pf, B.kpow[((size_t)row * p + S.lpole[i]) * (MAXE + 1) + ex]);
  }
  S.scale = mul(pf, (double)psign);
  return S;
}

// Operator slab of vertex v acting on block b, and the K-factor table of the vertex (nullptr: none).
// right = true selects the sign convention of multiply_right_vertex (block_sparse_backbone.cpp:488-495).
__device__ __forceinline__ const double *corr_vertex_op(const DevBasis &B, const CorrClass &C, const CorrItem &S, int v, int b,
                                                        int dvp, int dv, bool right, const double **ktab, int *kcol) {
  const int line = C.vline[v], s = C.vset[v], qo = C.vqo[v], p = B.p;
  const int l = S.lpole[line];
  long off;
  switch (C.vkind[v]) {
    case 0: off = B.F_off[s * B.nb + b] + (long)qo * dvp * dv; break;
    case 1: off = B.Fd_off[s * B.nb + b] + (long)qo * dvp * dv; break;
    case 2: off = B.Fb_off[s * B.nb + b] + ((long)qo * p + l) * dvp * dv; break;
    default: off = B.Fdb_off[s * B.nb + b] + ((long)qo * p + l) * dvp * dv; break;
  }
  *ktab = nullptr;
  *kcol = 0;
  if (line > 0 && S.caseA[line]) {
    const int fwd = (C.fbmask >> line) & 1;
    const int ks = (v == C.la[line]) ? (fwd ? -1 : 1) : (fwd ? 1 : -1);
    const bool neg = right ? (ks > 0) : (ks < 0);
    *ktab = neg ? B.kitm : B.kitp;
    *kcol = l;
  }
  return B.ops + off;
}

// Edge-table offset of edge e of block b (fc = K^-1 (G_b prod K), then W fc).
__device__ __forceinline__ long corr_edge_tab(const DevBasis &B, const CorrClass &C, const CorrItem &S, int e, int b, int dd) {
  const int m = C.m, p = B.p, r = B.r;
  int nf = 0, sg[2] = {0, 0}, lp[2] = {0, 0};
  for (int i = 1; i < m; ++i)
    if (!S.caseA[i] && e >= C.la[i] && e < C.lb[i]) {
      sg[nf] = ((C.fbmask >> i) & 1) ? 0 : 1;
      lp[nf] = S.lpole[i];
      nf++;
    }
  long sig = 0;
  if (nf == 1) sig = 1 + (long)sg[0] * p + lp[0];
  if (nf == 2) sig = 1 + 2L * p + ((long)sg[0] * p + lp[0]) * 2 * p + (long)sg[1] * p + lp[1];
  return B.tab_off[b] + sig * 2 * r * dd;
}

// Barrier of the threads that share one item: the warp (CTA = false) or the whole CTA.
template <bool CTA>
__device__ __forceinline__ void item_sync() {
  if (CTA)
    __syncthreads();
  else
    __syncwarp();
}

// Time-ordered DLR convolution of one edge for one item, in place in T (r x rows x cols), X and Y scratch,
// by the `nt` threads of a warp (CTA = false, lane = thread index) or of a CTA (CTA = true).
// LEFT: T <- conv(GK, T) with GK (d x d) = table, T (d x cols) (integrate_left_edge);
// RIGHT: T <- conv(T, GK) with T (rows x d) (integrate_right_edge).  The table holds fc = K^-1 GK and W fc.
template <int RP, bool LEFT, bool CTA = false>
__device__ __forceinline__ void corr_edge(const DevBasis &B, const double *sLU, const double *sW, const double *sBK, const int *sPerm,
                                          const double *tb, int rows, int cols, int d, double *T, double *X, double *Y, int lane,
                                          int nt = 32) {
  const int r = B.r, dc = rows * cols, dd = d * d;
  // (a) coefficients of T (in place) and their Hilbert transform W Tc (into X), one column per lane
  for (int col = lane; col < dc; col += nt) {
    double x[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) {
      const int src = sPerm[i];
      x[i] = src >= 0 ? T[src * dc + col] : 0.0;
    }
    lu_solve_reg<RP>(sLU, x);
#pragma unroll
    for (int i = 0; i < RP; ++i)
      if (i < r) T[i * dc + col] = x[i];
    matvec_reg<RP>(sW, x, r, X + col, dc);
  }
  item_sync<CTA>();
  const double *fc = tb, *fw = tb + (long)r * dd;
  // (b) Q_l (into Y); the CTA form of a left edge runs the products on the FP64 tensor cores (the same
  // chains: k' = 2y takes f gt, k' = 2y + 1 takes Wf g)
  if constexpr (CTA && LEFT) {
    const double *fc0 = tb, *fw0 = tb + (long)r * dd, *Tc = T, *Xc = X;
    warp_gemm_dmma(
        r, rows, cols, 2 * d,
        [&](int l, int x, int k) { return ((k & 1) ? fw0 : fc0)[(long)l * dd + x * d + (k >> 1)]; },
        [&](int l, int k, int z) { return ((k & 1) ? Tc : Xc)[(long)l * dc + (k >> 1) * cols + z]; },
        [&](int l, int x, int z, double a) { Y[(long)l * dc + x * cols + z] = a; }, lane >> 5, nt >> 5);
  } else
  for (int idx = lane; idx < r * dc; idx += nt) {
    const int l = idx / dc, rem = idx - l * dc, x = rem / cols, z = rem - x * cols;
    double a = 0.0;
    if (LEFT) {
      // f = table (d x d), g = T coefficients (d x cols): fma(Wf, g, fma(f, Wg, a))
      const double *f = fc + l * dd, *ft = fw + l * dd, *g = T + l * dc, *gt = X + l * dc;
      for (int y = 0; y < d; ++y) a = fmad(ft[x * d + y], g[y * cols + z], fmad(f[x * d + y], gt[y * cols + z], a));
    } else {
      // f = T coefficients (rows x d), g = table (d x d)
      const double *f = T + l * dc, *ft = X + l * dc, *g = fc + l * dd, *gt = fw + l * dd;
      for (int y = 0; y < d; ++y) a = fmad(ft[x * d + y], g[y * d + z], fmad(f[x * d + y], gt[y * d + z], a));
    }
    Y[idx] = a;
  }
  item_sync<CTA>();
  // (c) h1 = (beta K) Q (into X)
  for (int col = lane; col < dc; col += nt) {
    double q[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) q[i] = i < r ? Y[i * dc + col] : 0.0;
    matvec_reg<RP>(sBK, q, r, X + col, dc);
  }
  item_sync<CTA>();
  // (d) P'_l = K(0, om_l) (f_l g_l) (into Y)
  if constexpr (CTA && LEFT) {
    const double *fc0 = tb, *Tc = T;
    warp_gemm_dmma(
        r, rows, cols, d, [&](int l, int x, int y) { return fc0[(long)l * dd + x * d + y]; },
        [&](int l, int y, int z) { return Tc[(long)l * dc + y * cols + z]; },
        [&](int l, int x, int z, double a) { Y[(long)l * dc + x * cols + z] = mul(B.k0[l], a); }, lane >> 5, nt >> 5);
  } else
  for (int idx = lane; idx < r * dc; idx += nt) {
    const int l = idx / dc, rem = idx - l * dc, x = rem / cols, z = rem - x * cols;
    double a = 0.0;
    if (LEFT) {
      const double *f = fc + l * dd, *g = T + l * dc;
      for (int y = 0; y < d; ++y) a = fmad(f[x * d + y], g[y * cols + z], a);
    } else {
      const double *f = T + l * dc, *g = fc + l * dd;
      for (int y = 0; y < d; ++y) a = fmad(f[x * d + y], g[y * d + z], a);
    }
    Y[idx] = mul(B.k0[l], a);
  }
  item_sync<CTA>();
  // (e) h = h1 + t_i (beta K) P' (into T)
  for (int col = lane; col < dc; col += nt) {
    double q[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) q[i] = i < r ? Y[i * dc + col] : 0.0;
    constexpr int CH = 8;
#pragma unroll 1
    for (int l0 = 0; l0 < RP; l0 += CH) {
      if (l0 >= r) break;
      double a[CH];
#pragma unroll
      for (int jj = 0; jj < CH; ++jj) a[jj] = 0.0;
#pragma unroll
      for (int k = 0; k < RP; ++k) {
#pragma unroll
        for (int jj = 0; jj < CH; ++jj) a[jj] = fmad(sBK[k * RP + l0 + jj], q[k], a[jj]);
      }
#pragma unroll
      for (int jj = 0; jj < CH; ++jj) {
        const int i = l0 + jj;
        if (i < r) T[i * dc + col] = fmad(B.tabs[i], a[jj], X[i * dc + col]);
      }
    }
  }
  item_sync<CTA>();
}

// Dynamic shared memory: LU (+ reciprocal diagonal) | W | BK | RF (column-major) | perm (RP ints).
// Per-warp global scratch (`warp_doubles` each): T | X | Y (r * nmax^2 each), right chains and left chains
// (nb slots of r * nmax^2 each), accumulator (r * nmu * nka).
template <int RP>
__global__ void __launch_bounds__(128) correlator_kernel(DevBasis B, CorrBasis CB, const CorrClass *__restrict__ classes,
                                                         const CorrChain *__restrict__ chains, const CorrTerm *__restrict__ terms,
                                                         const WorkUnit *__restrict__ units, int n_units, int *__restrict__ unit_counter,
                                                         const double *__restrict__ G, double *__restrict__ gout, double scale,
                                                         int nmax, double *__restrict__ scratch, long warp_doubles) {
  extern __shared__ __align__(16) double smem[];
  double *sLU = smem, *sW = sLU + RP * RP + RP, *sBK = sW + RP * RP, *sRF = sBK + RP * RP;
  int *sPerm = reinterpret_cast<int *>(sRF + RP * RP);
  for (int i = threadIdx.x; i < RP * RP + RP; i += blockDim.x) sLU[i] = B.LUp[i];
  for (int i = threadIdx.x; i < RP * RP; i += blockDim.x) {
    sW[i] = B.Wp[i];
    sBK[i] = B.BKp[i];
    sRF[i] = CB.RFp[i];
  }
  for (int i = threadIdx.x; i < RP; i += blockDim.x) sPerm[i] = B.perm[i];
  __syncthreads();
  const int r = B.r, nb = B.nb, nmu = CB.nmu, nka = CB.nka;
  const int lane = threadIdx.x & 31;
  const long gw = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long slab = (long)r * nmax * nmax;
  double *wb = scratch + gw * warp_doubles;
  double *T = wb, *X = wb + slab, *Y = wb + 2 * slab;
  double *Rs = wb + 3 * slab, *Ls = Rs + (long)nb * slab;
  double *acc = Ls + (long)nb * slab;
  for (int i = lane; i < r * nmu * nka; i += 32) acc[i] = 0.0;
  __syncwarp();
  bool any = false;
  while (true) {
    int u = 0;
    if (lane == 0) u = atomicAdd(unit_counter, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= n_units) break;
    const WorkUnit wu = units[u];
    const CorrClass &C = classes[wu.cls];
    const int m = C.m, vct0 = C.vct0;
    any = true;
    for (int it = 0; it < wu.count; ++it) {
      const CorrItem S = corr_decode(B, C, wu.first + it);
      // ---- right chains
      for (int j = 0; j < C.n_right; ++j) {
        const CorrChain &H = chains[C.chain0 + j];
        const int d1 = H.bd[1];
        const double *g = G + B.goff[H.gblock];
        for (int i = lane; i < r * d1 * d1; i += 32) T[i] = g[i];
        __syncwarp();
        for (int v = 1; v < vct0; ++v) {
          const int b = H.path[v - 1], dv = H.bd[v], dvp = H.bd[v + 1];
          const double *ktab;
          int kcol;
          const double *F = corr_vertex_op(B, C, S, v, b, dvp, dv, false, &ktab, &kcol);
          const int per = r * dvp * d1;
          for (int idx = lane; idx < per; idx += 32) {
            const int t = idx / (dvp * d1), rem = idx - t * dvp * d1, x = rem / d1, z = rem - x * d1;
            const double *Tt = T + t * dv * d1;
            double a = 0.0;
            for (int y = 0; y < dv; ++y) a = fmad(F[x * dv + y], Tt[y * d1 + z], a);
            if (ktab) a = mul(a, ktab[(size_t)t * B.p + kcol]);
            X[idx] = a;
          }
          __syncwarp();
          for (int idx = lane; idx < per; idx += 32) T[idx] = X[idx];
          __syncwarp();
          const int eb = H.path[v], d = H.bd[v + 1];
          corr_edge<RP, true>(B, sLU, sW, sBK, sPerm, B.tab + corr_edge_tab(B, C, S, v, eb, d * d), d, d1, d, T, X, Y, lane);
        }
        double *R = Rs + (long)j * slab;
        for (int i = lane; i < r * H.rows * H.cols; i += 32) R[i] = mul(T[i], S.scale);
        __syncwarp();
      }
      // ---- left chains
      for (int j = 0; j < C.n_left; ++j) {
        const CorrChain &H = chains[C.chain0 + C.n_right + j];
        const int nrow = H.bd[2 * m];
        const double *g = G + B.goff[H.gblock];
        for (int i = lane; i < r * nrow * nrow; i += 32) T[i] = g[i];
        __syncwarp();
        for (int v = 2 * m - 1; v > vct0; --v) {
          // U(t) <- U(t) F (nrow x bd(v+1)) (bd(v+1) x bd(v)), K factor
          const int b = H.path[v - 1], K = H.bd[v], Rr = H.bd[v + 1];
          const double *ktab;
          int kcol;
          const double *F = corr_vertex_op(B, C, S, v, b, Rr, K, true, &ktab, &kcol);
          const int per = r * nrow * K;
          for (int idx = lane; idx < per; idx += 32) {
            const int t = idx / (nrow * K), rem = idx - t * nrow * K, x = rem / K, z = rem - x * K;
            const double *Ut = T + t * nrow * Rr;
            double a = 0.0;
            for (int y = 0; y < Rr; ++y) a = fmad(Ut[x * Rr + y], F[y * K + z], a);
            if (ktab) a = mul(a, ktab[(size_t)t * B.p + kcol]);
            X[idx] = a;
          }
          __syncwarp();
          for (int idx = lane; idx < per; idx += 32) T[idx] = X[idx];
          __syncwarp();
          const int eb = H.path[v - 1], d = H.bd[v];
          corr_edge<RP, false>(B, sLU, sW, sBK, sPerm, B.tab + corr_edge_tab(B, C, S, v - 1, eb, d * d), nrow, d, d, T, X, Y, lane);
        }
        // L = reflect(U): K(t_i, -om_l) K^-1 U, one column per lane
        const int dc = H.rows * H.cols;
        double *L = Ls + (long)j * slab;
        for (int col = lane; col < dc; col += 32) {
          double x[RP];
#pragma unroll
          for (int i = 0; i < RP; ++i) {
            const int src = sPerm[i];
            x[i] = src >= 0 ? T[src * dc + col] : 0.0;
          }
          lu_solve_reg<RP>(sLU, x);
          matvec_reg<RP>(sRF, x, r, L + col, dc);
        }
        __syncwarp();
      }
      // ---- trace contraction g(t)[mu][ka] += sum Tr[L F_mu R F^dag_ka]: per node t, s = sum_{i, j ascending}
      // fma(tm_ij, Ok_ji, s) with tm_ij = sum_k L_ik tp_kj and tp_kj = sum_q Om_kq R_qj (fused multiply-adds
      // from zero, inner index ascending).  Two forms with the same values: one lane per node forming every
      // tp_kj again for each i (c3 c0 c2 (c1 + 1) dependent operations per node; faster when c0 c1 c2 c3 <= 64,
      // as for the two-orbital blocks of dimension <= 4), or tp (r x c2 x c0, into X) and tm (r x c3 x c0,
      // into Y) formed once per term by all lanes (faster from the 3 x 3 and 9 x 9 blocks of three orbitals
      // on, measured; T, X and Y are free once the chains are stored).
      for (int k = 0; k < C.n_terms; ++k) {
        const CorrTerm &P = terms[C.term0 + k];
        const double *R = Rs + (long)P.rchain * slab;
        const double *L = Ls + (long)P.lchain * slab;
        const double *Om = CB.ops + CB.mu_off[P.mu * nb + P.e0];  // (c2 x c1)
        const double *Ok = CB.ops + CB.ka_off[P.ka * nb + P.e2];  // (c0 x c3)
        const int c0 = P.c0, c1 = P.c1, c2 = P.c2, c3 = P.c3;
        if (c0 * c1 * c2 * c3 <= 64) {
          for (int t = lane; t < r; t += 32) {
            const double *Rt = R + (long)t * c1 * c0, *Lt = L + (long)t * c3 * c2;
            double s = 0.0;
            for (int i = 0; i < c3; ++i)
              for (int jj = 0; jj < c0; ++jj) {
                double tm = 0.0;
                for (int kk = 0; kk < c2; ++kk) {
                  double tp = 0.0;
                  for (int q = 0; q < c1; ++q) tp = fmad(Om[kk * c1 + q], Rt[q * c0 + jj], tp);
                  tm = fmad(Lt[i * c2 + kk], tp, tm);
                }
                s = fmad(tm, Ok[jj * c3 + i], s);
              }
            double *a = acc + ((long)t * nmu + P.mu) * nka + P.ka;
            *a = add(*a, s);
          }
          __syncwarp();
          continue;
        }
        for (int idx = lane; idx < r * c2 * c0; idx += 32) {
          const int t = idx / (c2 * c0), rem = idx - t * c2 * c0, kk = rem / c0, jj = rem - kk * c0;
          const double *Rt = R + (long)t * c1 * c0;
          double tp = 0.0;
          for (int q = 0; q < c1; ++q) tp = fmad(Om[kk * c1 + q], Rt[q * c0 + jj], tp);
          X[idx] = tp;
        }
        __syncwarp();
        for (int idx = lane; idx < r * c3 * c0; idx += 32) {
          const int t = idx / (c3 * c0), rem = idx - t * c3 * c0, i = rem / c0, jj = rem - i * c0;
          const double *Lt = L + (long)t * c3 * c2, *tpt = X + (long)t * c2 * c0;
          double tm = 0.0;
          for (int kk = 0; kk < c2; ++kk) tm = fmad(Lt[i * c2 + kk], tpt[kk * c0 + jj], tm);
          Y[idx] = tm;
        }
        __syncwarp();
        for (int t = lane; t < r; t += 32) {
          const double *tmt = Y + (long)t * c3 * c0;
          double s = 0.0;
          for (int i = 0; i < c3; ++i)
            for (int jj = 0; jj < c0; ++jj) s = fmad(tmt[i * c0 + jj], Ok[jj * c3 + i], s);
          double *a = acc + ((long)t * nmu + P.mu) * nka + P.ka;
          *a = add(*a, s);
        }
        __syncwarp();
      }
    }
  }
  if (any)
    for (int i = lane; i < r * nmu * nka; i += 32) atomicAdd(gout + i, mul(scale, acc[i]));
}

}  // namespace xca
