// Sigma backbone evaluation on the device, panel form (plain FP64 path).
//
// A CTA of PANEL_THREADS threads takes a run of pole tuples of one path class (work unit) and evaluates
// `batch` of them together.  The T slabs of the batch's items sit side by side as the columns of a
// shared-memory panel (RP rows = tau nodes, NC columns = item x matrix entry), so every r x r DLR
// operator of an edge acts on all of them at once:
//   K^-1 T     blocked substitution by the whole CTA (8-row blocks: register-tiled rectangular updates,
//              then the in-block solve), every element in dtrsm order;
//   W gc, (beta K) Q and (beta K) P'   register-tiled products (TR x TC outputs per thread, operand pairs
//                                   loaded as double2 from shared memory; the last two in one pass),
//                                   each output one chain of fused multiply-adds over k ascending from zero;
// and the per-item steps (vertex products with the item's operator and K factor, Q and P' with the
// item's edge table, the zero vertex) run with the threads striding over panel entries.  Every element
// sees exactly the operations, in the same order, as in the CPU restatement, so each item's contribution
// is bit-identical to it (sigma_kernel.cuh documents the item arithmetic and its reference lines).
#pragma once
#include "sigma_kernel.cuh"

namespace xca {

constexpr int PANEL_THREADS = 256;
constexpr int PANEL_BMAX = 128;  // items per batch at most

template <int RP>
struct PanelCfg;
template <>
struct PanelCfg<32> { static constexpr int NC = 192, TR = 4, TC = 6; };
template <>
struct PanelCfg<48> { static constexpr int NC = 128, TR = 6, TC = 4; };
template <>
struct PanelCfg<64> { static constexpr int NC = 64, TR = 4, TC = 4; };

template <int RP>
__host__ __device__ constexpr int panel_nc() { return PanelCfg<RP>::NC; }

// Dynamic shared memory of the panel kernels, in doubles.
template <int RP>
__host__ __device__ constexpr size_t panel_smem_doubles() {
  return 3 * (size_t)RP * RP + RP + 3 * (size_t)RP * PanelCfg<RP>::NC + (sizeof(ItemState) * PANEL_BMAX + 7) / 8 + RP;
}

// A thread group of NT threads working on a panel of NCG columns (row stride NCG).
template <int RP, int G>
struct PanelGrp {
  static constexpr int NT = PANEL_THREADS / G, NCG = PanelCfg<RP>::NC / G;
  static constexpr int TR = PanelCfg<RP>::TR, TC = PanelCfg<RP>::TC, CT = NCG / TC;
  static_assert((RP / TR) * CT == NT, "panel tiling must cover the thread group");
};

// Barrier of thread group g (named barrier 1 + g of NT threads; the whole CTA when G == 1).
template <int G>
__device__ __forceinline__ void group_sync(int g) {
  if (G == 1)
    __syncthreads();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(PANEL_THREADS / G) : "memory");
}

// Y[i][c] = sum_{k < r} M[i][k] X[k][c] for i < r, c < ncols (M column-major RP x RP; X, Y panels with row
// stride NCG); t is the thread's index in its group.  EPI: Y[i][c] = fma(t_i, (M X)[i][c], H1[i][c]).
// Each thread owns TR rows x TC columns: the column pairs 2 (ct + q CT) .. + 1 (q < TC / 2), so that
// neighbouring lanes read consecutive 16-byte pairs of a panel row (no bank conflict); lanes that share
// a row tile read the same M operands (broadcasts).
template <int RP, int G, bool EPI>
__device__ __forceinline__ void panel_gemm(const double *__restrict__ sM, const double *__restrict__ X, double *__restrict__ Y, int r,
                                           int ncols, const double *__restrict__ tabs, const double *__restrict__ H1, int t) {
  using P = PanelGrp<RP, G>;
  constexpr int NCG = P::NCG, TR = P::TR, TC = P::TC, CT = P::CT;
  const int rt = t / CT, ct = t - rt * CT;
  const int i0 = rt * TR;
  if (i0 >= r || 2 * ct >= ncols) return;
  double acc[TR][TC];
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) acc[a][b] = 0.0;
#pragma unroll 2
  for (int k = 0; k < r; ++k) {
    double mv[TR], xv[TC];
    const double2 *mp = reinterpret_cast<const double2 *>(sM + k * RP + i0);
#pragma unroll
    for (int a = 0; a < TR / 2; ++a) {
      const double2 v = mp[a];
      mv[2 * a] = v.x;
      mv[2 * a + 1] = v.y;
    }
#pragma unroll
    for (int q = 0; q < TC / 2; ++q) {
      const double2 v = *reinterpret_cast<const double2 *>(X + k * NCG + 2 * (ct + q * CT));
      xv[2 * q] = v.x;
      xv[2 * q + 1] = v.y;
    }
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) acc[a][b] = fmad(mv[a], xv[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < TR; ++a) {
    const int i = i0 + a;
    if (i >= r) break;
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      const int c = 2 * (ct + (b / 2) * CT) + (b & 1);
      if (c < ncols) Y[i * NCG + c] = EPI ? fmad(tabs[i], acc[a][b], H1[i * NCG + c]) : acc[a][b];
    }
  }
}

// Y[i][c] = fma(t_i, (M X2)[i][c], (M X1)[i][c]) for i < r, c < ncols: the two products of one operand M
// in one pass (each accumulator one fused multiply-add chain over k ascending from zero), tiled as
// panel_gemm.
template <int RP, int G>
__device__ __forceinline__ void panel_gemm2(const double *__restrict__ sM, const double *__restrict__ X1, const double *__restrict__ X2,
                                            double *__restrict__ Y, int r, int ncols, const double *__restrict__ tabs, int t) {
  using P = PanelGrp<RP, G>;
  constexpr int NCG = P::NCG, TR = P::TR, TC = P::TC, CT = P::CT;
  const int rt = t / CT, ct = t - rt * CT;
  const int i0 = rt * TR;
  if (i0 >= r || 2 * ct >= ncols) return;
  double a1[TR][TC], a2[TR][TC];
#pragma unroll
  for (int a = 0; a < TR; ++a)
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      a1[a][b] = 0.0;
      a2[a][b] = 0.0;
    }
#pragma unroll 1
  for (int k = 0; k < r; ++k) {
    double mv[TR], xv[TC], yv[TC];
    const double2 *mp = reinterpret_cast<const double2 *>(sM + k * RP + i0);
#pragma unroll
    for (int a = 0; a < TR / 2; ++a) {
      const double2 v = mp[a];
      mv[2 * a] = v.x;
      mv[2 * a + 1] = v.y;
    }
#pragma unroll
    for (int q = 0; q < TC / 2; ++q) {
      const double2 v = *reinterpret_cast<const double2 *>(X1 + k * NCG + 2 * (ct + q * CT));
      const double2 w = *reinterpret_cast<const double2 *>(X2 + k * NCG + 2 * (ct + q * CT));
      xv[2 * q] = v.x;
      xv[2 * q + 1] = v.y;
      yv[2 * q] = w.x;
      yv[2 * q + 1] = w.y;
    }
#pragma unroll
    for (int a = 0; a < TR; ++a)
#pragma unroll
      for (int b = 0; b < TC; ++b) {
        a1[a][b] = fmad(mv[a], xv[b], a1[a][b]);
        a2[a][b] = fmad(mv[a], yv[b], a2[a][b]);
      }
  }
#pragma unroll
  for (int a = 0; a < TR; ++a) {
    const int i = i0 + a;
    if (i >= r) break;
#pragma unroll
    for (int b = 0; b < TC; ++b) {
      const int c = 2 * (ct + (b / 2) * CT) + (b & 1);
      if (c < ncols) Y[i * NCG + c] = fmad(tabs[i], a2[a][b], a1[a][b]);
    }
  }
}

// P[:, c] <- K^-1 P[:, c] for c < nc on a panel whose rows are already in pivot order (row i holds the
// original row perm[i]), by the whole thread group: 8-row blocks, each a rectangular update (every thread
// a 2 x 2 tile, operand pairs as double2) followed by the in-block substitution (one thread per column).
// Every element receives exactly the fused multiply-adds of lu_solve_reg in the same order — forward
// k ascending, backward k descending with the reciprocal diagonal applied at k = i — so the result is
// bit-identical to it; rows r .. RP-1 (padding) are neither read nor written.
template <int RP, int NCG, int NT, int NG>
__device__ __forceinline__ void panel_trsm(const double *__restrict__ sLU, double *P, int r, int nc, int t, int g) {
  const int nblk = (r + 7) >> 3, ncp = (nc + 1) >> 1;
  for (int J = 0; J < nblk; ++J) {
    const int j0 = J << 3, j1 = min(r, j0 + 8);
    if (J > 0) {
      const int nrp = (j1 - j0 + 1) >> 1;
      for (int w = t; w < nrp * ncp; w += NT) {
        const int rp = w / ncp, c = 2 * (w - rp * ncp), i = j0 + 2 * rp;
        const bool two = i + 1 < j1;
        double2 a0 = *reinterpret_cast<const double2 *>(P + i * NCG + c);
        double2 a1 = two ? *reinterpret_cast<const double2 *>(P + (i + 1) * NCG + c) : make_double2(0.0, 0.0);
#pragma unroll 4
        for (int k = 0; k < j0; ++k) {
          const double2 l = *reinterpret_cast<const double2 *>(sLU + k * RP + i);  // L[i][k], L[i+1][k]
          const double2 x = *reinterpret_cast<const double2 *>(P + k * NCG + c);
          a0.x = fmad(-l.x, x.x, a0.x);
          a0.y = fmad(-l.x, x.y, a0.y);
          a1.x = fmad(-l.y, x.x, a1.x);
          a1.y = fmad(-l.y, x.y, a1.y);
        }
        *reinterpret_cast<double2 *>(P + i * NCG + c) = a0;
        if (two) *reinterpret_cast<double2 *>(P + (i + 1) * NCG + c) = a1;
      }
      group_sync<NG>(g);
    }
    for (int c = t; c < nc; c += NT) {
      double xb[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) xb[q] = (j0 + q < j1) ? P[(j0 + q) * NCG + c] : 0.0;
#pragma unroll
      for (int kk = 0; kk < 7; ++kk)
#pragma unroll
        for (int q = kk + 1; q < 8; ++q)
          if (j0 + q < j1) xb[q] = fmad(-sLU[(j0 + kk) * RP + j0 + q], xb[kk], xb[q]);
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (j0 + q < j1) P[(j0 + q) * NCG + c] = xb[q];
    }
    group_sync<NG>(g);
  }
  const double *dinv = sLU + RP * RP;
  for (int J = nblk - 1; J >= 0; --J) {
    const int j0 = J << 3, j1 = min(r, j0 + 8);
    if (j1 < r) {
      const int nrp = (j1 - j0 + 1) >> 1;
      for (int w = t; w < nrp * ncp; w += NT) {
        const int rp = w / ncp, c = 2 * (w - rp * ncp), i = j0 + 2 * rp;
        const bool two = i + 1 < j1;
        double2 a0 = *reinterpret_cast<const double2 *>(P + i * NCG + c);
        double2 a1 = two ? *reinterpret_cast<const double2 *>(P + (i + 1) * NCG + c) : make_double2(0.0, 0.0);
#pragma unroll 4
        for (int k = r - 1; k >= j1; --k) {
          const double2 u = *reinterpret_cast<const double2 *>(sLU + k * RP + i);  // U[i][k], U[i+1][k]
          const double2 x = *reinterpret_cast<const double2 *>(P + k * NCG + c);
          a0.x = fmad(-u.x, x.x, a0.x);
          a0.y = fmad(-u.x, x.y, a0.y);
          a1.x = fmad(-u.y, x.x, a1.x);
          a1.y = fmad(-u.y, x.y, a1.y);
        }
        *reinterpret_cast<double2 *>(P + i * NCG + c) = a0;
        if (two) *reinterpret_cast<double2 *>(P + (i + 1) * NCG + c) = a1;
      }
      group_sync<NG>(g);
    }
    for (int c = t; c < nc; c += NT) {
      double xb[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) xb[q] = (j0 + q < j1) ? P[(j0 + q) * NCG + c] : 0.0;
#pragma unroll
      for (int kk = 7; kk >= 0; --kk) {
        if (j0 + kk < j1) {
          xb[kk] = mul(xb[kk], dinv[j0 + kk]);
#pragma unroll
          for (int q = 0; q < kk; ++q) xb[q] = fmad(-sLU[(j0 + kk) * RP + j0 + q], xb[kk], xb[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
        if (j0 + q < j1) P[(j0 + q) * NCG + c] = xb[q];
    }
    group_sync<NG>(g);
  }
}

// Stage the DLR matrices; sPerm receives the pivot gather (RP ints) followed by its inverse (RP ints: the
// pivot-order position of tau node t, -1 in the pad).
template <int RP>
__device__ __forceinline__ void stage_basis(const DevBasis &B, double *sLU, double *sW, double *sBK, int *sPerm) {
  for (int i = threadIdx.x; i < RP * RP + RP; i += blockDim.x) sLU[i] = B.LUp[i];
  for (int i = threadIdx.x; i < RP * RP; i += blockDim.x) {
    sW[i] = B.Wp[i];
    sBK[i] = B.BKp[i];
  }
  for (int i = threadIdx.x; i < RP; i += blockDim.x) {
    sPerm[i] = B.perm[i];
    sPerm[RP + i] = B.pinv[i];
  }
  __syncthreads();
}

// Edge tables (see edge_table_kernel): for block b and signature sig, fc = K^-1 (G_b prod K) and W fc.
// A CTA takes NC consecutive (sig, entry) columns of one block: gather with the K factors, K^-1, write fc,
// W fc, write.  `chunks` lists (block, first column) pairs.
template <int RP>
__global__ void __launch_bounds__(PANEL_THREADS, 1) edge_tables_panel_kernel(DevBasis B, const double *__restrict__ G,
                                                                              const int2 *__restrict__ chunks, int n_chunks) {
  constexpr int NC = PanelCfg<RP>::NC;
  extern __shared__ double smem[];
  double *sLU = smem, *sW = sLU + RP * RP + RP, *sBK = sW + RP * RP;
  double *PA = sBK + RP * RP, *PB = PA + RP * NC;
  int *sPerm = reinterpret_cast<int *>(PB + RP * NC);
  stage_basis<RP>(B, sLU, sW, sBK, sPerm);
  const int r = B.r, p = B.p;
  for (int ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    const int b = chunks[ch].x, col0 = chunks[ch].y;
    const int d = B.dims[b], dd = d * d;
    const long total = (long)B.nsig * dd;
    const int ncols = (int)min((long)NC, total - col0);
    const double *g = G + B.goff[b];
    // gather: column c is (sig, e) = divmod(col0 + c, dd); rows are the tau nodes
    for (int idx = threadIdx.x; idx < r * ncols; idx += PANEL_THREADS) {
      const int t = idx / ncols, c = idx - t * ncols;
      const long q = col0 + c;
      const int sig = (int)(q / dd), e = (int)(q - (long)sig * dd);
      int nf = 0, s1 = 0, l1 = 0, s2 = 0, l2 = 0;
      if (sig >= 1 && sig < 1 + 2 * p) {
        nf = 1;
        s1 = (sig - 1) / p;
        l1 = (sig - 1) - s1 * p;
      } else if (sig >= 1 + 2 * p) {
        nf = 2;
        const int qq = sig - 1 - 2 * p;
        const int a = qq / (2 * p), cc = qq - a * (2 * p);
        s1 = a / p; l1 = a - s1 * p;
        s2 = cc / p; l2 = cc - s2 * p;
      }
      double v = g[t * dd + e];
      if (nf >= 1) v = mul(v, (s1 ? B.kitm : B.kitp)[(size_t)t * p + l1]);
      if (nf >= 2) v = mul(v, (s2 ? B.kitm : B.kitp)[(size_t)t * p + l2]);
      PA[sPerm[RP + t] * NC + c] = v;
    }
    __syncthreads();
    panel_trsm<RP, NC, PANEL_THREADS, 1>(sLU, PA, r, ncols, threadIdx.x, 0);
    panel_gemm<RP, 1, false>(sW, PA, PB, r, ncols, nullptr, nullptr, threadIdx.x);
    __syncthreads();
    double *out = const_cast<double *>(B.tab) + B.tab_off[b];
    for (int idx = threadIdx.x; idx < r * ncols; idx += PANEL_THREADS) {
      const int t = idx / ncols, c = idx - t * ncols;
      const long q = col0 + c;
      const long sig = q / dd, e = q - sig * dd;
      double *o = out + sig * 2 * r * dd;
      o[t * dd + e] = PA[t * NC + c];
      o[(long)r * dd + t * dd + e] = PB[t * NC + c];
    }
    __syncthreads();
  }
}

// Dynamic shared memory: LU (+ reciprocal diagonal) | W | BK (column-major) | per thread group: panels A, B,
// C (RP x NC / NG each) | per thread group: item states (PANEL_BMAX / NG) | perm (RP ints).  The NG thread
// groups of the CTA run independent work loops (own units, batches and barriers) over the shared DLR
// matrices, so that one group's substitution phase overlaps another group's products.
template <int RP, int NG>
__global__ void __launch_bounds__(PANEL_THREADS, 1) sigma_panel_kernel(DevBasis B, const ClassRec *__restrict__ classes,
                                                                        const WorkUnit *__restrict__ units, int n_units,
                                                                        int *__restrict__ unit_counter, const double *__restrict__ G,
                                                                        double *__restrict__ Sigma, double scale) {
  using GP = PanelGrp<RP, NG>;
  constexpr int NC = GP::NCG, NT = GP::NT, BG = PANEL_BMAX / NG;
  extern __shared__ double smem[];
  double *sLU = smem, *sW = sLU + RP * RP + RP, *sBK = sW + RP * RP;
  const int g = threadIdx.x / NT, tid = threadIdx.x - g * NT;
  double *PA = sBK + RP * RP + (size_t)g * 3 * RP * NC, *PB = PA + RP * NC, *PC = PB + RP * NC;
  ItemState *ist = reinterpret_cast<ItemState *>(sBK + RP * RP + (size_t)3 * RP * NC * NG) + g * BG;
  int *sPerm = reinterpret_cast<int *>(sBK + RP * RP + (size_t)3 * RP * NC * NG + (sizeof(ItemState) * PANEL_BMAX + 7) / 8);
  __shared__ int s_unit_all[NG];
  __shared__ unsigned long long s_max_all[PANEL_BMAX];
  int &s_unit = s_unit_all[g];
  unsigned long long *s_max = s_max_all + g * BG;
  stage_basis<RP>(B, sLU, sW, sBK, sPerm);
  const int r = B.r, p = B.p, n = B.n;

  while (true) {
    if (tid == 0) s_unit = atomicAdd(unit_counter, 1);
    group_sync<NG>(g);
    const int u = s_unit;
    group_sync<NG>(g);
    if (u >= n_units) break;
    const WorkUnit wu = units[u];
    const ClassRec &C = classes[wu.cls];
    const int m = C.m, vct0 = C.vct0;
    const int d0 = C.bdims[0], d1 = C.bdims[1];
    const int dout = C.bdims[2 * m];
    const int cap = C.batch;
    const int nops = 4 * m - 3;

    for (int first = 0; first < wu.count; first += cap) {
      const int nbi = min(cap, wu.count - first);
      // ---- decode the pole tuples (Backbone::set_pole_inds, backbone.cpp:86-150)
      if (tid < nbi) {
        ItemState &S = ist[tid];
        int q = wu.first + first + tid;
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
        int dsign = (m % 2 == 0) ? -1 : 1;
        if (!(C.fbmask & 1)) dsign = -dsign;
        S.scale = mul(pf, (double)(psign * dsign));
        s_max[tid] = 0ull;
      }
      double *T = PA, *X = PB, *Y = PC;
      // T := G[ind_path[0]] (d1 x d1) for every item
      {
        const double *g = G + B.goff[C.ind_path[0]];
        const int dc = d1 * d1, nc = nbi * dc, tpc = NT / nc, c = tid % nc, t0 = tid / nc;
        if (t0 < tpc) {
          const int e = c % dc;
          for (int t = t0; t < r; t += tpc) T[t * NC + c] = g[t * dc + e];
        }
      }
      group_sync<NG>(g);

      // op order: for v < vct0: vertex v, edge v; zero vertex; for v > vct0: edge v - 1, vertex v
      const int pre = 2 * (vct0 - 1);
      auto op_kind = [&](int o) -> int {
        if (o < pre) return (o & 1) ? 1 : 0;
        if (o == pre) return 2;
        return ((o - pre - 1) & 1) ? 0 : 1;
      };
      for (int op = 0; op < nops; ++op) {
        int v;
        const int kind = op_kind(op);
        if (op < pre) v = 1 + op / 2;
        else if (op == pre) v = vct0;
        else v = vct0 + 1 + (op - pre - 1) / 2;
        const int ncol = v < vct0 ? d1 : d0;
        // a vertex feeding an edge writes its rows in pivot order (the order the substitution works in)
        const int *rowpos = (op + 1 < nops && op_kind(op + 1) == 1) ? sPerm + RP : nullptr;

        if (kind == 0) {
          // ---- vertex v: T(t) <- k(t) F T(t)  (multiply_left_vertex)
          const int line = C.vline[v];
          const int b = C.ind_path[v - 1];
          const int dv = C.bdims[v], dvp = C.bdims[v + 1];
          const int s = C.vset[v], qo = C.vqo[v];
          if (tid < nbi) {
            ItemState &S = ist[tid];
            const int l = S.lpole[line];
            long off;
            switch (C.vkind[v]) {
              case 0: off = B.F_off[s * B.nb + b] + (long)qo * dvp * dv; break;
              case 1: off = B.Fd_off[s * B.nb + b] + (long)qo * dvp * dv; break;
              case 2: off = B.Fb_off[s * B.nb + b] + ((long)qo * p + l) * dvp * dv; break;
              default: off = B.Fdb_off[s * B.nb + b] + ((long)qo * p + l) * dvp * dv; break;
            }
            S.opoff = off;
            S.kcol = -1;
            if (line > 0 && S.caseA[line]) {
              const int fwd = (C.fbmask >> line) & 1;
              const int ks = (v == C.la[line]) ? (fwd ? -1 : 1) : (fwd ? 1 : -1);
              S.kcol = l;
              S.kneg = ks < 0;
            }
          }
          group_sync<NG>(g);
          const int dci = dv * ncol, dco = dvp * ncol, nc = nbi * dco, tpc = NT / nc, c = tid % nc, t0 = tid / nc;
          if (t0 < tpc) {
            const int j = c / dco, e = c - j * dco, x = e / ncol, z = e - x * ncol;
            const ItemState &S = ist[j];
            const double *F = B.ops + S.opoff + x * dv;
            const double *kt = S.kcol >= 0 ? (S.kneg ? B.kitm : B.kitp) + S.kcol : nullptr;
            const double *Tc = T + j * dci + z;
            for (int t = t0; t < r; t += tpc) {
              const double *Tt = Tc + t * NC;
              double a = 0.0;
              for (int y = 0; y < dv; ++y) a = fmad(F[y], Tt[y * ncol], a);
              if (kt) a = mul(a, kt[(size_t)t * p]);
              X[(rowpos ? rowpos[t] : t) * NC + c] = a;
            }
          }
          group_sync<NG>(g);
          double *tmp = T; T = X; X = tmp;
        } else if (kind == 1) {
          // ---- edge e: T <- conv(G_b prod K, T)  (integrate_left_edge, time-ordered convolution)
          const int e = v < vct0 ? v : v - 1;
          const int b = C.ind_path[e];
          const int d = C.bdims[e + 1];
          const int dd = d * d, dc = d * ncol, nc = nbi * dc;
          if (tid < nbi) {
            ItemState &S = ist[tid];
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
            S.taboff = B.tab_off[b] + sig * 2 * r * dd;
          }
          // (a) gc = K^-1 T (in place), then Gt = W gc (into X)
          panel_trsm<RP, NC, NT, NG>(sLU, T, r, nc, tid, g);
          panel_gemm<RP, NG, false>(sW, T, X, r, nc, nullptr, nullptr, tid);
          group_sync<NG>(g);
          // (b) per row l (one warp per row; Q and P' of row l read only row l of gc and Gt):
          //     Q_l = Ft_l gc_l + fc_l Gt_l (into Y) and P'_l = K(0, om_l) (fc_l gc_l) (over Gt, into X)
          {
            constexpr int CPL = (NC + 31) / 32;
            const int lane = tid & 31, warp = tid >> 5;
            const double *tbq[CPL];
            int coff[CPL];
            bool cval[CPL];
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
              const int c = lane + 32 * q;
              cval[q] = c < nc;
              const int cc = cval[q] ? c : 0;
              const int j = cc / dc, ee = cc - j * dc, x = ee / ncol, z = ee - x * ncol;
              tbq[q] = B.tab + ist[j].taboff + x * d;
              coff[q] = j * dc + z;
            }
            for (int l = warp; l < r; l += NT / 32) {
              double qv[CPL], pv[CPL];
#pragma unroll
              for (int q = 0; q < CPL; ++q) {
                double aq = 0.0, ap = 0.0;
                if (cval[q]) {
                  const double *fl = tbq[q] + l * dd, *ftl = tbq[q] + (long)r * dd + l * dd;
                  const double *gl = T + l * NC + coff[q], *gtl = X + l * NC + coff[q];
                  for (int y = 0; y < d; ++y) {
                    aq = fmad(ftl[y], gl[y * ncol], fmad(fl[y], gtl[y * ncol], aq));
                    ap = fmad(fl[y], gl[y * ncol], ap);
                  }
                }
                qv[q] = aq;
                pv[q] = mul(B.k0[l], ap);
              }
              __syncwarp();
#pragma unroll
              for (int q = 0; q < CPL; ++q)
                if (cval[q]) {
                  const int c = lane + 32 * q;
                  Y[l * NC + c] = qv[q];
                  X[l * NC + c] = pv[q];
                }
            }
          }
          group_sync<NG>(g);
          // (c) h = fma(t_i, (beta K) P', (beta K) Q) (into T; gc is no longer needed)
          panel_gemm2<RP, NG>(sBK, Y, X, T, r, nc, B.tabs, tid);
          group_sync<NG>(g);
        } else {
          // ---- zero vertex (multiply_left_vertex_and_right_zero_vertex)
          const int b_mu = C.ind_path[v - 1];
          const int dv = C.bdims[v], dvp = C.bdims[v + 1];
          const bool fwd = C.fbmask & 1;
          const int pk = C.pk;
          const long ok_off = fwd ? B.F_off[pk * B.nb + C.b_out] : B.Fd_off[pk * B.nb + C.b_out];
          const long om_off = fwd ? B.Fd_off[pk * B.nb + b_mu] : B.F_off[pk * B.nb + b_mu];
          const double hs = fwd ? 1.0 : -1.0;
          int qs = 0;
          for (int i = 0; i < n; ++i)
            if (B.set_to_orb[pk * n + i] >= 0) qs = i + 1;
          const int dci = dv * d1, dmid = dv * d0, dco = dvp * d0;
          const int ncm = nbi * dmid, nco = nbi * dco;
          const int tpo = NT / nco, co = tid % nco, to0 = tid / nco;
          const int tpm = NT / ncm, cm = tid % ncm, tm0 = tid / ncm;
          if (to0 < tpo)
            for (int t = to0; t < r; t += tpo) X[(rowpos ? rowpos[t] : t) * NC + co] = 0.0;
          group_sync<NG>(g);
          for (int mu = 0; mu < qs; ++mu) {
            const int om = B.set_to_orb[pk * n + mu];
            if (tm0 < tpm) {
              const int c = cm, j = c / dmid, ee = c - j * dmid, x = ee / d0, z = ee - x * d0;
              const double *Tc = T + j * dci + x * d1;
              for (int t = tm0; t < r; t += tpm) {
                const double *Tt = Tc + t * NC;
                double a = 0.0;
                for (int kap = 0; kap < qs; ++kap) {
                  const int ok = B.set_to_orb[pk * n + kap];
                  const double h = fwd ? B.hval[((size_t)t * n + om) * n + ok] : B.hrefl[((size_t)t * n + ok) * n + om];
                  if (h == 0.0) continue;
                  const double *Fk = B.ops + ok_off + (size_t)kap * d1 * d0 + z;
                  double tf = 0.0;
                  for (int y = 0; y < d1; ++y) tf = fmad(Tt[y], Fk[y * d0], tf);
                  a = fmad(mul(hs, h), tf, a);
                }
                Y[t * NC + c] = a;
              }
            }
            group_sync<NG>(g);
            const double *Fm = B.ops + om_off + (size_t)mu * dvp * dv;
            if (to0 < tpo) {
              const int c = co, j = c / dco, ee = c - j * dco, x = ee / d0, z = ee - x * d0;
              const double *Fx = Fm + x * dv, *Yc = Y + j * dmid + z;
              for (int t = to0; t < r; t += tpo) {
                const double *Yt = Yc + t * NC;
                double a = 0.0;
                for (int y = 0; y < dv; ++y) a = fmad(Fx[y], Yt[y * d0], a);
                const int row = rowpos ? rowpos[t] : t;
                X[row * NC + c] = add(X[row * NC + c], a);
              }
            }
            group_sync<NG>(g);
          }
          double *tmp = T; T = X; X = tmp;
        }
      }
      // ---- prefactor and signs, the |T| > 1e-16 guard, accumulation
      const int dco = dout * d0, nc = nbi * dco;
      {
        const int tpc = NT / nc, c = tid % nc, t0 = tid / nc;
        if (t0 < tpc) {
          const int j = c / dco;
          const double sc = ist[j].scale;
          double mx = 0.0;
          for (int t = t0; t < r; t += tpc) mx = fmax(mx, fabs(mul(T[t * NC + c], sc)));
          atomicMax(&s_max[j], (unsigned long long)__double_as_longlong(mx));  // non-negative doubles order as integers
        }
      }
      group_sync<NG>(g);
      double *dst = Sigma + B.goff[C.b_out];
      for (int idx = tid; idx < r * dco; idx += NT) {
        const int t = idx / dco, ee = idx - t * dco;
        double a = 0.0;
        bool keep_any = false;
        for (int j = 0; j < nbi; ++j)
          if (__longlong_as_double((long long)s_max[j]) > 1e-16) {
            a = add(a, mul(T[t * NC + j * dco + ee], ist[j].scale));
            keep_any = true;
          }
        if (keep_any) atomicAdd(dst + idx, mul(scale, a));
      }
      group_sync<NG>(g);
    }
  }
}

}  // namespace xca
