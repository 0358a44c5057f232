// Sigma backbone evaluation on the device, panel form (plain FP64 path).
//
// A CTA of PANEL_THREADS threads takes a run of pole tuples of one path class (work unit) and evaluates
// `batch` of them together.  The T slabs of the batch's items sit side by side as the columns of a
// shared-memory panel (RP rows = tau nodes, NC columns = item x matrix entry), so every r x r DLR
// operator of an edge acts on all of them at once, on the FP64 tensor cores (mma.sync m8n8k4 f64):
//   K^-1 T     blocked substitution by the whole CTA: per 8-row block an MMA rectangular update, then the
//              in-block solve (one thread per column);
//   W gc, and (beta K) Q with (beta K) P' in one pass   warp-tiled MMA products.
// One FP64 MMA computes every element of its 8 x 8 tile as four fused multiply-adds in ascending k,
// each correctly rounded — the same values as the scalar chain fma(a3, b3, fma(a2, b2, fma(a1, b1,
// fma(a0, b0, c)))), which this build checks on the device bit for bit.  So each output element is
// still one chain of fused multiply-adds over k ascending from zero (descending in the backward
// substitution, fed as reversed k inside each group of four), exactly as in the CPU restatement, and
// each item's contribution stays bit-identical to it.  The per-item steps (vertex products with the
// item's operator and K factor, Q and P' with the item's edge table, the zero vertex) run on the CUDA
// cores with threads owning panel columns.  sigma_kernel.cuh documents the item arithmetic and its
// reference lines.
#pragma once
#include "sigma_kernel.cuh"

namespace xca {

constexpr int PANEL_THREADS = 512;
constexpr int PANEL_WARPS = PANEL_THREADS / 32;

// NC usable panel columns; rows are stored with stride LDP = NC + 8 and the DLR matrices' columns with
// stride RP + 8 (both 8 mod 16 doubles), so that the four k rows of an MMA fragment fall on distinct
// shared-memory banks.
template <int RP>
struct PanelCfg;
template <>
struct PanelCfg<32> { static constexpr int NC = 128, LDP = 136; };
template <>
struct PanelCfg<48> { static constexpr int NC = 128, LDP = 136; };
template <>
struct PanelCfg<64> { static constexpr int NC = 64, LDP = 72; };

template <int RP>
__host__ __device__ constexpr int mat_stride() { return RP + 8; }

// Warp tiling of the MMA products: NTL column tiles and MT row tiles of 8; each warp owns NPW column tiles
// and MPG row tiles (the row tiles are split into MG groups when there are fewer column tiles than warps).
template <int RP>
struct MmaMap {
  static constexpr int NTL = PanelCfg<RP>::NC / 8, MT = RP / 8;
  static constexpr int NPW = NTL >= PANEL_WARPS ? NTL / PANEL_WARPS : 1;
  static constexpr int MG = NTL >= PANEL_WARPS ? 1 : PANEL_WARPS / NTL;
  static constexpr int MPG = MT / MG;
  static_assert(NTL >= PANEL_WARPS ? NTL % PANEL_WARPS == 0 : (PANEL_WARPS % NTL == 0 && MT % MG == 0), "MMA warp tiling");
  __device__ static int n0(int warp) { return MG == 1 ? warp * NPW : warp % NTL; }
  __device__ static int m0(int warp) { return MG == 1 ? 0 : (warp / NTL) * MPG; }
};

template <int RP>
__host__ __device__ constexpr int panel_nc() { return PanelCfg<RP>::NC; }

// Dynamic shared memory of the panel kernels, in doubles: LU (stride RP + 8) + reciprocal diagonal | W | BK
// | panels A, B, C (RP x LDP each) | item states | pivot gather and its inverse (2 RP ints).
template <int RP>
__host__ __device__ constexpr size_t panel_smem_doubles() {
  return 3 * (size_t)mat_stride<RP>() * RP + RP + 3 * (size_t)RP * PanelCfg<RP>::LDP + (sizeof(ItemState) * PANEL_BMAX + 7) / 8 + RP;
}

template <int RP>
__device__ __forceinline__ void panel_layout(double *smem, double *&sLU, double *&sW, double *&sBK, double *&PA, ItemState *&ist,
                                             int *&sPerm) {
  constexpr int S = mat_stride<RP>();
  sLU = smem;
  sW = sLU + S * RP + RP;
  sBK = sW + S * RP;
  PA = sBK + S * RP;
  ist = reinterpret_cast<ItemState *>(PA + 3 * RP * PanelCfg<RP>::LDP);
  sPerm = reinterpret_cast<int *>(reinterpret_cast<double *>(ist) + (sizeof(ItemState) * PANEL_BMAX + 7) / 8);
}

// Stage the DLR matrices (global: column stride RP) into shared memory with column stride RP + 8; the
// reciprocal diagonal follows the LU columns; sPerm receives the pivot gather (RP ints) followed by its
// inverse (RP ints: the pivot-order position of tau node t, -1 in the pad).
template <int RP>
__device__ __forceinline__ void stage_basis(const DevBasis &B, double *sLU, double *sW, double *sBK, int *sPerm) {
  constexpr int S = mat_stride<RP>();
  for (int e = threadIdx.x; e < RP * RP; e += blockDim.x) {
    const int k = e / RP, i = e - k * RP;
    sLU[k * S + i] = B.LUp[e];
    sW[k * S + i] = B.Wp[e];
    sBK[k * S + i] = B.BKp[e];
  }
  for (int i = threadIdx.x; i < RP; i += blockDim.x) {
    sLU[S * RP + i] = B.LUp[RP * RP + i];
    sPerm[i] = B.perm[i];
    sPerm[RP + i] = B.pinv[i];
  }
  __syncthreads();
}


// Y[i][c] = sum_{k < r} M[i][k] X1[k][c] (DUAL: Y[i][c] = fma(t_i, (M X2)[i][c], (M X1)[i][c])) for i < r,
// c < nc.  M is column-major with stride RP + 8 (zero beyond column r); X rows k >= r are masked to zero.
// Warps own column and row tiles as MmaMap lays them out.
template <int RP, bool DUAL>
__device__ __forceinline__ void panel_mma(const double *__restrict__ sM, const double *__restrict__ X1, const double *__restrict__ X2,
                                          double *__restrict__ Y, int r, int nc, const double *__restrict__ tabs, int warp, int lane) {
  using MM = MmaMap<RP>;
  constexpr int S = mat_stride<RP>(), LDP = PanelCfg<RP>::LDP, MT = MM::MPG, NPW = MM::NPW;
  const int g = lane >> 2, q = lane & 3;
  const int n0 = MM::n0(warp), mb = MM::m0(warp);
  if (n0 * 8 >= nc) return;
  const int mt = ((r + 7) >> 3) - mb;
  double a1[MT][NPW][2], a2[MT][NPW][2];
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int t = 0; t < NPW; ++t) {
      a1[m][t][0] = a1[m][t][1] = 0.0;
      a2[m][t][0] = a2[m][t][1] = 0.0;
    }
  for (int k0 = 0; k0 < r; k0 += 4) {
    const int k = k0 + q;
    const bool kv = k < r;
    double b1[NPW], b2[NPW];
#pragma unroll
    for (int t = 0; t < NPW; ++t) {
      const int c = (n0 + t) * 8 + g;
      b1[t] = kv ? X1[k * LDP + c] : 0.0;
      if (DUAL) b2[t] = kv ? X2[k * LDP + c] : 0.0;
    }
#pragma unroll
    for (int m = 0; m < MT; ++m) {
      if (m < mt) {
        const double a = sM[k * S + (mb + m) * 8 + g];
#pragma unroll
        for (int t = 0; t < NPW; ++t) {
          dmma(a1[m][t][0], a1[m][t][1], a, b1[t]);
          if (DUAL) dmma(a2[m][t][0], a2[m][t][1], a, b2[t]);
        }
      }
    }
  }
#pragma unroll
  for (int m = 0; m < MT; ++m) {
    const int i = (mb + m) * 8 + g;
    if (m < mt && i < r) {
#pragma unroll
      for (int t = 0; t < NPW; ++t)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = (n0 + t) * 8 + 2 * q + e;
          if (c < nc) Y[i * LDP + c] = DUAL ? fmad(tabs[i], a2[m][t][e], a1[m][t][e]) : a1[m][t][e];
        }
    }
  }
}

// In-block substitution of panel column c over rows j0 .. j1 - 1 of one 8-row block, one thread: forward
// with the unit lower L, backward with U and the reciprocal diagonal, in the operation order of
// lu_solve_reg.  A full block (j1 = j0 + 8) loads every operand before the first operation, the L / U
// columns and the diagonal as 16-byte pairs; the last, partial block keeps each step behind its row guard.
template <int RP>
__device__ __forceinline__ void inblock_forward(const double *__restrict__ sLU, double *P, int j0, int j1, int c) {
  constexpr int S = mat_stride<RP>(), LDP = PanelCfg<RP>::LDP;
  double xb[8];
  if (j1 == j0 + 8) {
    double L[8][8];  // L[qq][kk] = L[j0 + qq][j0 + kk] for qq > kk
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) xb[qq] = P[(j0 + qq) * LDP + c];
#pragma unroll
    for (int kk = 0; kk < 7; ++kk)
#pragma unroll
      for (int pr = (kk + 1) & ~1; pr < 8; pr += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(sLU + (j0 + kk) * S + j0 + pr);
        L[pr][kk] = v.x;
        L[pr + 1][kk] = v.y;
      }
#pragma unroll
    for (int kk = 0; kk < 7; ++kk)
#pragma unroll
      for (int qq = kk + 1; qq < 8; ++qq) xb[qq] = fmad(-L[qq][kk], xb[kk], xb[qq]);
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) P[(j0 + qq) * LDP + c] = xb[qq];
  } else {
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) xb[qq] = (j0 + qq < j1) ? P[(j0 + qq) * LDP + c] : 0.0;
#pragma unroll
    for (int kk = 0; kk < 7; ++kk)
#pragma unroll
      for (int qq = kk + 1; qq < 8; ++qq)
        if (j0 + qq < j1) xb[qq] = fmad(-sLU[(j0 + kk) * S + j0 + qq], xb[kk], xb[qq]);
#pragma unroll
    for (int qq = 0; qq < 8; ++qq)
      if (j0 + qq < j1) P[(j0 + qq) * LDP + c] = xb[qq];
  }
}

template <int RP>
__device__ __forceinline__ void inblock_backward(const double *__restrict__ sLU, double *P, int j0, int j1, int c) {
  constexpr int S = mat_stride<RP>(), LDP = PanelCfg<RP>::LDP;
  const double *dinv = sLU + S * RP;
  double xb[8];
  if (j1 == j0 + 8) {
    double U[8][8], dv[8];  // U[qq][kk] = U[j0 + qq][j0 + kk] for qq < kk
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) xb[qq] = P[(j0 + qq) * LDP + c];
#pragma unroll
    for (int pr = 0; pr < 8; pr += 2) {
      const double2 v = *reinterpret_cast<const double2 *>(dinv + j0 + pr);
      dv[pr] = v.x;
      dv[pr + 1] = v.y;
    }
#pragma unroll
    for (int kk = 1; kk < 8; ++kk)
#pragma unroll
      for (int pr = 0; pr < kk; pr += 2) {
        const double2 v = *reinterpret_cast<const double2 *>(sLU + (j0 + kk) * S + j0 + pr);
        U[pr][kk] = v.x;
        U[pr + 1][kk] = v.y;
      }
#pragma unroll
    for (int kk = 7; kk >= 0; --kk) {
      xb[kk] = mul(xb[kk], dv[kk]);
#pragma unroll
      for (int qq = 0; qq < kk; ++qq) xb[qq] = fmad(-U[qq][kk], xb[kk], xb[qq]);
    }
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) P[(j0 + qq) * LDP + c] = xb[qq];
  } else {
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) xb[qq] = (j0 + qq < j1) ? P[(j0 + qq) * LDP + c] : 0.0;
#pragma unroll
    for (int kk = 7; kk >= 0; --kk) {
      if (j0 + kk < j1) {
        xb[kk] = mul(xb[kk], dinv[j0 + kk]);
#pragma unroll
        for (int qq = 0; qq < kk; ++qq) xb[qq] = fmad(-sLU[(j0 + kk) * S + j0 + qq], xb[kk], xb[qq]);
      }
    }
#pragma unroll
    for (int qq = 0; qq < 8; ++qq)
      if (j0 + qq < j1) P[(j0 + qq) * LDP + c] = xb[qq];
  }
}

// P[:, c] <- K^-1 P[:, c] for c < nc on a panel whose rows are already in pivot order (row i holds the
// original row perm[i]).  Columns are independent, so each warp solves its own column tiles alone, with
// no CTA barrier until the end.  Right-looking over 8-row blocks: the warp keeps every block's rows of
// its tiles in MMA accumulators; once block K is solved (one lane per column runs the in-block
// substitution in shared memory), its rows, read back as MMA B fragments, update all later blocks'
// accumulators at once (A = -L, or -U going backward) — independent MMA chains whose fragments are all
// loaded before the first MMA of the step (every address lies inside the LU and the panel).  Every
// element still receives exactly the fused multiply-adds of lu_solve_reg in the same order — forward k
// ascending, backward k descending with the reciprocal diagonal applied at k = i — so the result is
// bit-identical to it (a masked MMA term, k >= r, adds 0 * 0); padding rows are not written.
template <int RP>
__device__ __forceinline__ void panel_trsm_mma(const double *__restrict__ sLU, double *P, int r, int nc, int tid, int warp, int lane) {
  using MM = MmaMap<RP>;
  constexpr int S = mat_stride<RP>(), LDP = PanelCfg<RP>::LDP, NPW = MM::NPW, MT = RP / 8;
  const int g = lane >> 2, q = lane & 3, n0 = MM::n0(warp);
  const bool wact = (MM::MG == 1 || warp < MM::NTL) && n0 * 8 < nc;  // one row tile: the first row group's warps
  const int nblk = (r + 7) >> 3;
  const int cs = n0 * 8 + lane;  // the column this lane substitutes in-block (lanes < 8 NPW)
  const bool sact = lane < 8 * NPW && cs < nc;
  if (wact) {
    double acc[MT][NPW][2];
    // accumulators of row g of every block, columns 2q, 2q + 1 of each tile (rows past r: unused)
    auto load_acc = [&]() {
#pragma unroll
      for (int J = 0; J < MT; ++J)
#pragma unroll
        for (int t = 0; t < NPW; ++t)
#pragma unroll
          for (int e = 0; e < 2; ++e) acc[J][t][e] = P[(J * 8 + g) * LDP + (n0 + t) * 8 + 2 * q + e];
      __syncwarp();
    };
    auto store_acc = [&](int K) {
      const int i = K * 8 + g;
      if (i < r)
#pragma unroll
        for (int t = 0; t < NPW; ++t)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int c = (n0 + t) * 8 + 2 * q + e;
            if (c < nc) P[i * LDP + c] = acc[K][t][e];
          }
      __syncwarp();
    };
    load_acc();
#pragma unroll
    for (int K = 0; K < MT; ++K) {
      if (K < nblk) {
        const int j0 = K * 8, j1 = min(r, j0 + 8);
        if (K > 0) store_acc(K);  // block 0's rows are P's rows
        if (sact) inblock_forward<RP>(sLU, P, j0, j1, cs);
        __syncwarp();
        if (K + 1 < nblk) {  // block K is full here: rows j0 .. j0 + 7 < r
          double bf[2][NPW], af[MT][2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
#pragma unroll
            for (int t = 0; t < NPW; ++t) bf[h][t] = P[(j0 + 4 * h + q) * LDP + (n0 + t) * 8 + g];
#pragma unroll
            for (int J = K + 1; J < MT; ++J) af[J][h] = -sLU[(j0 + 4 * h + q) * S + J * 8 + g];  // -L[8 J + g][k]
          }
#pragma unroll
          for (int J = K + 1; J < MT; ++J)
            if (J < nblk)
#pragma unroll
              for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int t = 0; t < NPW; ++t) dmma(acc[J][t][0], acc[J][t][1], af[J][h], bf[h][t]);
        }
      }
    }
    load_acc();
#pragma unroll
    for (int K = MT - 1; K >= 0; --K) {
      if (K < nblk) {
        const int j0 = K * 8, j1 = min(r, j0 + 8);
        if (K + 1 < nblk) store_acc(K);  // the last block's rows are P's rows
        if (sact) inblock_backward<RP>(sLU, P, j0, j1, cs);
        __syncwarp();
        if (K > 0) {
          // group h feeds k = j0 + 7 - 4 h - q: the MMA's ascending order inside a group is the
          // descending order of the substitution
          double bf[2][NPW], af[MT][2];
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int k = j0 + 7 - 4 * h - q;
            const bool kv = k < j1;
#pragma unroll
            for (int t = 0; t < NPW; ++t) {
              const double pv = P[k * LDP + (n0 + t) * 8 + g];
              bf[h][t] = kv ? pv : 0.0;
            }
#pragma unroll
            for (int J = 0; J < K; ++J) {
              const double u = sLU[k * S + J * 8 + g];  // U[8 J + g][k]
              af[J][h] = kv ? -u : 0.0;
            }
          }
#pragma unroll
          for (int J = 0; J < K; ++J)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
              for (int t = 0; t < NPW; ++t) dmma(acc[J][t][0], acc[J][t][1], af[J][h], bf[h][t]);
        }
      }
    }
  }
  // a warp's column tiles in the products that follow are its own here unless the row tiles are split
  if (MM::MG > 1) __syncthreads();
}

// Edge tables: for block b and signature sig, fc = K^-1 (G_b prod K) and W fc (sig 0: no factor;
// 1 + s p + l: one factor, s = 0: K(t, +beta w_l), 1: K(t, -beta w_l); 1 + 2p + (s1 p + l1) 2p + s2 p + l2:
// two factors, the lower line's first).  A CTA takes NC consecutive (sig, entry) columns of one block:
// gather with the K factors (rows in pivot order), K^-1, write fc, W fc, write.  `chunks` lists
// (block, first column) pairs.
template <int RP>
__global__ void __launch_bounds__(PANEL_THREADS, 1) edge_tables_panel_kernel(DevBasis B, const double *__restrict__ G,
                                                                              const int2 *__restrict__ chunks, int n_chunks) {
  constexpr int NCU = PanelCfg<RP>::NC, LDP = PanelCfg<RP>::LDP;
  extern __shared__ __align__(16) double smem[];
  double *sLU, *sW, *sBK, *PA;
  ItemState *ist;
  int *sPerm;
  panel_layout<RP>(smem, sLU, sW, sBK, PA, ist, sPerm);
  double *PB = PA + RP * LDP;
  stage_basis<RP>(B, sLU, sW, sBK, sPerm);
  const int r = B.r, p = B.p, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int ch = blockIdx.x; ch < n_chunks; ch += gridDim.x) {
    const int b = chunks[ch].x, col0 = chunks[ch].y;
    const int d = B.dims[b], dd = d * d;
    const long total = (long)B.nsig * dd;
    const int ncols = (int)min((long)NCU, total - col0);
    const double *g = G + B.goff[b];
    for (int idx = tid; idx < r * ncols; idx += PANEL_THREADS) {
      const int t = idx / ncols, c = idx - t * ncols;
      const long qc = col0 + c;
      const int sig = (int)(qc / dd), e = (int)(qc - (long)sig * dd);
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
      PA[sPerm[RP + t] * LDP + c] = v;
    }
    __syncthreads();
    panel_trsm_mma<RP>(sLU, PA, r, ncols, tid, warp, lane);
    panel_mma<RP, false>(sW, PA, nullptr, PB, r, ncols, nullptr, warp, lane);
    __syncthreads();
    double *out = const_cast<double *>(B.tab) + B.tab_off[b];
    for (int idx = tid; idx < r * ncols; idx += PANEL_THREADS) {
      const int t = idx / ncols, c = idx - t * ncols;
      const long qc = col0 + c;
      const long sig = qc / dd, e = qc - sig * dd;
      double *o = out + sig * 2 * r * dd;
      o[t * dd + e] = PA[t * LDP + c];
      o[(long)r * dd + t * dd + e] = PB[t * LDP + c];
    }
    __syncthreads();
  }
}

// One vertex of a class: operator table base (F, F^dag, or their pole-resolved reflected forms), the
// operator's index within its set, the vertex's hybridization line and the sign of its K factor.
struct VertexOp {
  long base;
  int qo, line, ks;
  bool pole;
};

// Vertex pass: X(t) <- k(t) F T(t) for every item of the batch (multiply_left_vertex), thread per output
// column over a stride of tau rows.  DV > 0 is the input block dimension known at compile time (the
// operator row is held in registers across the rows and every load of a row is issued before its
// fused multiply-adds); DV = 0 takes dv at run time.  The operation order is the same either way.
template <int RP, int DV>
__device__ __forceinline__ void vertex_pass(const DevBasis &B, const VertexOp &vo, const ItemState *ist, const double *T, double *X,
                                            const int *rowpos, int r, int dv, int dvp, int ncol, int nbi, int tid) {
  constexpr int NC = PanelCfg<RP>::LDP, NT = PANEL_THREADS;
  const int dci = dv * ncol, dco = dvp * ncol, nc = nbi * dco, tpc = NT / nc, c = tid % nc, t0 = tid / nc;
  if (t0 >= tpc) return;
  const int p = B.p;
  const int j = c / dco, e = c - j * dco, x = e / ncol, z = e - x * ncol;
  const ItemState &S = ist[j];
  const int l = S.lpole[vo.line];
  const long opoff = vo.base + (vo.pole ? (long)vo.qo * p + l : (long)vo.qo) * dvp * dv;
  const double *F = B.ops + opoff + x * dv;
  // a line in its case-A form contributes its K factor at both of its vertices
  const double *kt = (vo.line > 0 && S.caseA[vo.line]) ? (vo.ks < 0 ? B.kitm : B.kitp) + l : nullptr;
  const double *Tc = T + j * dci + z;
  double f[DV > 0 ? DV : 1];
#pragma unroll
  for (int y = 0; y < DV; ++y) f[y] = F[y];
  for (int t = t0; t < r; t += tpc) {
    const double *Tt = Tc + t * NC;
    double a = 0.0;
    if (DV > 0) {
      double tv[DV > 0 ? DV : 1];
#pragma unroll
      for (int y = 0; y < DV; ++y) tv[y] = Tt[y * ncol];
#pragma unroll
      for (int y = 0; y < DV; ++y) a = fmad(f[y], tv[y], a);
    } else {
      for (int y = 0; y < dv; ++y) a = fmad(F[y], Tt[y * ncol], a);
    }
    if (kt) a = mul(a, kt[(size_t)t * p]);
    X[(rowpos ? rowpos[t] : t) * NC + c] = a;
  }
}

// Q / P' pass of an edge, one warp per tau row l (Q and P' of row l read only row l of gc and Gt):
// Q_l = Ft_l gc_l + fc_l Gt_l (into Y) and P'_l = K(0, om_l) (fc_l gc_l) (over Gt, into X).  D > 0 is the
// edge's block dimension known at compile time (all loads of an entry are issued before its fused
// multiply-adds); D = 0 takes d at run time.  The operation order is the same either way.
template <int RP, int D>
__device__ __forceinline__ void qp_pass(const DevBasis &B, const ItemState *ist, const double *T, double *X, double *Y, int r, int d,
                                        int ncol, int nc, int warp, int lane) {
  constexpr int NC = PanelCfg<RP>::LDP, NCU = PanelCfg<RP>::NC, NT = PANEL_THREADS;
  constexpr int CPL = (NCU + 31) / 32;
  const int dd = d * d, dc = d * ncol;
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
        if (D > 0) {
          constexpr int DD = D > 0 ? D : 1;
          double f[DD], ft[DD], gv[DD], gtv[DD];
#pragma unroll
          for (int y = 0; y < D; ++y) {
            f[y] = fl[y];
            ft[y] = ftl[y];
            gv[y] = gl[y * ncol];
            gtv[y] = gtl[y * ncol];
          }
#pragma unroll
          for (int y = 0; y < D; ++y) {
            aq = fmad(ft[y], gv[y], fmad(f[y], gtv[y], aq));
            ap = fmad(f[y], gv[y], ap);
          }
        } else {
          for (int y = 0; y < d; ++y) {
            aq = fmad(ftl[y], gl[y * ncol], fmad(fl[y], gtl[y * ncol], aq));
            ap = fmad(fl[y], gl[y * ncol], ap);
          }
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

// Zero vertex, inner pass for operator mu (multiply_left_vertex_and_right_zero_vertex): Y(t) =
// sum_kappa (+-h(t)[om, ok]) (T(t) F_kappa), thread per Y column over a stride of tau rows.  D1 > 0 is
// the first block's dimension known at compile time (the row of T is loaded once for every kappa);
// D1 = 0 takes d1 at run time.  The operation order is the same either way.
template <int RP, int D1>
__device__ __forceinline__ void zv_inner_pass(const DevBasis &B, const double *T, double *Y, int r, int pk, int qs, int om, bool fwd,
                                              double hs, long ok_off, int d0, int d1, int dv, int nbi, int tid) {
  constexpr int NC = PanelCfg<RP>::LDP, NT = PANEL_THREADS;
  const int n = B.n, dci = dv * d1, dmid = dv * d0, ncm = nbi * dmid, tpm = NT / ncm, c = tid % ncm, tm0 = tid / ncm;
  if (tm0 >= tpm) return;
  const int j = c / dmid, ee = c - j * dmid, x = ee / d0, z = ee - x * d0;
  const double *Tc = T + j * dci + x * d1;
  for (int t = tm0; t < r; t += tpm) {
    const double *Tt = Tc + t * NC;
    double tv[D1 > 0 ? D1 : 1];
#pragma unroll
    for (int y = 0; y < D1; ++y) tv[y] = Tt[y];
    double a = 0.0;
    for (int kap = 0; kap < qs; ++kap) {
      const int ok = B.set_to_orb[pk * n + kap];
      const double h = fwd ? B.hval[((size_t)t * n + om) * n + ok] : B.hrefl[((size_t)t * n + ok) * n + om];
      if (h == 0.0) continue;
      const double *Fk = B.ops + ok_off + (size_t)kap * d1 * d0 + z;
      double tf = 0.0;
      if (D1 > 0) {
        double fv[D1 > 0 ? D1 : 1];
#pragma unroll
        for (int y = 0; y < D1; ++y) fv[y] = Fk[y * d0];
#pragma unroll
        for (int y = 0; y < D1; ++y) tf = fmad(tv[y], fv[y], tf);
      } else {
        for (int y = 0; y < d1; ++y) tf = fmad(Tt[y], Fk[y * d0], tf);
      }
      a = fmad(mul(hs, h), tf, a);
    }
    Y[t * NC + c] = a;
  }
}

// Zero vertex, outer pass for operator mu: X(t) += F_mu Y(t) (first = true: X(t) = 0 + F_mu Y(t)), thread
// per output column over a stride of tau rows; rows go to rowpos[t] when given.  DV > 0: the block
// dimension known at compile time (the operator row is held in registers); DV = 0 takes dv at run time.
template <int RP, int DV>
__device__ __forceinline__ void zv_outer_pass(const double *Fm, const double *Y, double *X, const int *rowpos, int r, int d0, int dv,
                                              int dvp, int nbi, int tid, bool first) {
  constexpr int NC = PanelCfg<RP>::LDP, NT = PANEL_THREADS;
  const int dmid = dv * d0, dco = dvp * d0, nco = nbi * dco, tpo = NT / nco, c = tid % nco, to0 = tid / nco;
  if (to0 >= tpo) return;
  const int j = c / dco, ee = c - j * dco, x = ee / d0, z = ee - x * d0;
  const double *Fx = Fm + x * dv, *Yc = Y + j * dmid + z;
  double f[DV > 0 ? DV : 1];
#pragma unroll
  for (int y = 0; y < DV; ++y) f[y] = Fx[y];
  for (int t = to0; t < r; t += tpo) {
    const double *Yt = Yc + t * NC;
    double a = 0.0;
    if (DV > 0) {
      double yv[DV > 0 ? DV : 1];
#pragma unroll
      for (int y = 0; y < DV; ++y) yv[y] = Yt[y * d0];
#pragma unroll
      for (int y = 0; y < DV; ++y) a = fmad(f[y], yv[y], a);
    } else {
      for (int y = 0; y < dv; ++y) a = fmad(Fx[y], Yt[y * d0], a);
    }
    const int row = rowpos ? rowpos[t] : t;
    X[row * NC + c] = add(first ? 0.0 : X[row * NC + c], a);
  }
}

// One work unit (a run of pole tuples of one path class, staged in shared memory as C) on the CTA's panels:
// batches of `C.batch` items (see the file comment).  Shared by the single-job and the job-batched kernels.
template <int RP>
__device__ __forceinline__ void panel_unit(const DevBasis &B, const ClassRec &C, const WorkUnit &wu, int u, const double *__restrict__ G,
                                           const SigmaOut &out, const double *sLU, const double *sW, const double *sBK,
                                           double *PA, ItemState *ist, const int *sPerm, unsigned long long *s_max) {
  constexpr int NC = PanelCfg<RP>::LDP, NT = PANEL_THREADS;  // NC: panel row stride
  double *PB = PA + RP * NC, *PC = PB + RP * NC;
  const int r = B.r, p = B.p, n = B.n, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m = C.m, vct0 = C.vct0;
  const int d0 = C.bdims[0], d1 = C.bdims[1];
  const int dout = C.bdims[2 * m];
  const int cap = C.batch;
  const int nops = 4 * m - 3;
  if (path_meets_zero_block(B, C.ind_path, m)) {
    // the reference drops this path: no items (an ordered-mode slot still receives its zeros)
    if (out.slots)
      for (int idx = tid; idx < r * dout * d0; idx += NT) out.slots[out.slot_off[u] + idx] = 0.0;
    __syncthreads();
    return;
  }

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
    __syncthreads();

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
        // operator base of this vertex (uniform); the pole-dependent part and the K factor are per item
        const int vk = C.vkind[v];
        const long vbase = vk == 0 ? B.F_off[s * B.nb + b] : vk == 1 ? B.Fd_off[s * B.nb + b]
                         : vk == 2 ? B.Fb_off[s * B.nb + b] : B.Fdb_off[s * B.nb + b];
        int ks = 0;
        if (line > 0) {
          const int fwd = (C.fbmask >> line) & 1;
          ks = (v == C.la[line]) ? (fwd ? -1 : 1) : (fwd ? 1 : -1);
        }
        const VertexOp vo{vbase, qo, line, ks, vk >= 2};
        switch (dv) {
          case 1: vertex_pass<RP, 1>(B, vo, ist, T, X, rowpos, r, dv, dvp, ncol, nbi, tid); break;
          case 2: vertex_pass<RP, 2>(B, vo, ist, T, X, rowpos, r, dv, dvp, ncol, nbi, tid); break;
          case 3: vertex_pass<RP, 3>(B, vo, ist, T, X, rowpos, r, dv, dvp, ncol, nbi, tid); break;
          case 4: vertex_pass<RP, 4>(B, vo, ist, T, X, rowpos, r, dv, dvp, ncol, nbi, tid); break;
          default: vertex_pass<RP, 0>(B, vo, ist, T, X, rowpos, r, dv, dvp, ncol, nbi, tid); break;
        }
        __syncthreads();
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
        panel_trsm_mma<RP>(sLU, T, r, nc, tid, warp, lane);
        panel_mma<RP, false>(sW, T, nullptr, X, r, nc, nullptr, warp, lane);
        __syncthreads();
        // (b) per row l (one warp per row; Q and P' of row l read only row l of gc and Gt):
        //     Q_l = Ft_l gc_l + fc_l Gt_l (into Y) and P'_l = K(0, om_l) (fc_l gc_l) (over Gt, into X)
        switch (d) {
          case 1: qp_pass<RP, 1>(B, ist, T, X, Y, r, d, ncol, nc, warp, lane); break;
          case 2: qp_pass<RP, 2>(B, ist, T, X, Y, r, d, ncol, nc, warp, lane); break;
          case 3: qp_pass<RP, 3>(B, ist, T, X, Y, r, d, ncol, nc, warp, lane); break;
          case 4: qp_pass<RP, 4>(B, ist, T, X, Y, r, d, ncol, nc, warp, lane); break;
          default: qp_pass<RP, 0>(B, ist, T, X, Y, r, d, ncol, nc, warp, lane); break;
        }
        __syncthreads();
        // (c) h = fma(t_i, (beta K) P', (beta K) Q) (into T; gc is no longer needed)
        panel_mma<RP, true>(sBK, Y, X, T, r, nc, B.tabs, warp, lane);
        __syncthreads();
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
        if (qs == 0) {  // no operator pair: the zero vertex is zero
          const int nco = nbi * dvp * d0, tpo = NT / nco, co = tid % nco, to0 = tid / nco;
          if (to0 < tpo)
            for (int t = to0; t < r; t += tpo) X[(rowpos ? rowpos[t] : t) * NC + co] = 0.0;
          __syncthreads();
        }
        for (int mu = 0; mu < qs; ++mu) {
          const int om = B.set_to_orb[pk * n + mu];
          switch (d1) {
            case 1: zv_inner_pass<RP, 1>(B, T, Y, r, pk, qs, om, fwd, hs, ok_off, d0, d1, dv, nbi, tid); break;
            case 2: zv_inner_pass<RP, 2>(B, T, Y, r, pk, qs, om, fwd, hs, ok_off, d0, d1, dv, nbi, tid); break;
            case 3: zv_inner_pass<RP, 3>(B, T, Y, r, pk, qs, om, fwd, hs, ok_off, d0, d1, dv, nbi, tid); break;
            case 4: zv_inner_pass<RP, 4>(B, T, Y, r, pk, qs, om, fwd, hs, ok_off, d0, d1, dv, nbi, tid); break;
            default: zv_inner_pass<RP, 0>(B, T, Y, r, pk, qs, om, fwd, hs, ok_off, d0, d1, dv, nbi, tid); break;
          }
          __syncthreads();
          const double *Fm = B.ops + om_off + (size_t)mu * dvp * dv;
          switch (dv) {
            case 1: zv_outer_pass<RP, 1>(Fm, Y, X, rowpos, r, d0, dv, dvp, nbi, tid, mu == 0); break;
            case 2: zv_outer_pass<RP, 2>(Fm, Y, X, rowpos, r, d0, dv, dvp, nbi, tid, mu == 0); break;
            case 3: zv_outer_pass<RP, 3>(Fm, Y, X, rowpos, r, d0, dv, dvp, nbi, tid, mu == 0); break;
            case 4: zv_outer_pass<RP, 4>(Fm, Y, X, rowpos, r, d0, dv, dvp, nbi, tid, mu == 0); break;
            default: zv_outer_pass<RP, 0>(Fm, Y, X, rowpos, r, d0, dv, dvp, nbi, tid, mu == 0); break;
          }
          __syncthreads();
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
    __syncthreads();
    if (out.slots) {
      // ordered mode: the unit's running sum continues over its batches (a thread keeps the same
      // entries from batch to batch, so it reads back only what it wrote)
      double *dst = out.slots + out.slot_off[u];
      for (int idx = tid; idx < r * dco; idx += NT) {
        const int t = idx / dco, ee = idx - t * dco;
        double a = first == 0 ? 0.0 : dst[idx];
        for (int j = 0; j < nbi; ++j)
          if (__longlong_as_double((long long)s_max[j]) > 1e-16) a = add(a, mul(T[t * NC + j * dco + ee], ist[j].scale));
        dst[idx] = a;
      }
    } else {
      double *dst = out.Sigma + B.goff[C.b_out];
      for (int idx = tid; idx < r * dco; idx += NT) {
        const int t = idx / dco, ee = idx - t * dco;
        double a = 0.0;
        bool keep_any = false;
        for (int j = 0; j < nbi; ++j)
          if (__longlong_as_double((long long)s_max[j]) > 1e-16) {
            a = add(a, mul(T[t * NC + j * dco + ee], ist[j].scale));
            keep_any = true;
          }
        if (keep_any) atomicAdd(dst + idx, mul(out.scale, a));
      }
    }
    __syncthreads();
  }
}

// Dynamic shared memory: see panel_smem_doubles.
template <int RP>
__global__ void __launch_bounds__(PANEL_THREADS, 1) sigma_panel_kernel(DevBasis B, const ClassRec *__restrict__ classes,
                                                                        const WorkUnit *__restrict__ units, int n_units,
                                                                        int *__restrict__ unit_counter, const double *__restrict__ G,
                                                                        SigmaOut out) {
  constexpr int NT = PANEL_THREADS;
  extern __shared__ __align__(16) double smem[];
  double *sLU, *sW, *sBK, *PA;
  ItemState *ist;
  int *sPerm;
  panel_layout<RP>(smem, sLU, sW, sBK, PA, ist, sPerm);
  __shared__ int s_unit;
  __shared__ ClassRec s_cls;
  __shared__ unsigned long long s_max[PANEL_BMAX];
  stage_basis<RP>(B, sLU, sW, sBK, sPerm);
  const int tid = threadIdx.x;

  while (true) {
    if (tid == 0) s_unit = atomicAdd(unit_counter, 1);
    __syncthreads();
    const int u = s_unit;
    __syncthreads();
    if (u >= n_units) break;
    const WorkUnit wu = units[u];
    // the unit's class record, read by every per-item set-up step, staged in shared memory
    static_assert(sizeof(ClassRec) % sizeof(int) == 0, "ClassRec holds ints only");
    {
      const int *src = reinterpret_cast<const int *>(classes + wu.cls);
      for (int i = tid; i < (int)(sizeof(ClassRec) / sizeof(int)); i += NT) reinterpret_cast<int *>(&s_cls)[i] = src[i];
    }
    __syncthreads();
    panel_unit<RP>(B, s_cls, wu, u, G, out, sLU, sW, sBK, PA, ist, sPerm, s_max);
  }
}

// Job-batched form: every work unit names its job (a solve's basis, model and edge tables, a topology's
// path classes, its G and its output).  The CTA stages a job's descriptor, and its DLR matrices when they
// differ from the staged ones, as the units change job (the host lists the units job by job), then runs the
// unit exactly as the single-job kernel does.  Fast (atomic) summation only.
template <int RP>
__global__ void __launch_bounds__(PANEL_THREADS, 1) sigma_panel_batch_kernel(const SigmaJob *__restrict__ jobs,
                                                                              const WorkUnit *__restrict__ units, int n_units,
                                                                              int *__restrict__ unit_counter) {
  constexpr int NT = PANEL_THREADS;
  extern __shared__ __align__(16) double smem[];
  double *sLU, *sW, *sBK, *PA;
  ItemState *ist;
  int *sPerm;
  panel_layout<RP>(smem, sLU, sW, sBK, PA, ist, sPerm);
  __shared__ int s_unit, s_job_id;
  __shared__ const double *s_staged;
  __shared__ SigmaJob s_job;
  __shared__ ClassRec s_cls;
  __shared__ unsigned long long s_max[PANEL_BMAX];
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_job_id = -1;
    s_staged = nullptr;
  }
  __syncthreads();
  static_assert(sizeof(SigmaJob) % sizeof(int) == 0, "job descriptor copied as ints");

  while (true) {
    if (tid == 0) s_unit = atomicAdd(unit_counter, 1);
    __syncthreads();
    const int u = s_unit;
    __syncthreads();
    if (u >= n_units) break;
    const WorkUnit wu = units[u];
    if (wu.job != s_job_id) {
      const int *src = reinterpret_cast<const int *>(jobs + wu.job);
      for (int i = tid; i < (int)(sizeof(SigmaJob) / sizeof(int)); i += NT) reinterpret_cast<int *>(&s_job)[i] = src[i];
      __syncthreads();
      if (s_job.B.LUp != s_staged) stage_basis<RP>(s_job.B, sLU, sW, sBK, sPerm);
      __syncthreads();
      if (tid == 0) {
        s_job_id = wu.job;
        s_staged = s_job.B.LUp;
      }
    }
    {
      const int *src = reinterpret_cast<const int *>(s_job.classes + wu.cls);
      for (int i = tid; i < (int)(sizeof(ClassRec) / sizeof(int)); i += NT) reinterpret_cast<int *>(&s_cls)[i] = src[i];
    }
    __syncthreads();
    panel_unit<RP>(s_job.B, s_cls, wu, u, s_job.G, s_job.out, sLU, sW, sBK, PA, ist, sPerm, s_max);
  }
}

}  // namespace xca
