// Sigma backbone evaluation with FP32 block products: the bulk arithmetic of the mixed-precision form.
//
// Same work decomposition as the FP64 panel kernel (sigma_panel.cuh): a CTA takes a work unit (a run of
// pole tuples of one path class) and evaluates `batch` items together as the columns of shared-memory
// panels, with the panel kernel's item set-up, pole decode (backbone.cpp:86-150), edge-table selection and
// row order (rows in pivot order before every edge).  What changes is the arithmetic: the panels, the DLR
// matrices (K^-1 as its LU factors, W, beta K) and every product are FP32 on the CUDA cores — the K^-1
// substitution, W gc and the (beta K) products one thread per panel column, the vertex, Q / P' and
// zero-vertex passes as in the FP64 kernel with FP32 operands (the operators, K factors, hybridization
// values and FP64 edge tables are rounded to FP32 as they are read).  Each item's prefactor and the
// accumulation into Sigma stay FP64 (atomics).  A CTA uses about half the shared memory of the FP64
// kernel, so two run per SM.  Accuracy, measured: the NCA diagram (no edge) is within FP32 rounding of the
// FP64 result (1e-7); any diagram with an edge is not usable — the edge's DLR convolution applies K^-1
// (cond ~ 1/eps) and sums over W_lk = K(0, om_k) / (om_k - om_l) whose terms cancel, and its FP32 error
// grows with 1/eps from 1e-1 at eps = 1e-3.  The mixed solve therefore runs only NCA iterations here.
#pragma once
#include "sigma_kernel.cuh"

namespace xca {

constexpr int F32_THREADS = 256;

// Panel columns: the FP64 panel width of the same rank, so the class batches (cut for that width) fit.
template <int RP>
struct F32Cfg;
template <>
struct F32Cfg<32> { static constexpr int NC = 128; };
template <>
struct F32Cfg<48> { static constexpr int NC = 128; };
template <>
struct F32Cfg<64> { static constexpr int NC = 64; };

template <int RP>
__host__ __device__ constexpr int f32_ld() { return F32Cfg<RP>::NC + 1; }  // odd row stride: conflict-free column walks

// Dynamic shared memory in bytes: item states | LU (RP x RP, column-major) + reciprocal diagonal | W | beta K
// (float) | panels T, X, Y (RP x LD floats) | pivot gather and its inverse (2 RP ints).
template <int RP>
__host__ __device__ constexpr size_t f32_smem_bytes() {
  return sizeof(ItemState) * PANEL_BMAX + (3 * (size_t)RP * RP + RP) * sizeof(float) + 3 * (size_t)RP * f32_ld<RP>() * sizeof(float) +
         2 * (size_t)RP * sizeof(int);
}

// x <- K^-1 x for one register-resident column already in pivot order: unit-lower forward and upper backward
// substitution with the padded factors (identity beyond r), FP32.
template <int RP>
__device__ __forceinline__ void f32_lu_solve(const float *__restrict__ sLU, float (&x)[RP]) {
#pragma unroll
  for (int k = 0; k < RP; ++k) {
    const float xk = x[k];
#pragma unroll
    for (int i = k + 1; i < RP; ++i) x[i] = fmaf(-sLU[k * RP + i], xk, x[i]);
  }
#pragma unroll
  for (int k = RP - 1; k >= 0; --k) {
    x[k] = x[k] * sLU[RP * RP + k];
    const float xk = x[k];
#pragma unroll
    for (int i = 0; i < k; ++i) x[i] = fmaf(-sLU[k * RP + i], xk, x[i]);
  }
}

// y_i = sum_k M[i][k] x_k for i < r (M column-major, stride RP), written to P[i * LD + c] (ACC: fma(t_i, y_i,
// P[i * LD + c]) instead).
template <int RP, bool ACC>
__device__ __forceinline__ void f32_matvec(const float *__restrict__ sM, const float (&x)[RP], int r, float *P, int c,
                                           const double *__restrict__ tabs) {
  constexpr int LD = f32_ld<RP>();
#pragma unroll 2
  for (int i = 0; i < r; ++i) {
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < RP; ++k) acc = fmaf(sM[k * RP + i], x[k], acc);
    P[i * LD + c] = ACC ? fmaf((float)tabs[i], acc, P[i * LD + c]) : acc;
  }
}

// Edge, step (a): T <- K^-1 T in place and X <- W (K^-1 T), one thread per column c < nc.
template <int RP>
__device__ __forceinline__ void f32_coefs(const float *sLU, const float *sW, float *T, float *X, int r, int nc, int tid) {
  constexpr int LD = f32_ld<RP>();
  for (int c = tid; c < nc; c += F32_THREADS) {
    float x[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) x[i] = i < r ? T[i * LD + c] : 0.0f;
    f32_lu_solve<RP>(sLU, x);
    for (int i = 0; i < r; ++i) T[i * LD + c] = x[i];
    f32_matvec<RP, false>(sW, x, r, X, c, nullptr);
  }
}

// Edge, step (c): T <- (beta K) Y + t_i (beta K) X (h = h1 + t_i h2), one thread per column.
template <int RP>
__device__ __forceinline__ void f32_dual(const float *sBK, const float *Y, const float *X, float *T, int r, int nc, int tid,
                                         const double *__restrict__ tabs) {
  constexpr int LD = f32_ld<RP>();
  for (int c = tid; c < nc; c += F32_THREADS) {
    float q[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) q[i] = i < r ? Y[i * LD + c] : 0.0f;
    f32_matvec<RP, false>(sBK, q, r, T, c, nullptr);
#pragma unroll
    for (int i = 0; i < RP; ++i) q[i] = i < r ? X[i * LD + c] : 0.0f;
    f32_matvec<RP, true>(sBK, q, r, T, c, tabs);
  }
}

// Vertex: X(t) <- k(t) F T(t) for every item of the batch, thread per output column over a stride of rows
// (rows to rowpos[t] when an edge follows).
__device__ __forceinline__ void f32_vertex(const DevBasis &B, long base, int qo, int line, int ks, bool pole, const ItemState *ist,
                                           const float *T, float *X, const int *rowpos, int r, int dv, int dvp, int ncol, int nbi,
                                           int tid, int LD) {
  const int dci = dv * ncol, dco = dvp * ncol, nc = nbi * dco, tpc = F32_THREADS / nc, c = tid % nc, t0 = tid / nc;
  if (t0 >= tpc) return;
  const int p = B.p;
  const int j = c / dco, e = c - j * dco, x = e / ncol, z = e - x * ncol;
  const ItemState &S = ist[j];
  const int l = S.lpole[line];
  const double *F = B.ops + base + (pole ? (long)qo * p + l : (long)qo) * dvp * dv + x * dv;
  const double *kt = (line > 0 && S.caseA[line]) ? (ks < 0 ? B.kitm : B.kitp) + l : nullptr;
  const float *Tc = T + j * dci + z;
  for (int t = t0; t < r; t += tpc) {
    const float *Tt = Tc + t * LD;
    float a = 0.0f;
    for (int y = 0; y < dv; ++y) a = fmaf((float)F[y], Tt[y * ncol], a);
    if (kt) a *= (float)kt[(size_t)t * p];
    X[(rowpos ? rowpos[t] : t) * LD + c] = a;
  }
}

// Edge, step (b), one warp per row l: Q_l = Wfc_l gc_l + fc_l Gt_l (into Y), P'_l = K(0, om_l) fc_l gc_l (over X).
// Every value of row l is computed before any is stored: P' overwrites the Gt row the other columns read.
template <int NC>
__device__ __forceinline__ void f32_qp(const DevBasis &B, const ItemState *ist, const float *T, float *X, float *Y, int r, int d,
                                       int ncol, int nc, int warp, int lane, int LD) {
  constexpr int CPL = (NC + 31) / 32;
  const int dd = d * d, dc = d * ncol;
  for (int l = warp; l < r; l += F32_THREADS / 32) {
    float qv[CPL], pv[CPL];
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lane + 32 * q;
      float aq = 0.0f, ap = 0.0f;
      if (c < nc) {
        const int j = c / dc, ee = c - j * dc, x = ee / ncol, z = ee - x * ncol;
        const double *fl = B.tab + ist[j].taboff + x * d + (long)l * dd, *ftl = fl + (long)r * dd;
        const float *gl = T + l * LD + j * dc + z, *gtl = X + l * LD + j * dc + z;
        for (int y = 0; y < d; ++y) {
          const float f = (float)fl[y], ft = (float)ftl[y], g = gl[y * ncol], gt = gtl[y * ncol];
          aq = fmaf(ft, g, fmaf(f, gt, aq));
          ap = fmaf(f, g, ap);
        }
      }
      qv[q] = aq;
      pv[q] = (float)B.k0[l] * ap;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < CPL; ++q) {
      const int c = lane + 32 * q;
      if (c < nc) {
        Y[l * LD + c] = qv[q];
        X[l * LD + c] = pv[q];
      }
    }
    __syncwarp();
  }
}

// Zero vertex, inner pass for operator mu: Y(t) = sum_kappa (+-h(t)[om, ok]) (T(t) F_kappa).
__device__ __forceinline__ void f32_zv_inner(const DevBasis &B, const float *T, float *Y, int r, int pk, int qs, int om, bool fwd,
                                             float hs, long ok_off, int d0, int d1, int dv, int nbi, int tid, int LD) {
  const int n = B.n, dci = dv * d1, dmid = dv * d0, ncm = nbi * dmid, tpm = F32_THREADS / ncm, c = tid % ncm, tm0 = tid / ncm;
  if (tm0 >= tpm) return;
  const int j = c / dmid, ee = c - j * dmid, x = ee / d0, z = ee - x * d0;
  const float *Tc = T + j * dci + x * d1;
  for (int t = tm0; t < r; t += tpm) {
    const float *Tt = Tc + t * LD;
    float a = 0.0f;
    for (int kap = 0; kap < qs; ++kap) {
      const int ok = B.set_to_orb[pk * n + kap];
      const double h = fwd ? B.hval[((size_t)t * n + om) * n + ok] : B.hrefl[((size_t)t * n + ok) * n + om];
      if (h == 0.0) continue;
      const double *Fk = B.ops + ok_off + (size_t)kap * d1 * d0 + z;
      float tf = 0.0f;
      for (int y = 0; y < d1; ++y) tf = fmaf(Tt[y], (float)Fk[y * d0], tf);
      a = fmaf(hs * (float)h, tf, a);
    }
    Y[t * LD + c] = a;
  }
}

// Zero vertex, outer pass for operator mu: X(t) (+)= F_mu Y(t), rows to rowpos[t] when an edge follows.
__device__ __forceinline__ void f32_zv_outer(const double *Fm, const float *Y, float *X, const int *rowpos, int r, int d0, int dv,
                                             int dvp, int nbi, int tid, bool first, int LD) {
  const int dmid = dv * d0, dco = dvp * d0, nco = nbi * dco, tpo = F32_THREADS / nco, c = tid % nco, to0 = tid / nco;
  if (to0 >= tpo) return;
  const int j = c / dco, ee = c - j * dco, x = ee / d0, z = ee - x * d0;
  const double *Fx = Fm + x * dv;
  const float *Yc = Y + j * dmid + z;
  for (int t = to0; t < r; t += tpo) {
    const float *Yt = Yc + t * LD;
    float a = 0.0f;
    for (int y = 0; y < dv; ++y) a = fmaf((float)Fx[y], Yt[y * d0], a);
    const int row = rowpos ? rowpos[t] : t;
    X[row * LD + c] = (first ? 0.0f : X[row * LD + c]) + a;
  }
}

// One launch over n_units work units of the panel classes, as the FP64 panel kernel; fast (atomic) output only.
template <int RP>
__global__ void __launch_bounds__(F32_THREADS, 2) sigma_f32_kernel(DevBasis B, const ClassRec *__restrict__ classes,
                                                                   const WorkUnit *__restrict__ units, int n_units,
                                                                   int *__restrict__ unit_counter, const double *__restrict__ G,
                                                                   SigmaOut out) {
  constexpr int NT = F32_THREADS, LD = f32_ld<RP>(), NC = F32Cfg<RP>::NC;
  extern __shared__ __align__(16) unsigned char f32_smem[];
  ItemState *ist = reinterpret_cast<ItemState *>(f32_smem);
  float *sLU = reinterpret_cast<float *>(ist + PANEL_BMAX);
  float *sW = sLU + RP * RP + RP, *sBK = sW + RP * RP;
  float *PA = sBK + RP * RP, *PB = PA + RP * LD, *PC = PB + RP * LD;
  int *sPerm = reinterpret_cast<int *>(PC + RP * LD);
  __shared__ int s_unit;
  __shared__ ClassRec s_cls;
  __shared__ unsigned long long s_max[PANEL_BMAX];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int e = tid; e < RP * RP; e += NT) {
    sLU[e] = (float)B.LUp[e];
    sW[e] = (float)B.Wp[e];
    sBK[e] = (float)B.BKp[e];
  }
  for (int i = tid; i < RP; i += NT) {
    sLU[RP * RP + i] = (float)B.LUp[RP * RP + i];
    sPerm[i] = B.perm[i];
    sPerm[RP + i] = B.pinv[i];
  }
  const int r = B.r, p = B.p, n = B.n;

  while (true) {
    if (tid == 0) s_unit = atomicAdd(unit_counter, 1);
    __syncthreads();
    const int u = s_unit;
    __syncthreads();
    if (u >= n_units) break;
    const WorkUnit wu = units[u];
    {
      const int *src = reinterpret_cast<const int *>(classes + wu.cls);
      for (int i = tid; i < (int)(sizeof(ClassRec) / sizeof(int)); i += NT) reinterpret_cast<int *>(&s_cls)[i] = src[i];
    }
    __syncthreads();
    const ClassRec &C = s_cls;
    const int m = C.m, vct0 = C.vct0, d0 = C.bdims[0], d1 = C.bdims[1], dout = C.bdims[2 * m];
    const int cap = C.batch, nops = 4 * m - 3, pre = 2 * (vct0 - 1);
    if (path_meets_zero_block(B, C.ind_path, m)) continue;  // uniform: every thread skips the unit

    for (int first = 0; first < wu.count; first += cap) {
      const int nbi = min(cap, wu.count - first);
      // ---- decode the pole tuples (Backbone::set_pole_inds, backbone.cpp:86-150), as the FP64 kernel
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
      float *T = PA, *X = PB, *Y = PC;
      {
        const double *g = G + B.goff[C.ind_path[0]];
        const int dc = d1 * d1, nc = nbi * dc, tpc = NT / nc, c = tid % nc, t0 = tid / nc;
        if (t0 < tpc) {
          const int e = c % dc;
          for (int t = t0; t < r; t += tpc) T[t * LD + c] = (float)g[t * dc + e];
        }
      }
      __syncthreads();
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
        const int *rowpos = (op + 1 < nops && op_kind(op + 1) == 1) ? sPerm + RP : nullptr;
        if (kind == 0) {
          const int line = C.vline[v], b = C.ind_path[v - 1], dv = C.bdims[v], dvp = C.bdims[v + 1];
          const int s = C.vset[v], qo = C.vqo[v], vk = C.vkind[v];
          const long vbase = vk == 0 ? B.F_off[s * B.nb + b] : vk == 1 ? B.Fd_off[s * B.nb + b]
                           : vk == 2 ? B.Fb_off[s * B.nb + b] : B.Fdb_off[s * B.nb + b];
          int ks = 0;
          if (line > 0) {
            const int fwd = (C.fbmask >> line) & 1;
            ks = (v == C.la[line]) ? (fwd ? -1 : 1) : (fwd ? 1 : -1);
          }
          f32_vertex(B, vbase, qo, line, ks, vk >= 2, ist, T, X, rowpos, r, dv, dvp, ncol, nbi, tid, LD);
          __syncthreads();
          float *tmp = T; T = X; X = tmp;
        } else if (kind == 1) {
          const int e = v < vct0 ? v : v - 1;
          const int b = C.ind_path[e];
          const int d = C.bdims[e + 1];
          const int dd = d * d, nc = nbi * d * ncol;
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
          f32_coefs<RP>(sLU, sW, T, X, r, nc, tid);
          __syncthreads();
          f32_qp<NC>(B, ist, T, X, Y, r, d, ncol, nc, warp, lane, LD);
          __syncthreads();
          f32_dual<RP>(sBK, Y, X, T, r, nc, tid, B.tabs);
          __syncthreads();
        } else {
          const int b_mu = C.ind_path[v - 1];
          const int dv = C.bdims[v], dvp = C.bdims[v + 1];
          const bool fwd = C.fbmask & 1;
          const int pk = C.pk;
          const long ok_off = fwd ? B.F_off[pk * B.nb + C.b_out] : B.Fd_off[pk * B.nb + C.b_out];
          const long om_off = fwd ? B.Fd_off[pk * B.nb + b_mu] : B.F_off[pk * B.nb + b_mu];
          const float hs = fwd ? 1.0f : -1.0f;
          int qs = 0;
          for (int i = 0; i < n; ++i)
            if (B.set_to_orb[pk * n + i] >= 0) qs = i + 1;
          if (qs == 0) {
            const int nco = nbi * dvp * d0, tpo = NT / nco, co = tid % nco, to0 = tid / nco;
            if (to0 < tpo)
              for (int t = to0; t < r; t += tpo) X[(rowpos ? rowpos[t] : t) * LD + co] = 0.0f;
            __syncthreads();
          }
          for (int mu = 0; mu < qs; ++mu) {
            const int om = B.set_to_orb[pk * n + mu];
            f32_zv_inner(B, T, Y, r, pk, qs, om, fwd, hs, ok_off, d0, d1, dv, nbi, tid, LD);
            __syncthreads();
            f32_zv_outer(B.ops + om_off + (size_t)mu * dvp * dv, Y, X, rowpos, r, d0, dv, dvp, nbi, tid, mu == 0, LD);
            __syncthreads();
          }
          float *tmp = T; T = X; X = tmp;
        }
      }
      // ---- prefactor and signs, the |T| > 1e-16 guard, accumulation in FP64
      const int dco = dout * d0, nc = nbi * dco;
      {
        const int tpc = NT / nc, c = tid % nc, t0 = tid / nc;
        if (t0 < tpc) {
          const int j = c / dco;
          const double sc = ist[j].scale;
          double mx = 0.0;
          for (int t = t0; t < r; t += tpc) mx = fmax(mx, fabs((double)T[t * LD + c] * sc));
          atomicMax(&s_max[j], (unsigned long long)__double_as_longlong(mx));
        }
      }
      __syncthreads();
      double *dst = out.Sigma + B.goff[C.b_out];
      for (int idx = tid; idx < r * dco; idx += NT) {
        const int t = idx / dco, ee = idx - t * dco;
        double a = 0.0;
        bool keep_any = false;
        for (int j = 0; j < nbi; ++j)
          if (__longlong_as_double((long long)s_max[j]) > 1e-16) {
            a += (double)T[t * LD + j * dco + ee] * ist[j].scale;
            keep_any = true;
          }
        if (keep_any) atomicAdd(dst + idx, out.scale * a);
      }
      __syncthreads();
    }
  }
}

}  // namespace xca
