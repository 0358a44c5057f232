// Sigma backbone evaluation for block chains too wide for a shared-memory panel (plain FP64 path).
//
// The panel kernel (sigma_panel.cuh) keeps a batch of items in shared memory, which bounds an item's widest
// state (rows x columns of its T slab) by the panel width.  Chains through large Fock-space blocks (the
// five-orbital d shell has blocks up to 100 x 100, states of up to 10^4 entries) run here instead: a CTA
// evaluates one item at a time with its T, X and Y slabs (r x widest state each) and one slab per
// zero-vertex operator in a per-CTA region of global memory, the threads striding over output entries.  The steps are those of
// eval_self_energy_fixed_indices (c++/triqs_xca/block_sparse_backbone.cpp:339-367) in the operation order of
// the CPU restatement, as in the panel kernel, so each item's contribution is bit-identical to it:
//   vertex       X(t) = k(t) (F T(t))                   fused multiply-adds over the inner index, then k
// The block products (vertex, zero-vertex operator products, the edge's Q and P') run on the FP64 tensor
// cores (warp_gemm_dmma), whose chains are those of the scalar loops; the r x r DLR steps per column.
//   edge         corr_edge: K^-1 per column (substitution order of getrs), W, Q / P', (beta K) products
//   zero vertex  T(t) F_kappa once per kappa, then Y(t) = sum_kappa (+-h) (T(t) F_kappa); X(t) += F_mu Y(t)
//   prefactor    T *= scale; the 1e-16 guard on max |T|; accumulation (atomics, or the ordered slots).
#pragma once
#include "sigma_kernel.cuh"
#include "spgf_kernel.cuh"

namespace xca {

constexpr int WIDE_THREADS = 256;

// Dynamic shared memory of the wide kernel: LU (+ reciprocal diagonal) | W | BK (column-major, stride RP) |
// perm (RP ints).
template <int RP>
__host__ __device__ constexpr size_t wide_smem_bytes() {
  return (3 * (size_t)RP * RP + RP) * sizeof(double) + RP * sizeof(int);
}

template <int RP>
__global__ void __launch_bounds__(WIDE_THREADS) sigma_wide_kernel(DevBasis B, const ClassRec *__restrict__ classes,
                                                                  const WorkUnit *__restrict__ units, int n_units,
                                                                  int *__restrict__ unit_counter, const double *__restrict__ G,
                                                                  SigmaOut out, double *__restrict__ scratch, long slab,
                                                                  long cta_doubles) {
  extern __shared__ __align__(16) double smem[];
  double *sLU = smem, *sW = sLU + RP * RP + RP, *sBK = sW + RP * RP;
  int *sPerm = reinterpret_cast<int *>(sBK + RP * RP);
  for (int i = threadIdx.x; i < RP * RP + RP; i += blockDim.x) sLU[i] = B.LUp[i];
  for (int i = threadIdx.x; i < RP * RP; i += blockDim.x) {
    sW[i] = B.Wp[i];
    sBK[i] = B.BKp[i];
  }
  for (int i = threadIdx.x; i < RP; i += blockDim.x) sPerm[i] = B.perm[i];
  __shared__ int s_unit;
  __shared__ ClassRec s_cls;
  __shared__ int s_lpole[MAXM], s_caseA[MAXM];
  __shared__ double s_scale;
  __shared__ double s_red[WIDE_THREADS / 32];
  __syncthreads();
  const int r = B.r, p = B.p, n = B.n, tid = threadIdx.x, NT = WIDE_THREADS, warp = tid >> 5, NWARPS = NT / 32;
  double *T0 = scratch + (long)blockIdx.x * cta_doubles;  // T | X | Y | one slab per zero-vertex operator

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
    const int nops = 4 * m - 3, pre = 2 * (vct0 - 1);
    if (path_meets_zero_block(B, C.ind_path, m)) {
      if (out.slots)
        for (int idx = tid; idx < r * dout * d0; idx += NT) out.slots[out.slot_off[u] + idx] = 0.0;
      __syncthreads();
      continue;
    }

    for (int it = 0; it < wu.count; ++it) {
      // ---- pole tuple (Backbone::set_pole_inds, backbone.cpp:86-150), prefactor and signs
      if (tid == 0) {
        int q = wu.first + it;
        for (int i = 0; i < MAXM; ++i) { s_lpole[i] = 0; s_caseA[i] = 0; }
        for (int i = 1; i < m; ++i) { s_lpole[i] = q % p; q /= p; }
        double pf = 1.0;
        int psign = 1;
        for (int i = 1; i < m; ++i) {
          const int fwd = (C.fbmask >> i) & 1;
          const double w = B.polesb[s_lpole[i]];
          s_caseA[i] = fwd ? (w <= 0.0) : (w >= 0.0);
          if (!fwd) psign = -psign;
          const int row = s_caseA[i] ? (fwd ? 1 : 0) : (fwd ? 0 : 1);
          const int ex = s_caseA[i] ? 1 : C.lb[i] - C.la[i] - 1;
          if (ex != 0) pf = mul(pf, B.kpow[((size_t)row * p + s_lpole[i]) * (MAXE + 1) + ex]);
        }
        int dsign = (m % 2 == 0) ? -1 : 1;
        if (!(C.fbmask & 1)) dsign = -dsign;
        s_scale = mul(pf, (double)(psign * dsign));
      }
      double *T = T0, *X = T0 + slab, *Y = T0 + 2 * slab;
      {
        const double *g = G + B.goff[C.ind_path[0]];
        for (int i = tid; i < r * d1 * d1; i += NT) T[i] = g[i];
      }
      __syncthreads();
      for (int op = 0; op < nops; ++op) {
        int v, kind;
        if (op < pre) { v = 1 + op / 2; kind = op & 1; }
        else if (op == pre) { v = vct0; kind = 2; }
        else { v = vct0 + 1 + (op - pre - 1) / 2; kind = ((op - pre - 1) & 1) ? 0 : 1; }
        const int ncol = v < vct0 ? d1 : d0;
        if (kind == 0) {
          // ---- vertex v: X(t) = k(t) F T(t) (multiply_left_vertex with multiply_kernel_on_vertex)
          const int line = C.vline[v], b = C.ind_path[v - 1], dv = C.bdims[v], dvp = C.bdims[v + 1];
          const int s = C.vset[v], qo = C.vqo[v], l = s_lpole[line];
          long off;
          switch (C.vkind[v]) {
            case 0: off = B.F_off[s * B.nb + b] + (long)qo * dvp * dv; break;
            case 1: off = B.Fd_off[s * B.nb + b] + (long)qo * dvp * dv; break;
            case 2: off = B.Fb_off[s * B.nb + b] + ((long)qo * p + l) * dvp * dv; break;
            default: off = B.Fdb_off[s * B.nb + b] + ((long)qo * p + l) * dvp * dv; break;
          }
          const double *F = B.ops + off;
          const double *kt = nullptr;
          if (line > 0 && s_caseA[line]) {
            const int fwd = (C.fbmask >> line) & 1;
            const int ks = (v == C.la[line]) ? (fwd ? -1 : 1) : (fwd ? 1 : -1);
            kt = (ks < 0 ? B.kitm : B.kitp) + l;
          }
          const int per = dvp * ncol;
          const double *Tc = T;
          double *Xc = X;
          warp_gemm_dmma(
              r, dvp, ncol, dv, [&](int, int x, int y) { return F[x * dv + y]; },
              [&](int t, int y, int z) { return Tc[(long)t * dv * ncol + y * ncol + z]; },
              [&](int t, int x, int z, double a) { Xc[(long)t * per + x * ncol + z] = kt ? mul(a, kt[(size_t)t * p]) : a; }, warp,
              NWARPS);
          __syncthreads();
          double *tmp = T; T = X; X = tmp;
        } else if (kind == 1) {
          // ---- edge e: T <- conv(G_b prod K, T) (integrate_left_edge), from the edge tables of G
          const int e = v < vct0 ? v : v - 1, b = C.ind_path[e], d = C.bdims[e + 1], dd = d * d;
          int nf = 0, sg[2] = {0, 0}, lp[2] = {0, 0};
          for (int i = 1; i < m; ++i)
            if (!s_caseA[i] && e >= C.la[i] && e < C.lb[i]) {
              sg[nf] = ((C.fbmask >> i) & 1) ? 0 : 1;
              lp[nf] = s_lpole[i];
              nf++;
            }
          long sig = 0;
          if (nf == 1) sig = 1 + (long)sg[0] * p + lp[0];
          if (nf == 2) sig = 1 + 2L * p + ((long)sg[0] * p + lp[0]) * 2 * p + (long)sg[1] * p + lp[1];
          const double *tb = B.tab + B.tab_off[b] + sig * 2 * r * dd;
          corr_edge<RP, true, true>(B, sLU, sW, sBK, sPerm, tb, d, ncol, d, T, X, Y, tid, NT);
        } else {
          // ---- zero vertex (multiply_left_vertex_and_right_zero_vertex)
          const int b_mu = C.ind_path[v - 1], dv = C.bdims[v], dvp = C.bdims[v + 1];
          const bool fwd = C.fbmask & 1;
          const int pk = C.pk;
          const long ok_off = fwd ? B.F_off[pk * B.nb + C.b_out] : B.Fd_off[pk * B.nb + C.b_out];
          const long om_off = fwd ? B.Fd_off[pk * B.nb + b_mu] : B.F_off[pk * B.nb + b_mu];
          const double hs = fwd ? 1.0 : -1.0;
          int qs = 0;
          for (int i = 0; i < n; ++i)
            if (B.set_to_orb[pk * n + i] >= 0) qs = i + 1;
          if (qs == 0) {
            for (int idx = tid; idx < r * dvp * d0; idx += NT) X[idx] = 0.0;
            __syncthreads();
          }
          // T(t) F_kappa for every kappa once (the same fused multiply-adds as forming it per mu)
          const int per = dv * d0;
          double *TK = T0 + 3 * slab;
          {
            const double *Tc = T, *Fk0 = B.ops + ok_off;
            warp_gemm_dmma(
                qs * r, dv, d0, d1, [&](int e, int x, int y) { return Tc[(long)(e % r) * dv * d1 + x * d1 + y]; },
                [&](int e, int y, int z) { return Fk0[(size_t)(e / r) * d1 * d0 + y * d0 + z]; },
                [&](int e, int x, int z, double a) { TK[(long)(e / r) * slab + (long)(e % r) * per + x * d0 + z] = a; }, warp, NWARPS);
          }
          __syncthreads();
          for (int mu = 0; mu < qs; ++mu) {
            const int om = B.set_to_orb[pk * n + mu];
            for (int idx = tid; idx < r * per; idx += NT) {
              const int t = idx / per;
              double a = 0.0;
              for (int kap = 0; kap < qs; ++kap) {
                const int ok = B.set_to_orb[pk * n + kap];
                const double h = fwd ? B.hval[((size_t)t * n + om) * n + ok] : B.hrefl[((size_t)t * n + ok) * n + om];
                if (h == 0.0) continue;
                a = fmad(mul(hs, h), TK[(long)kap * slab + idx], a);
              }
              Y[idx] = a;
            }
            __syncthreads();
            const double *Fm = B.ops + om_off + (size_t)mu * dvp * dv;
            const int per2 = dvp * d0;
            const double *Yc = Y;
            double *Xc = X;
            warp_gemm_dmma(
                r, dvp, d0, dv, [&](int, int x, int y) { return Fm[x * dv + y]; },
                [&](int t, int y, int z) { return Yc[(long)t * dv * d0 + y * d0 + z]; },
                [&](int t, int x, int z, double a) {
                  double *o = Xc + (long)t * per2 + x * d0 + z;
                  *o = add(mu == 0 ? 0.0 : *o, a);
                },
                warp, NWARPS);
            __syncthreads();
          }
          double *tmp = T; T = X; X = tmp;
        }
      }
      // ---- prefactor and signs, the |T| > 1e-16 guard, accumulation
      const double sc = s_scale;
      const int tot = r * dout * d0;
      double mx = 0.0;
      for (int idx = tid; idx < tot; idx += NT) mx = fmax(mx, fabs(mul(T[idx], sc)));
      mx = warp_max(mx);
      if ((tid & 31) == 0) s_red[tid >> 5] = mx;
      __syncthreads();
      double keep_mx = 0.0;
      for (int w = 0; w < NT / 32; ++w) keep_mx = fmax(keep_mx, s_red[w]);
      const bool keep = keep_mx > 1e-16;
      if (out.slots) {
        double *dst = out.slots + out.slot_off[u];
        for (int idx = tid; idx < tot; idx += NT) {
          double a = it == 0 ? 0.0 : dst[idx];
          if (keep) a = add(a, mul(T[idx], sc));
          dst[idx] = a;
        }
      } else if (keep) {
        double *dst = out.Sigma + B.goff[C.b_out];
        for (int idx = tid; idx < tot; idx += NT) atomicAdd(dst + idx, mul(out.scale, mul(T[idx], sc)));
      }
      __syncthreads();
    }
  }
}

}  // namespace xca
