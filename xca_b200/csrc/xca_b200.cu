// xca_b200: B200-native (sm_100a) pseudo-particle strong-coupling hot path behind a C-ABI.
//
// Device data layout (HBM): every block Green's function is one packed slab of real FP64, block b an
// (r, d_b, d_b) array at offset goff[b]; the field operators of every symmetry set are packed slabs
// (q_s, d_target, d_b) per present block column, and the barred operators (q_s, p, d_target, d_b).
// The DLR basis matrices (LU of K(t_i, om_l), the Hilbert weights W, K(t_i, om_l)) live in global
// memory and are staged into shared memory by every block of the Sigma kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/xca_b200.h"
#include "dlr_host.hpp"
#include "sigma_kernel.cuh"

namespace xca {

thread_local std::string g_err;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CUDA_CHECK(x)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) throw Error(XCA_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
struct DevBuf {
  T *ptr = nullptr;
  size_t n = 0;
  void resize(size_t count) {
    if (count <= n && ptr) return;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
    if (count == 0) return;
    CUDA_CHECK(cudaMalloc(&ptr, count * sizeof(T)));
    n = count;
  }
  void upload(const std::vector<T> &v, cudaStream_t s) {
    resize(std::max<size_t>(v.size(), 1));
    if (!v.empty()) CUDA_CHECK(cudaMemcpyAsync(ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
};

// -------------------------------------------------------------------------------- Sigma kernel
// Dynamic shared memory: [LU | W | Kit] (3 r^2 doubles) | piv (r ints, padded) | per-warp NBUF slabs of
// r * nmax^2 doubles.
__global__ void __launch_bounds__(256) sigma_items_kernel(DevBasis B, const ClassRec *__restrict__ classes,
                                                          const WorkUnit *__restrict__ units, int n_units,
                                                          int *__restrict__ unit_counter, const double *__restrict__ G,
                                                          double *__restrict__ Sigma, double scale) {
  extern __shared__ double smem[];
  const int r = B.r, p = B.p, n = B.n;
  const int r2 = r * r;
  double *sLU = smem;
  double *sW = sLU + r2;
  double *sK = sW + r2;
  int *sPiv = reinterpret_cast<int *>(sK + r2);
  const int pivpad = (r + 1) / 2;  // doubles occupied by r ints
  double *warp_base = sK + r2 + pivpad;
  for (int i = threadIdx.x; i < r2; i += blockDim.x) {
    sLU[i] = B.LU[i];
    sW[i] = B.W[i];
    sK[i] = B.Kit[i];
  }
  for (int i = threadIdx.x; i < r; i += blockDim.x) sPiv[i] = B.piv[i];
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int slab = r * B.nmax * B.nmax;
  double *bufA = warp_base + (size_t)warp * NBUF * slab;
  double *bufB = bufA + slab, *bufC = bufB + slab, *bufD = bufC + slab, *bufE = bufD + slab, *acc = bufE + slab;

  while (true) {
    int u = 0;
    if (lane == 0) u = atomicAdd(unit_counter, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= n_units) break;
    const WorkUnit wu = units[u];
    const ClassRec &C = classes[wu.cls];
    const int m = C.m, vct0 = C.vct0;
    const int d0 = C.bdims[0], d1 = C.bdims[1];
    const int dout = C.bdims[2 * m];
    for (int i = lane; i < r * dout * d0; i += 32) acc[i] = 0.0;
    bool any = false;

    for (int it = 0; it < wu.count; ++it) {
      int p_ix = wu.first + it;
      // ---- decode the pole tuple (Backbone::set_pole_inds, backbone.cpp:86-150)
      int lpole[MAXM] = {0, 0, 0};
      int caseA[MAXM] = {0, 0, 0};
      {
        int q = p_ix;
        for (int i = 1; i < m; ++i) {
          lpole[i] = q % p;
          q /= p;
        }
      }
      double pf = 1.0;
      int psign = 1;
      for (int i = 1; i < m; ++i) {
        int fwd = (C.fbmask >> i) & 1;
        double w = B.polesb[lpole[i]];
        caseA[i] = fwd ? (w <= 0.0) : (w >= 0.0);
        if (!fwd) psign = -psign;
        // prefactor *= pow(K^{+-}_l(0), -exp) in line order (Hybridization::multiply_kernels_prefactor)
        int row = caseA[i] ? (fwd ? 1 : 0) : (fwd ? 0 : 1);
        int ex = caseA[i] ? 1 : C.lb[i] - C.la[i] - 1;
        if (ex != 0) pf = mul(pf, B.kpow[((size_t)row * p + lpole[i]) * (MAXE + 1) + ex]);
      }
      int dsign = (m % 2 == 0) ? -1 : 1;
      if (!(C.fbmask & 1)) dsign = -dsign;
      const double total_scale = mul(pf, (double)(psign * dsign));

      // ---- T := G[ind_path[0]]  (d1 x d1)
      double *T = bufA, *S = bufB;
      {
        const double *g = G + B.goff[C.ind_path[0]];
        for (int i = lane; i < r * d1 * d1; i += 32) T[i] = g[i];
      }
      __syncwarp();

      // vertex multiply: T(t) <- k(t) * F * T(t) (multiply_left_vertex)
      auto vertex = [&](int v, int ncol) {
        const int line = C.vline[v];
        const int l = lpole[line];
        const int b = C.ind_path[v - 1];
        const int dv = C.bdims[v], dvp = C.bdims[v + 1];
        const int s = C.vset[v], qo = C.vqo[v];
        const double *F;
        switch (C.vkind[v]) {
          case 0: F = B.ops + B.F_off[s * B.nb + b] + (size_t)qo * dvp * dv; break;
          case 1: F = B.ops + B.Fd_off[s * B.nb + b] + (size_t)qo * dvp * dv; break;
          case 2: F = B.ops + B.Fb_off[s * B.nb + b] + ((size_t)qo * p + l) * dvp * dv; break;
          default: F = B.ops + B.Fdb_off[s * B.nb + b] + ((size_t)qo * p + l) * dvp * dv; break;
        }
        // K factor on this vertex: lines in case A carry K on both endpoints
        const double *kcol = nullptr;
        if (line > 0 && caseA[line]) {
          int fwd = (C.fbmask >> line) & 1;
          int ks = (v == C.la[line]) ? (fwd ? -1 : 1) : (fwd ? 1 : -1);
          kcol = (ks > 0 ? B.kitp : B.kitm) + l;
        }
        const int tot = r * dvp * ncol;
        for (int idx = lane; idx < tot; idx += 32) {
          int t = idx / (dvp * ncol);
          int rem = idx - t * dvp * ncol;
          int x = rem / ncol, z = rem - x * ncol;
          const double *Tt = T + t * dv * ncol;
          double sacc = 0.0;
          for (int y = 0; y < dv; ++y) sacc = add(sacc, mul(F[x * dv + y], Tt[y * ncol + z]));
          if (kcol) sacc = mul(sacc, kcol[(size_t)t * p]);
          S[idx] = sacc;
        }
        __syncwarp();
        double *tmp = T; T = S; S = tmp;
      };

      // edge e: T <- conv(G_b * prod K, T)  (integrate_left_edge + cppdlr time-ordered convolution)
      auto edge = [&](int e, int ncol) {
        const int b = C.ind_path[e];
        const int d = C.bdims[e + 1];
        const double *g = G + B.goff[b];
        // GK into S with the edge's K factors (lines in case B cover edges la..lb-1)
        const int dd = d * d;
        for (int idx = lane; idx < r * dd; idx += 32) {
          int t = idx / dd;
          double v = g[idx];
          for (int i = 1; i < m; ++i) {
            if (!caseA[i] && e >= C.la[i] && e < C.lb[i]) {
              int fwd = (C.fbmask >> i) & 1;
              v = mul(v, (fwd ? B.kitp : B.kitm)[(size_t)t * p + lpole[i]]);
            }
          }
          S[idx] = v;
        }
        __syncwarp();
        // coefficients: fc = K^{-1} GK (in S), gc = K^{-1} T (in T)
        lu_solve_cols(sLU, sPiv, r, S, dd, lane);
        lu_solve_cols(sLU, sPiv, r, T, d * ncol, lane);
        __syncwarp();
        // Hilbert sums: Ft = W fc (bufC/bufD as free scratch), Gt = W gc
        double *Ft = (S == bufA || T == bufA) ? ((S == bufB || T == bufB) ? bufC : bufB) : bufA;
        // pick three free slabs among A..E not equal to S or T
        double *freeb[5] = {bufA, bufB, bufC, bufD, bufE};
        double *fr[3];
        int nf = 0;
        for (int k = 0; k < 5 && nf < 3; ++k)
          if (freeb[k] != S && freeb[k] != T) fr[nf++] = freeb[k];
        Ft = fr[0];
        double *Gt = fr[1], *Q = fr[2];
        matvec_cols(sW, r, S, Ft, dd, lane);
        matvec_cols(sW, r, T, Gt, d * ncol, lane);
        __syncwarp();
        // Q_l = Ft_l gc_l + fc_l Gt_l
        const int dc = d * ncol;
        for (int idx = lane; idx < r * dc; idx += 32) {
          int l = idx / dc;
          int rem = idx - l * dc;
          int x = rem / ncol, z = rem - x * ncol;
          const double *fl = S + l * dd, *ftl = Ft + l * dd, *gl = T + l * dc, *gtl = Gt + l * dc;
          double s = 0.0;
          for (int y = 0; y < d; ++y) s = add(s, add(mul(ftl[x * d + y], gl[y * ncol + z]), mul(fl[x * d + y], gtl[y * ncol + z])));
          Q[idx] = s;
        }
        __syncwarp();
        // P_l = fc_l gc_l  (into Ft, no longer needed)
        for (int idx = lane; idx < r * dc; idx += 32) {
          int l = idx / dc;
          int rem = idx - l * dc;
          int x = rem / ncol, z = rem - x * ncol;
          const double *fl = S + l * dd, *gl = T + l * dc;
          double s = 0.0;
          for (int y = 0; y < d; ++y) s = add(s, mul(fl[x * d + y], gl[y * ncol + z]));
          Ft[idx] = s;
        }
        __syncwarp();
        // h(t_i) = sum_l (beta K(t_i, om_l)) (Q_l + (t_i K(0, om_l)) P_l)  -> written into Gt, becomes T
        for (int idx = lane; idx < r * dc; idx += 32) {
          int i = idx / dc;
          int c = idx - i * dc;
          const double *kr = sK + i * r;
          double ti = B.tabs[i];
          double s = 0.0;
          for (int l = 0; l < r; ++l)
            s = add(s, mul(mul(B.beta, kr[l]), add(Q[l * dc + c], mul(mul(ti, B.k0[l]), Ft[l * dc + c]))));
          Gt[idx] = s;
        }
        __syncwarp();
        T = Gt;
        // S: any slab that is not T
        S = (T == bufA) ? bufB : bufA;
      };

      for (int v = 1; v < vct0; ++v) {
        vertex(v, d1);
        edge(v, d1);
      }
      // ---- zero vertex (multiply_left_vertex_and_right_zero_vertex)
      {
        const int v = vct0;
        const int b_mu = C.ind_path[v - 1];
        const int dv = C.bdims[v], dvp = C.bdims[v + 1];
        const bool fwd = C.fbmask & 1;
        const int pk = C.pk;
        const long ok_off = fwd ? B.F_off[pk * B.nb + C.b_out] : B.Fd_off[pk * B.nb + C.b_out];
        const long om_off = fwd ? B.Fd_off[pk * B.nb + b_mu] : B.F_off[pk * B.nb + b_mu];
        const double hs = fwd ? 1.0 : -1.0;
        // set size: count orbitals of set pk
        int qs = 0;
        for (int i = 0; i < n; ++i)
          if (B.set_to_orb[pk * n + i] >= 0) qs = i + 1;
        double *X = (S == bufC || T == bufC) ? bufD : bufC;
        if (X == S || X == T) X = bufE;
        for (int i = lane; i < r * dvp * d0; i += 32) S[i] = 0.0;
        __syncwarp();
        for (int mu = 0; mu < qs; ++mu) {
          const int om = B.set_to_orb[pk * n + mu];
          // X(t) = sum_kap hs Delta_{mu kap}(t) T(t) F_kap
          for (int idx = lane; idx < r * dv * d0; idx += 32) {
            int t = idx / (dv * d0);
            int rem = idx - t * dv * d0;
            int x = rem / d0, z = rem - x * d0;
            const double *Tt = T + t * dv * d1;
            double s = 0.0;
            for (int kap = 0; kap < qs; ++kap) {
              const int ok = B.set_to_orb[pk * n + kap];
              double h = fwd ? B.hval[((size_t)t * n + om) * n + ok] : B.hrefl[((size_t)t * n + ok) * n + om];
              if (h == 0.0) continue;
              const double *Fk = B.ops + ok_off + (size_t)kap * d1 * d0;
              double tf = 0.0;
              for (int y = 0; y < d1; ++y) tf = add(tf, mul(Tt[x * d1 + y], Fk[y * d0 + z]));
              s = add(s, mul(mul(hs, h), tf));
            }
            X[idx] = s;
          }
          __syncwarp();
          const double *Fm = B.ops + om_off + (size_t)mu * dvp * dv;
          for (int idx = lane; idx < r * dvp * d0; idx += 32) {
            int t = idx / (dvp * d0);
            int rem = idx - t * dvp * d0;
            int x = rem / d0, z = rem - x * d0;
            double s = 0.0;
            for (int y = 0; y < dv; ++y) s = add(s, mul(Fm[x * dv + y], X[t * dv * d0 + y * d0 + z]));
            S[idx] = add(S[idx], s);
          }
          __syncwarp();
        }
        double *tmp = T; T = S; S = tmp;
      }
      for (int v = vct0 + 1; v < 2 * m; ++v) {
        edge(v - 1, d0);
        vertex(v, d0);
      }
      // ---- prefactor, sign and the |T| > 1e-16 guard, then accumulate
      {
        const int tot = r * dout * d0;
        double mx = 0.0;
        for (int i = lane; i < tot; i += 32) mx = fmax(mx, fabs(mul(T[i], total_scale)));
        mx = warp_max(mx);
        if (mx > 1e-16) {
          for (int i = lane; i < tot; i += 32) acc[i] = add(acc[i], mul(T[i], total_scale));
          any = true;
        }
        __syncwarp();
      }
    }
    if (any) {
      double *dst = Sigma + B.goff[C.b_out];
      for (int i = lane; i < r * dout * d0; i += 32) atomicAdd(dst + i, mul(scale, acc[i]));
    }
    __syncwarp();
  }
}

__global__ void block_maxabs_kernel(const double *G, const long *goff, const int *dims, int r, int nb, double *out) {
  int b = blockIdx.x;
  if (b >= nb) return;
  long n = (long)r * dims[b] * dims[b];
  double mx = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fabs(G[goff[b] + i]));
  __shared__ double red[256];
  red[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[b] = red[0];
}

__global__ void zero_kernel(double *x, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) x[i] = 0.0;
}

// -------------------------------------------------------------------------------- host context
struct Topology {
  int m;
  int t[MAXM][2];
};

struct ClassSet {
  std::vector<ClassRec> classes;
  std::vector<WorkUnit> units;
  DevBuf<ClassRec> d_classes;
  DevBuf<WorkUnit> d_units;
  // item order for the reference's flat-index walk: per (fb_ix, o_ix) the classes in (b, pk) order
  std::vector<std::vector<int>> by_fbo;
  long long n_items = 0;
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  long launches = 0;
  bool ready = false;
  // model
  int r = 0, p = 0, n = 0, nb = 0, nq = 0, nmax = 0;
  double beta = 0, lam = 0, eps = 0;
  std::vector<double> rf, it, tabs, k0, polesb;
  std::vector<int> dims;
  std::vector<long> goff;
  long slab = 0;
  std::vector<long> labels, sinds, ssizes;
  std::vector<int> set_to_orb;
  std::vector<int> F_idx, Fd_idx;
  std::vector<long> F_off, Fd_off, Fb_off, Fdb_off;
  std::vector<double> ops;
  std::vector<double> hval, hrefl, kitp, kitm, k0p, k0m, kpow;
  std::vector<double> LU, W, Kit;
  std::vector<int> piv;
  // device copies
  DevBuf<double> d_LU, d_W, d_Kit, d_tabs, d_k0, d_kitp, d_kitm, d_k0p, d_k0m, d_kpow, d_polesb, d_hval, d_hrefl, d_ops;
  DevBuf<int> d_piv, d_dims, d_set_to_orb;
  DevBuf<long> d_goff, d_F_off, d_Fd_off, d_Fb_off, d_Fdb_off;
  DevBuf<int> d_counter;
  DevBuf<double> d_G, d_Sig, d_maxabs;
  std::vector<std::unique_ptr<DevBuf<double>>> user_bufs;
  std::map<std::string, std::unique_ptr<ClassSet>> class_cache;
  int unit_size = 16;

  DevBasis basis() const {
    DevBasis B;
    B.r = r; B.p = p; B.n = n; B.nb = nb; B.nq = nq; B.nmax = nmax; B.beta = beta;
    B.LU = d_LU.ptr; B.piv = d_piv.ptr; B.W = d_W.ptr; B.Kit = d_Kit.ptr; B.tabs = d_tabs.ptr; B.k0 = d_k0.ptr;
    B.kitp = d_kitp.ptr; B.kitm = d_kitm.ptr; B.k0p = d_k0p.ptr; B.k0m = d_k0m.ptr; B.kpow = d_kpow.ptr; B.polesb = d_polesb.ptr;
    B.hval = d_hval.ptr; B.hrefl = d_hrefl.ptr; B.goff = d_goff.ptr; B.dims = d_dims.ptr; B.ops = d_ops.ptr;
    B.F_off = d_F_off.ptr; B.Fd_off = d_Fd_off.ptr; B.Fb_off = d_Fb_off.ptr; B.Fdb_off = d_Fdb_off.ptr;
    B.set_to_orb = d_set_to_orb.ptr;
    return B;
  }
};

static void set_device(Ctx *c) { CUDA_CHECK(cudaSetDevice(c->device)); }

static Topology parse_topology(int m, const int *topo) {
  if (m < 1 || m > MAXM) throw Error(XCA_ERR_UNSUPPORTED, "topology order " + std::to_string(m) + " not supported (1..3)");
  Topology T;
  T.m = m;
  for (int i = 0; i < m; ++i) {
    T.t[i][0] = topo[2 * i];
    T.t[i][1] = topo[2 * i + 1];
    if (T.t[i][0] >= T.t[i][1]) throw Error(XCA_ERR_INVALID, "first row of topology must contain smaller-numbered vertices");
    if (T.t[i][1] >= 2 * m || T.t[i][0] < 0) throw Error(XCA_ERR_INVALID, "topology vertex out of range");
  }
  if (T.t[0][0] != 0) throw Error(XCA_ERR_INVALID, "topology(0,0) must be 0");
  return T;
}

static long ipow(long a, int e) {
  long r = 1;
  for (int i = 0; i < e; ++i) r *= a;
  return r;
}

// K0 work-list builder: path classes of find_path_self_energy (block_sparse_backbone.cpp:229-314).
// Validity of a block path depends on the directions, the orbital tuple, the output block, the
// symmetry set and the zero-block flags of G, never on the pole tuple, so it is enumerated once per
// (topology, zero pattern) and every valid path class stands for p^(m-1) items.
static ClassSet *get_classes(Ctx *c, const Topology &T, const std::vector<int> &zero) {
  std::ostringstream key;
  key << T.m;
  for (int i = 0; i < T.m; ++i) key << ":" << T.t[i][0] << "," << T.t[i][1];
  key << "|";
  for (int z : zero) key << (z ? '0' : '1');
  auto itc = c->class_cache.find(key.str());
  if (itc != c->class_cache.end()) return itc->second.get();
  auto cs = std::make_unique<ClassSet>();
  const int m = T.m, nv = 2 * m, vct0 = T.t[0][1];
  const long fbmax = 1L << m, omax = ipow(c->n, m - 1);
  const long npt = ipow(c->p, m - 1);
  if (npt > INT32_MAX) throw Error(XCA_ERR_UNSUPPORTED, "too many pole tuples");
  cs->by_fbo.resize(fbmax * omax);
  for (long fb = 0; fb < fbmax; ++fb)
    for (long o = 0; o < omax; ++o) {
      int fbv[MAXM];
      long q = fb;
      for (int i = 0; i < m; ++i) { fbv[i] = q % 2; q /= 2; }
      int dag[MAXV] = {0}, bar[MAXV] = {0}, orb[MAXV], vline[MAXV];
      for (int v = 0; v < nv; ++v) { orb[v] = -1; vline[v] = 0; }
      // set_directions (backbone.cpp:35-76)
      if (fbv[0] == 1) { dag[0] = 0; dag[T.t[0][1]] = 1; } else { dag[0] = 1; dag[T.t[0][1]] = 0; }
      for (int i = 1; i < m; ++i) {
        bar[T.t[i][0]] = 0; bar[T.t[i][1]] = 1;
        if (fbv[i] == 1) { dag[T.t[i][0]] = 0; dag[T.t[i][1]] = 1; } else { dag[T.t[i][0]] = 1; dag[T.t[i][1]] = 0; }
        vline[T.t[i][0]] = i; vline[T.t[i][1]] = i;
      }
      // set_orb_inds (backbone.cpp:165-186)
      long oq = o;
      for (int i = 1; i < m; ++i) {
        int ov = (int)(oq % c->n);
        oq /= c->n;
        orb[T.t[i][0]] = ov;
        orb[T.t[i][1]] = ov;
      }
      auto idx_of = [&](int v, int set, int b) -> int {
        return dag[v] ? c->Fd_idx[set * c->nb + b] : c->F_idx[set * c->nb + b];
      };
      for (int b = 0; b < c->nb; ++b)
        for (int pk = 0; pk < c->nq; ++pk) {
          int path[2 * MAXM], bd[2 * MAXM + 1];
          bool bad = false;
          int ip = -1;
          for (int v = 0; v < vct0; ++v) {
            int set = (v == 0) ? pk : (int)c->labels[orb[v]];
            ip = idx_of(v, set, v == 0 ? b : ip);
            bad = (ip == -1) || (v < nv - 1 && zero[ip]);
            if (bad) break;
            path[v] = ip;
          }
          if (bad) continue;
          bd[0] = c->dims[b];
          bd[1] = c->dims[idx_of(0, pk, b)];
          for (int v = 0; v < vct0 - 1; ++v) bd[v + 2] = c->dims[idx_of(v + 1, (int)c->labels[orb[v + 1]], path[v])];
          ip = path[vct0 - 1];
          for (int v = vct0; v < nv; ++v) {
            int set = (v == vct0) ? pk : (int)c->labels[orb[v]];
            ip = idx_of(v, set, ip);
            bad = (ip == -1) || (v < nv - 1 && zero[ip]);
            if (bad) break;
            if (v < nv - 1) path[v] = ip;
          }
          if (bad) continue;
          bd[vct0 + 1] = c->dims[idx_of(vct0, pk, path[vct0 - 1])];
          for (int v = vct0; v < nv - 1; ++v) bd[v + 2] = c->dims[idx_of(v + 1, (int)c->labels[orb[v + 1]], path[v])];
          if (bd[nv] != c->dims[b] || bd[0] != c->dims[b])
            throw Error(XCA_ERR_INVALID, "BlockDiagOpFun::add_block: contribution shape does not match block " + std::to_string(b));
          ClassRec R;
          std::memset(&R, 0, sizeof(R));
          R.m = m; R.vct0 = vct0; R.b_out = b; R.pk = pk; R.npt = (int)npt;
          R.fbmask = 0;
          for (int i = 0; i < m; ++i) R.fbmask |= fbv[i] << i;
          for (int i = 0; i < m; ++i) { R.la[i] = T.t[i][0]; R.lb[i] = T.t[i][1]; }
          for (int i = 0; i < nv - 1; ++i) R.ind_path[i] = path[i];
          for (int i = 0; i <= nv; ++i) R.bdims[i] = bd[i];
          for (int v = 0; v < nv; ++v) {
            R.vline[v] = vline[v];
            if (v == 0 || v == vct0) { R.vkind[v] = 0; R.vset[v] = pk; R.vqo[v] = 0; continue; }
            R.vkind[v] = bar[v] ? (dag[v] ? 3 : 2) : (dag[v] ? 1 : 0);
            R.vset[v] = (int)c->labels[orb[v]];
            R.vqo[v] = (int)c->sinds[orb[v]];
          }
          cs->by_fbo[fb * omax + o].push_back((int)cs->classes.size());
          cs->classes.push_back(R);
        }
    }
  for (size_t k = 0; k < cs->classes.size(); ++k) {
    for (long s = 0; s < npt; s += c->unit_size) {
      WorkUnit u;
      u.cls = (int)k;
      u.first = (int)s;
      u.count = (int)std::min<long>(c->unit_size, npt - s);
      cs->units.push_back(u);
    }
  }
  cs->n_items = (long long)cs->classes.size() * npt;
  cs->d_classes.upload(cs->classes, c->stream);
  cs->d_units.upload(cs->units, c->stream);
  ClassSet *ret = cs.get();
  c->class_cache[key.str()] = std::move(cs);
  return ret;
}

static size_t sigma_smem_bytes(const Ctx *c, int warps) {
  size_t base = (size_t)3 * c->r * c->r + (c->r + 1) / 2;
  size_t per = (size_t)NBUF * c->r * c->nmax * c->nmax;
  return (base + per * warps) * sizeof(double);
}

static int sigma_warps(const Ctx *c) {
  int dev = c->device;
  int maxsm = 0;
  cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  int w = 8;
  while (w > 1 && sigma_smem_bytes(c, w) > (size_t)maxsm) --w;
  if (sigma_smem_bytes(c, w) > (size_t)maxsm)
    throw Error(XCA_ERR_UNSUPPORTED, "block dimension too large for the shared-memory Sigma kernel (nmax = " + std::to_string(c->nmax) + ")");
  return w;
}

static std::vector<int> zero_flags_device(Ctx *c, const double *G_dev) {
  c->d_maxabs.resize(c->nb);
  block_maxabs_kernel<<<c->nb, 256, 0, c->stream>>>(G_dev, c->d_goff.ptr, c->d_dims.ptr, c->r, c->nb, c->d_maxabs.ptr);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
  std::vector<double> mx(c->nb);
  CUDA_CHECK(cudaMemcpyAsync(mx.data(), c->d_maxabs.ptr, c->nb * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  std::vector<int> z(c->nb);
  for (int b = 0; b < c->nb; ++b) z[b] = mx[b] < 1e-16 ? 1 : 0;
  return z;
}

static void launch_sigma(Ctx *c, ClassSet *cs, const double *G_dev, double *Sig_dev, double scale) {
  if (cs->units.empty()) return;
  int warps = sigma_warps(c);
  size_t smem = sigma_smem_bytes(c, warps);
  CUDA_CHECK(cudaFuncSetAttribute(sigma_items_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  c->d_counter.resize(1);
  CUDA_CHECK(cudaMemsetAsync(c->d_counter.ptr, 0, sizeof(int), c->stream));
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  int grid = std::max(1, std::min<int>(nsm, (int)((cs->units.size() + warps - 1) / warps)));
  sigma_items_kernel<<<grid, 32 * warps, smem, c->stream>>>(c->basis(), cs->d_classes.ptr, cs->d_units.ptr, (int)cs->units.size(),
                                                           c->d_counter.ptr, G_dev, Sig_dev, scale);
  c->launches++;
  CUDA_CHECK(cudaGetLastError());
}

// real part of a host complex slab, rejecting non-zero imaginary parts
static void real_part(const double *cplx, long n, std::vector<double> &out, const char *what) {
  out.resize(n);
  for (long i = 0; i < n; ++i) {
    if (cplx[2 * i + 1] != 0.0)
      throw Error(XCA_ERR_UNSUPPORTED, std::string(what) + " has a non-zero imaginary part; the device path computes in real FP64");
    out[i] = cplx[2 * i];
  }
}

}  // namespace xca

using namespace xca;

#define API_BEGIN try {
#define API_END                                     \
  return XCA_OK;                                    \
  }                                                 \
  catch (const Error &e) {                          \
    g_err = e.what();                               \
    return e.code;                                  \
  }                                                 \
  catch (const std::invalid_argument &e) {          \
    g_err = e.what();                               \
    return XCA_ERR_INVALID;                         \
  }                                                 \
  catch (const std::exception &e) {                 \
    g_err = e.what();                               \
    return XCA_ERR_RUNTIME;                         \
  }

extern "C" {

const char *xca_last_error(void) { return g_err.c_str(); }

int xca_abi_version(void) { return 1; }

int xca_dlr_build_rf(double lambda, double eps, double *rf_out, int max_r, int *r_out) {
  API_BEGIN
  if (!(lambda > 0) || !(eps > 0)) throw Error(XCA_ERR_INVALID, "Lambda and eps must be positive");
  auto rf = build_dlr_rf(lambda, eps);
  *r_out = (int)rf.size();
  if ((int)rf.size() > max_r) throw Error(XCA_ERR_INVALID, "rf_out too small: rank " + std::to_string(rf.size()));
  std::copy(rf.begin(), rf.end(), rf_out);
  API_END
}

int xca_dlr_build_it(double lambda, const double *rf, int r, double *it_out) {
  API_BEGIN
  std::vector<double> v(rf, rf + r);
  auto it = build_dlr_it(lambda, v);
  std::copy(it.begin(), it.end(), it_out);
  API_END
}

int xca_ctx_create(int device, xca_ctx **out) {
  API_BEGIN
  auto *c = new Ctx();
  c->device = device;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    delete c;
    throw Error(XCA_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  }
  set_device(c);
  CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  *out = reinterpret_cast<xca_ctx *>(c);
  API_END
}

int xca_ctx_destroy(xca_ctx *ctx) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c) return XCA_OK;
  set_device(c);
  cudaStreamSynchronize(c->stream);
  cudaStream_t s = c->stream;
  delete c;
  if (s) cudaStreamDestroy(s);
  API_END
}

int xca_evaluator_setup(xca_ctx *ctx, double beta, double lambda, double eps, int r, const double *rf, const double *it, int p,
                        const double *hyb_poles, const double *hyb_coeffs, int n, const long *labels, int n_blocks,
                        const int *block_dims, const int *F_index, const double *F_data, const int *Fd_index, const double *Fd_data) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (r <= 0 || p <= 0 || n <= 0 || n_blocks <= 0) throw Error(XCA_ERR_INVALID, "empty basis, hybridization or block structure");
  c->r = r; c->p = p; c->n = n; c->nb = n_blocks; c->beta = beta; c->lam = lambda; c->eps = eps;
  c->rf.assign(rf, rf + r);
  c->it.assign(it, it + r);
  c->dims.assign(block_dims, block_dims + n_blocks);
  c->labels.assign(labels, labels + n);
  long nq = 0;
  for (int i = 0; i < n; ++i) {
    if (labels[i] < 0) throw Error(XCA_ERR_INVALID, "negative symmetry-set label");
    nq = std::max(nq, labels[i] + 1);
  }
  c->nq = (int)nq;
  c->sinds.assign(n, 0); c->ssizes.assign(nq, 0); c->set_to_orb.assign((size_t)nq * n, -1);
  for (int i = 0; i < n; ++i) {
    c->sinds[i] = c->ssizes[labels[i]];
    c->set_to_orb[(size_t)labels[i] * n + c->sinds[i]] = i;
    c->ssizes[labels[i]]++;
  }
  for (long s = 0; s < nq; ++s)
    if (c->ssizes[s] == 0) throw Error(XCA_ERR_INVALID, "BlockOpSymQuartet: symmetry set " + std::to_string(s) + " has no orbital");
  c->nmax = 1;
  for (int b = 0; b < n_blocks; ++b) {
    if (block_dims[b] <= 0) throw Error(XCA_ERR_INVALID, "block dimension must be positive");
    c->nmax = std::max(c->nmax, block_dims[b]);
  }
  c->goff.resize(n_blocks);
  long off = 0;
  for (int b = 0; b < n_blocks; ++b) { c->goff[b] = off; off += (long)r * block_dims[b] * block_dims[b]; }
  c->slab = off;
  // hybridization coefficients: real part, block-diagonality in the symmetry sets (block_sparse.cpp:443-492)
  std::vector<double> coef;
  real_part(hyb_coeffs, (long)p * n * n, coef, "hyb_coeffs");
  double mx = 0;
  for (double x : coef) mx = std::max(mx, std::fabs(x));
  if (!std::isfinite(mx)) throw Error(XCA_ERR_INVALID, "DiagramEvaluator: hyb_coeffs contains a non-finite entry");
  for (int l = 0; l < p; ++l)
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        if (labels[i] != labels[j] && std::fabs(coef[((size_t)l * n + i) * n + j]) > 1e-12 * mx)
          throw Error(XCA_ERR_INVALID, "DiagramEvaluator: hyb_coeffs couples different symmetry sets, which the symmetry-set storage cannot represent");
  // operators: F, F^dag slabs, then the barred operators (BlockOpSymQuartet, block_sparse.cpp:555-576)
  c->F_idx.assign(F_index, F_index + nq * n_blocks);
  c->Fd_idx.assign(Fd_index, Fd_index + nq * n_blocks);
  c->ops.clear();
  c->F_off.assign(nq * n_blocks, -1); c->Fd_off.assign(nq * n_blocks, -1);
  c->Fb_off.assign(nq * n_blocks, -1); c->Fdb_off.assign(nq * n_blocks, -1);
  auto load = [&](const std::vector<int> &idx, const double *data, std::vector<long> &offs, const char *what) {
    long pos = 0;
    for (long s = 0; s < nq; ++s)
      for (int b = 0; b < n_blocks; ++b) {
        int tg = idx[s * n_blocks + b];
        if (tg < -1 || tg >= n_blocks) throw Error(XCA_ERR_INVALID, std::string(what) + ": block index out of range");
        if (tg < 0) continue;
        long sz = c->ssizes[s] * block_dims[tg] * block_dims[b];
        offs[s * n_blocks + b] = (long)c->ops.size();
        std::vector<double> re;
        real_part(data + 2 * pos, sz, re, what);
        c->ops.insert(c->ops.end(), re.begin(), re.end());
        pos += sz;
      }
  };
  load(c->F_idx, F_data, c->F_off, "F");
  load(c->Fd_idx, Fd_data, c->Fd_off, "F_dag");
  for (long s = 0; s < nq; ++s) {
    long q = c->ssizes[s];
    for (int b = 0; b < n_blocks; ++b) {
      if (c->Fd_idx[s * n_blocks + b] >= 0) {
        long bs = (long)block_dims[c->Fd_idx[s * n_blocks + b]] * block_dims[b];
        c->Fdb_off[s * n_blocks + b] = (long)c->ops.size();
        c->ops.resize(c->ops.size() + q * p * bs, 0.0);
      }
      if (c->F_idx[s * n_blocks + b] >= 0) {
        long bs = (long)block_dims[c->F_idx[s * n_blocks + b]] * block_dims[b];
        c->Fb_off[s * n_blocks + b] = (long)c->ops.size();
        c->ops.resize(c->ops.size() + q * p * bs, 0.0);
      }
    }
    for (int l = 0; l < p; ++l)
      for (long lam = 0; lam < q; ++lam)
        for (long nu = 0; nu < q; ++nu) {
          int lo = c->set_to_orb[s * n + lam], no = c->set_to_orb[s * n + nu];
          double cf = coef[((size_t)l * n + no) * n + lo];
          if (cf == 0.0) continue;
          for (int b = 0; b < n_blocks; ++b) {
            if (c->Fd_idx[s * n_blocks + b] >= 0) {
              long bs = (long)block_dims[c->Fd_idx[s * n_blocks + b]] * block_dims[b];
              double *dst = c->ops.data() + c->Fdb_off[s * n_blocks + b] + ((size_t)lam * p + l) * bs;
              const double *src = c->ops.data() + c->Fd_off[s * n_blocks + b] + (size_t)nu * bs;
              for (long x = 0; x < bs; ++x) dst[x] += cf * src[x];
            }
            if (c->F_idx[s * n_blocks + b] >= 0) {
              long bs = (long)block_dims[c->F_idx[s * n_blocks + b]] * block_dims[b];
              double *dst = c->ops.data() + c->Fb_off[s * n_blocks + b] + ((size_t)nu * p + l) * bs;
              const double *src = c->ops.data() + c->F_off[s * n_blocks + b] + (size_t)lam * bs;
              for (long x = 0; x < bs; ++x) dst[x] += -cf * src[x];
            }
          }
        }
  }
  // DLR basis matrices
  c->tabs.resize(r); c->k0.resize(r);
  for (int i = 0; i < r; ++i) c->tabs[i] = it[i] < 0 ? 1.0 + it[i] : it[i];
  for (int l = 0; l < r; ++l) c->k0[l] = k_abs(0.0, rf[l]);
  c->Kit.resize((size_t)r * r); c->W.assign((size_t)r * r, 0.0);
  for (int i = 0; i < r; ++i)
    for (int l = 0; l < r; ++l) c->Kit[(size_t)i * r + l] = k_it(it[i], rf[l]);
  for (int l = 0; l < r; ++l)
    for (int k = 0; k < r; ++k)
      if (k != l) c->W[(size_t)l * r + k] = c->k0[k] / (rf[k] - rf[l]);
  c->LU = c->Kit;
  lu_factor(c->LU, r, c->piv);
  // hybridization tables (Hybridization ctor, hyb.cpp:15-44)
  c->polesb.resize(p); c->kitp.resize((size_t)r * p); c->kitm.resize((size_t)r * p); c->k0p.resize(p); c->k0m.resize(p);
  for (int l = 0; l < p; ++l) {
    c->polesb[l] = hyb_poles[l] * beta;
    c->k0p[l] = k_it(0.0, c->polesb[l]);
    c->k0m[l] = k_it(0.0, -c->polesb[l]);
    for (int t = 0; t < r; ++t) {
      c->kitp[(size_t)t * p + l] = k_it(it[t], c->polesb[l]);
      c->kitm[(size_t)t * p + l] = k_it(it[t], -c->polesb[l]);
    }
  }
  c->kpow.assign((size_t)2 * p * (MAXE + 1), 1.0);
  for (int row = 0; row < 2; ++row)
    for (int l = 0; l < p; ++l)
      for (int e = 1; e <= MAXE; ++e) c->kpow[((size_t)row * p + l) * (MAXE + 1) + e] = std::pow(row == 0 ? c->k0p[l] : c->k0m[l], -e);
  c->hval.assign((size_t)r * n * n, 0.0);
  for (int t = 0; t < r; ++t)
    for (int l = 0; l < p; ++l) {
      double k = c->kitp[(size_t)t * p + l];
      for (int z = 0; z < n * n; ++z) c->hval[(size_t)t * n * n + z] += k * coef[(size_t)l * n * n + z];
    }
  // values_reflect = reflect(values) through the DLR basis (hyb.cpp:84)
  {
    std::vector<double> cfs = c->hval;
    long nc = (long)n * n;
    for (int k = 0; k < r; ++k)
      if (c->piv[k] != k)
        for (long j = 0; j < nc; ++j) std::swap(cfs[(size_t)k * nc + j], cfs[(size_t)c->piv[k] * nc + j]);
    for (int i = 1; i < r; ++i)
      for (int k = 0; k < i; ++k) {
        double f = c->LU[(size_t)i * r + k];
        for (long j = 0; j < nc; ++j) cfs[(size_t)i * nc + j] -= f * cfs[(size_t)k * nc + j];
      }
    for (int i = r - 1; i >= 0; --i) {
      for (int k = i + 1; k < r; ++k) {
        double f = c->LU[(size_t)i * r + k];
        for (long j = 0; j < nc; ++j) cfs[(size_t)i * nc + j] -= f * cfs[(size_t)k * nc + j];
      }
      for (long j = 0; j < nc; ++j) cfs[(size_t)i * nc + j] /= c->LU[(size_t)i * r + i];
    }
    c->hrefl.assign((size_t)r * nc, 0.0);
    for (int i = 0; i < r; ++i)
      for (int l = 0; l < r; ++l) {
        double k = k_it(it[i], -rf[l]);
        for (long j = 0; j < nc; ++j) c->hrefl[(size_t)i * nc + j] += k * cfs[(size_t)l * nc + j];
      }
  }
  // upload
  cudaStream_t s = c->stream;
  c->d_LU.upload(c->LU, s); c->d_piv.upload(c->piv, s); c->d_W.upload(c->W, s); c->d_Kit.upload(c->Kit, s);
  c->d_tabs.upload(c->tabs, s); c->d_k0.upload(c->k0, s); c->d_kitp.upload(c->kitp, s); c->d_kitm.upload(c->kitm, s);
  c->d_k0p.upload(c->k0p, s); c->d_k0m.upload(c->k0m, s); c->d_kpow.upload(c->kpow, s); c->d_polesb.upload(c->polesb, s);
  c->d_hval.upload(c->hval, s); c->d_hrefl.upload(c->hrefl, s); c->d_ops.upload(c->ops, s);
  c->d_dims.upload(c->dims, s); c->d_set_to_orb.upload(c->set_to_orb, s); c->d_goff.upload(c->goff, s);
  c->d_F_off.upload(c->F_off, s); c->d_Fd_off.upload(c->Fd_off, s); c->d_Fb_off.upload(c->Fb_off, s); c->d_Fdb_off.upload(c->Fdb_off, s);
  c->class_cache.clear();
  CUDA_CHECK(cudaStreamSynchronize(s));
  c->ready = true;
  API_END
}

int xca_num_self_energy_backbones(xca_ctx *ctx, int m, const int *topology, long *out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  parse_topology(m, topology);
  *out = (1L << m) * ipow(c->n, m - 1) * ipow(c->p, m - 1);
  API_END
}

int xca_num_single_ptcle_gf_backbones(xca_ctx *ctx, int m, const int *topology, long *out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  parse_topology(m, topology);
  *out = (1L << (m - 1)) * ipow(c->n, m - 1) * ipow(c->p, m - 1);
  API_END
}

int xca_compute_self_energy_device(xca_ctx *ctx, const double *G_dev, int m, const int *topology, double scale, double *Sigma_dev) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  Topology T = parse_topology(m, topology);
  auto zero = zero_flags_device(c, G_dev);
  ClassSet *cs = get_classes(c, T, zero);
  launch_sigma(c, cs, G_dev, Sigma_dev, scale);
  API_END
}

int xca_compute_self_energy(xca_ctx *ctx, const double *G, int m, const int *topology, const long *f_ix, long n_fix, double *Sigma_out) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  set_device(c);
  Topology T = parse_topology(m, topology);
  long nmaxb = (1L << m) * ipow(c->n, m - 1) * ipow(c->p, m - 1);
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  c->d_G.resize(c->slab);
  c->d_Sig.resize(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(c->d_G.ptr, g.data(), c->slab * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  zero_kernel<<<64, 256, 0, c->stream>>>(c->d_Sig.ptr, c->slab);
  c->launches++;
  auto zero = zero_flags_device(c, c->d_G.ptr);
  ClassSet *cs = get_classes(c, T, zero);
  if (f_ix == nullptr) {
    launch_sigma(c, cs, c->d_G.ptr, c->d_Sig.ptr, 1.0);
  } else {
    // subset of flat indices: build a dedicated unit list (one unit per listed f_ix and valid class)
    const long omax = ipow(c->n, m - 1), npt = ipow(c->p, m - 1);
    std::vector<WorkUnit> units;
    for (long z = 0; z < n_fix; ++z) {
      long f = f_ix[z];
      if (f < 0 || f >= nmaxb) throw Error(XCA_ERR_RUNTIME, "DiagramEvaluator::eval_self_energy: f_ix out of range");
      long o = f % omax, q = f / omax;
      long pix = q % npt, fb = q / npt;
      for (int k : cs->by_fbo[fb * omax + o]) units.push_back(WorkUnit{k, (int)pix, 1});
    }
    if (!units.empty()) {
      ClassSet tmp;
      tmp.classes = cs->classes;
      tmp.units = units;
      tmp.d_classes.upload(tmp.classes, c->stream);
      tmp.d_units.upload(tmp.units, c->stream);
      launch_sigma(c, &tmp, c->d_G.ptr, c->d_Sig.ptr, 1.0);
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
    }
  }
  std::vector<double> out(c->slab);
  CUDA_CHECK(cudaMemcpyAsync(out.data(), c->d_Sig.ptr, c->slab * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  // blocks that end below 1e-16 come back as exact zeros (set_zero_block_indices, bsb.cpp:386-395)
  for (int b = 0; b < c->nb; ++b) {
    long o = c->goff[b], sz = (long)c->r * c->dims[b] * c->dims[b];
    double mx = 0;
    for (long i = 0; i < sz; ++i) mx = std::max(mx, std::fabs(out[o + i]));
    if (mx < 1e-16)
      for (long i = 0; i < sz; ++i) out[o + i] = 0.0;
  }
  for (long i = 0; i < c->slab; ++i) {
    Sigma_out[2 * i] = out[i];
    Sigma_out[2 * i + 1] = 0.0;
  }
  API_END
}

int xca_self_energy_items(xca_ctx *ctx, const double *G, int m, const int *topology, long *rows, long max_rows, long *n_items) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  if (!c->ready) throw Error(XCA_ERR_INVALID, "evaluator not set up");
  Topology T = parse_topology(m, topology);
  std::vector<double> g;
  real_part(G, c->slab, g, "G");
  std::vector<int> zero(c->nb);
  for (int b = 0; b < c->nb; ++b) {
    long o = c->goff[b], sz = (long)c->r * c->dims[b] * c->dims[b];
    double mx = 0;
    for (long i = 0; i < sz; ++i) mx = std::max(mx, std::fabs(g[o + i]));
    zero[b] = mx < 1e-16;
  }
  set_device(c);
  ClassSet *cs = get_classes(c, T, zero);
  const long omax = ipow(c->n, m - 1), npt = ipow(c->p, m - 1), fbmax = 1L << m;
  const int width = 3 + 2 * m - 1;
  long count = 0;
  for (long fb = 0; fb < fbmax; ++fb)
    for (long pix = 0; pix < npt; ++pix)
      for (long o = 0; o < omax; ++o) {
        const auto &lst = cs->by_fbo[fb * omax + o];
        if (!rows || count >= max_rows) {
          count += (long)lst.size();
          continue;
        }
        long f = o + omax * (pix + npt * fb);
        for (int k : lst) {
          if (count < max_rows) {
            long *rw = rows + count * width;
            const ClassRec &R = cs->classes[k];
            rw[0] = f; rw[1] = R.b_out; rw[2] = R.pk;
            for (int i = 0; i < 2 * m - 1; ++i) rw[3 + i] = R.ind_path[i];
          }
          count++;
        }
      }
  *n_items = count;
  API_END
}

int xca_slab_info(xca_ctx *ctx, long *n_doubles, int *r) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  *n_doubles = c->slab;
  *r = c->r;
  API_END
}

int xca_device_buffer(xca_ctx *ctx, int slot, long bytes, double **dev_ptr) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  if (slot < 0 || slot > 63) throw Error(XCA_ERR_INVALID, "buffer slot out of range");
  while ((int)c->user_bufs.size() <= slot) c->user_bufs.emplace_back(new DevBuf<double>());
  c->user_bufs[slot]->resize((bytes + 7) / 8);
  *dev_ptr = c->user_bufs[slot]->ptr;
  API_END
}

int xca_copy_to_device(xca_ctx *ctx, double *dev, const double *host, long n) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  CUDA_CHECK(cudaMemcpyAsync(dev, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_copy_to_host(xca_ctx *ctx, double *host, const double *dev, long n) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  CUDA_CHECK(cudaMemcpyAsync(host, dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_synchronize(xca_ctx *ctx) {
  API_BEGIN
  auto *c = reinterpret_cast<Ctx *>(ctx);
  set_device(c);
  CUDA_CHECK(cudaStreamSynchronize(c->stream));
  API_END
}

int xca_kernel_launches(xca_ctx *ctx, long *out) {
  API_BEGIN
  *out = reinterpret_cast<Ctx *>(ctx)->launches;
  API_END
}

}  // extern "C"
