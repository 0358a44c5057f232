// Pseudo-particle Dyson solve, trace and normalisation on the device (plain FP64 path).
//
// Per Fock-space block b (d = d_b, N = r d), following cppdlr's dyson_it_ppsc::solve
// (c++/triqs_xca/dlr_dyson_ppsc.hpp:135-168) as called by solve_dyson
// (python/triqs_xca/block_sparse_solver.py:572-590):
//   sigc = K^-1 Sigma_b                                  (vals2coefs)
//   ggs  = -(conv_TO(g0c, sigc) + eta G0_b)              (time-ordered DLR convolution, closed form)
//   f    = K^-1 ggs,  ft = W f                           (coefficients of the system kernel)
//   M    = convmat(f): (M g)(t_i) = int_0^tau f(tau - s) g(s) ds on the nodes, M = A K^-1
//   (I + M) G = G0                                       (getrf with partial pivoting, getrs)
//   G   <- (G + G^T) / 2                                 (hermitize, real data)
// Matrices of all blocks are factorised concurrently, one CTA per block, in global memory (L2 resident
// for the block sizes of the configurations here: sum_b (r d_b)^2 doubles).
#pragma once
#include "sigma_kernel.cuh"

namespace xca {


// K^T z = a for one register-resident row vector, with K = P L U (the factors of lu_factor): U^T y = a
// row by row (i ascending: subtract U_ki y_k for k < i ascending, then divide by U_ii), L^T w = y
// (i descending: subtract L_ki w_k for k > i ascending), each product and difference separately
// rounded; then z = P w, i.e. z[perm[i]] = w[i] (the caller scatters).  Padding rows of LUT are the
// identity.  LUT is column-major: LUT[i * RP + k] = LU(row k, column i).
template <int RP>
__device__ __forceinline__ void lu_solve_transposed_reg(const double *__restrict__ LUT, double (&x)[RP]) {
#pragma unroll
  for (int i = 0; i < RP; ++i) {
#pragma unroll
    for (int k = 0; k < i; ++k) x[i] = __dsub_rn(x[i], mul(LUT[i * RP + k], x[k]));
    x[i] = __ddiv_rn(x[i], LUT[i * RP + i]);
  }
#pragma unroll
  for (int i = RP - 1; i >= 0; --i) {
#pragma unroll
    for (int k = i + 1; k < RP; ++k) x[i] = __dsub_rn(x[i], mul(LUT[i * RP + k], x[k]));
  }
}

// y_l = sum_k M[l][k] x_k for l < r with every product and sum separately rounded, k ascending from zero
// (MT = M column-major); y written with stride `ld`.
template <int RP>
__device__ __forceinline__ void matvec_sep_reg(const double *__restrict__ MT, const double (&x)[RP], int r, double *y, int ld) {
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
      for (int j = 0; j < CH; ++j) acc[j] = add(acc[j], mul(MT[k * RP + l0 + j], x[k]));
    }
#pragma unroll
    for (int j = 0; j < CH; ++j)
      if (l0 + j < r) y[(l0 + j) * ld] = acc[j];
  }
}

// Stage the padded LU (with its reciprocal diagonal) and W into shared memory (2 RP^2 + RP doubles) and
// the pivot gather (RP ints).
template <int RP>
__device__ __forceinline__ void stage_lu_w(const DysonBasis &B, double *sLU, double *sW, int *sPerm) {
  for (int i = threadIdx.x; i < RP * RP + RP; i += blockDim.x) sLU[i] = B.LUp[i];
  for (int i = threadIdx.x; i < RP * RP; i += blockDim.x) sW[i] = B.Wp[i];
  for (int i = threadIdx.x; i < RP; i += blockDim.x) sPerm[i] = B.perm[i];
  __syncthreads();
}

// Columns (r-vectors with stride dd) of `src`: coefficients K^-1 src into `c` and W K^-1 src into `ct`
// (fused multiply-adds as the convolution's Hilbert sums, or separately rounded as the convolution matrix's).
template <int RP, bool FUSED>
__device__ __forceinline__ void coefs_and_hilbert(const double *sLU, const double *sW, const int *sPerm, int r, int dd,
                                                  const double *src, double *c, double *ct) {
  for (int col = threadIdx.x; col < dd; col += blockDim.x) {
    double x[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) {
      const int s = sPerm[i];
      x[i] = s >= 0 ? src[(size_t)s * dd + col] : 0.0;
    }
    lu_solve_reg<RP>(sLU, x);
#pragma unroll
    for (int i = 0; i < RP; ++i)
      if (i < r) c[(size_t)i * dd + col] = x[i];
    if (FUSED)
      matvec_reg<RP>(sW, x, r, ct + col, dd);
    else
      matvec_sep_reg<RP>(sW, x, r, ct + col, dd);
  }
}

// One CTA per block: sigc, gt, Q, P', ggs, then f = K^-1 ggs and ft = W f into the block's work area
// [sigc | gt | Q | P' | f | ft], each r d^2 doubles.
template <int RP>
__global__ void __launch_bounds__(256) dyson_coef_kernel(DysonBasis B, const double *__restrict__ Sigma, double eta,
                                                         const double *__restrict__ op) {
  extern __shared__ __align__(16) double smem[];
  double *sLU = smem;
  double *sW = sLU + RP * RP + RP;
  int *sPerm = reinterpret_cast<int *>(sW + RP * RP);
  const int b = blockIdx.x;
  if (b >= B.nb) return;
  stage_lu_w<RP>(B, sLU, sW, sPerm);
  const int r = B.r, d = B.dims[b], dd = d * d;
  const long rdd = (long)r * dd;
  double *w = B.work + B.woff[b];
  double *sigc = w, *gt = w + rdd, *Q = w + 2 * rdd, *P = w + 3 * rdd, *f = w + 4 * rdd, *ft = w + 5 * rdd;
  const double *sig = Sigma + B.goff[b];
  const double *g0 = B.g0 + B.goff[b], *g0c = B.g0c + B.goff[b], *g0t = B.g0t + B.goff[b];
  coefs_and_hilbert<RP, true>(sLU, sW, sPerm, r, dd, sig, sigc, gt);
  __syncthreads();
  // Q_l = ft_l g_l + f_l gt_l and P'_l = K_l(0) (f_l g_l) with f = g0c, g = sigc
  for (long e = threadIdx.x; e < rdd; e += blockDim.x) {
    const int l = (int)(e / dd), xz = (int)(e - (long)l * dd), x = xz / d, z = xz - x * d;
    const double *fl = g0c + (long)l * dd, *fhl = g0t + (long)l * dd, *gl = sigc + (long)l * dd, *ghl = gt + (long)l * dd;
    double sq = 0.0, sp = 0.0;
    for (int y = 0; y < d; ++y) {
      sq = fmad(fhl[x * d + y], gl[y * d + z], fmad(fl[x * d + y], ghl[y * d + z], sq));
      sp = fmad(fl[x * d + y], gl[y * d + z], sp);
    }
    Q[e] = sq;
    P[e] = mul(B.k0[l], sp);
  }
  __syncthreads();
  // ggs(t_i) = -(h(t_i) + eta G0(t_i)), h = fma(t_i, h2, h1); stored in the sigc slot (no longer read).  With an
  // operator (solve_with_op, dlr_dyson_ppsc.hpp:188-196): ggs(t_i) = -((h + eta G0) + G0(t_i) op), the
  // product summed over the inner index ascending, each product and sum separately rounded.
  const double *ob = op;
  if (op)
    for (int bb = 0; bb < b; ++bb) ob += (long)B.dims[bb] * B.dims[bb];
  for (long e = threadIdx.x; e < rdd; e += blockDim.x) {
    const int i = (int)(e / dd), xz = (int)(e - (long)i * dd);
    double h1 = 0.0, h2 = 0.0;
    for (int l = 0; l < r; ++l) {
      const double bk = B.BKp[l * RP + i];
      h1 = fmad(bk, Q[(long)l * dd + xz], h1);
      h2 = fmad(bk, P[(long)l * dd + xz], h2);
    }
    const double h = fmad(B.tabs[i], h2, h1);
    if (ob) {
      const int x = xz / d, z = xz - x * d;
      const double *g0r = g0 + (long)i * dd + x * d;
      double mop = 0.0;
      for (int y = 0; y < d; ++y) mop = add(mop, mul(g0r[y], ob[y * d + z]));
      sigc[e] = -add(add(h, mul(eta, g0[e])), mop);
    } else {
      sigc[e] = -add(h, mul(eta, g0[e]));
    }
  }
  __syncthreads();
  coefs_and_hilbert<RP, false>(sLU, sW, sPerm, r, dd, sigc, f, ft);
}

// Rows of the system matrix I + M, one thread per (block, i, x, y) row vector of A (convmat_inplace,
// cppdlr; call site dlr_dyson_ppsc.hpp:149), in the operation order of the CPU restatement:
//   A[i][k](x,y) = (beta K_ik) (ft_k + (t_i K_k(0)) f_k) + sum_{l != k, ascending} [((beta K_il) K_k(0)) / (om_k - om_l)] f_l
// (the bracketed weights come from the basis's table convw), then M[(i,x), (i',y)] = (A K^-1)[i'] through
// K^T z = a.  grid.y = block, 64 threads per CTA.
template <int RP>
__global__ void __launch_bounds__(64) dyson_convmat_kernel(DysonBasis B) {
  __shared__ double sf[RP * 64];
  const int b = blockIdx.y;
  const int r = B.r, d = B.dims[b], dd = d * d;
  const long row = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = row < (long)r * dd;
  const int i = active ? (int)(row / dd) : 0;
  const int xy = active ? (int)(row - (long)i * dd) : 0;
  const double *w = B.work + B.woff[b];
  const long rdd = (long)r * dd;
  const double *f = w + 4 * rdd, *ft = w + 5 * rdd;
  // f_l of this thread's (x, y), one column of sf per thread
  for (int l = 0; l < RP; ++l) sf[l * 64 + threadIdx.x] = (active && l < r) ? f[(long)l * dd + xy] : 0.0;
  if (!active) return;
  const double ti = B.tabs[i];
  double a[RP];
#pragma unroll
  for (int k = 0; k < RP; ++k) {
    double acc = 0.0;
    if (k < r) {
      const double k0k = B.k0[k];
      acc = mul(B.BKp[k * RP + i], add(ft[(long)k * dd + xy], mul(mul(ti, k0k), sf[k * 64 + threadIdx.x])));
      const double *wk = B.convw + (long)k * RP * RP + i;
      for (int l = 0; l < r; ++l) {
        if (l == k) continue;
        acc = add(acc, mul(wk[(long)l * RP], sf[l * 64 + threadIdx.x]));
      }
    }
    a[k] = acc;
  }
  lu_solve_transposed_reg<RP>(B.LUp, a);
  const int x = xy / d, y = xy - x * d;
  const long N = (long)r * d;
  double *Mrow = B.mats + B.moff[b] + ((long)i * d + x) * N;
#pragma unroll
  for (int k = 0; k < RP; ++k) {
    if (k < r) {
      const int ip = B.perm[k];  // z[perm[k]] = w[k]
      Mrow[(long)ip * d + y] = (ip == i && x == y) ? add(a[k], 1.0) : a[k];
    }
  }
}

// (value, row) arg-max reduction within a CTA; ties keep the smaller row (idamax returns the first).
__device__ __forceinline__ void argmax_combine(double &v, int &ix, double v2, int ix2) {
  if (v2 > v || (v2 == v && ix2 < ix)) { v = v2; ix = ix2; }
}

// One CTA per block: LU with partial pivoting of the N x N system (row-major in global memory; elimination
// updates a_ij - l_ik u_kj separately rounded, as the CPU restatement's getrf), then the
// solve with the d right-hand-side columns G0 (rows (t, i), columns j: the packed slab layout), row
// interchanges, unit-lower forward and upper backward substitution, and the (optional) hermitization
// G(t) <- (G(t) + G(t)^T) / 2 into G_out.  rhs is the block's scratch copy of G0.
// SMEM: the matrix (row stride N + 1, against bank conflicts on column accesses) and the right-hand sides
// are copied into dynamic shared memory first (systems up to DYSON_SMEM_MAX_N), so that every elimination
// step works at shared-memory latency; the operations and their order are the same either way.
template <bool SMEM>
__global__ void __launch_bounds__(1024) dyson_lu_solve_kernel(DysonBasis B, double *__restrict__ rhs, double *__restrict__ G_out,
                                                              int hermitize, int *__restrict__ status) {
  extern __shared__ __align__(16) double smA[];
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv;
  const int b = blockIdx.x;
  if (b >= B.nb) return;
  const int r = B.r, d = B.dims[b], dd = d * d;
  const int N = r * d;
  const long lda = SMEM ? N + 1 : N;
  double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  const double *g0 = B.g0 + B.goff[b];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  if (SMEM) {
    for (long e = tid; e < (long)N * N; e += nt) {
      const long i = e / N, j = e - i * N;
      smA[i * lda + j] = A[e];
    }
    A = smA;
    x = smA + (long)N * lda;
  }
  for (long e = tid; e < (long)N * d; e += nt) x[e] = g0[e];
  if (SMEM) __syncthreads();
  bool singular = false;
  for (int k = 0; k < N; ++k) {
    // pivot search in column k, rows k..N-1
    double bv = -1.0;
    int bi = N;
    for (int i = k + tid; i < N; i += nt) argmax_combine(bv, bi, fabs(A[(long)i * lda + k]), i);
    for (int o = 16; o > 0; o >>= 1) {
      double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
      int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
      argmax_combine(bv, bi, v2, i2);
    }
    if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
    __syncthreads();
    if (warp == 0) {
      bv = lane < (nt >> 5) ? red_v[lane] : -1.0;
      bi = lane < (nt >> 5) ? red_i[lane] : N;
      for (int o = 16; o > 0; o >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        argmax_combine(bv, bi, v2, i2);
      }
      if (lane == 0) s_piv = bi;
    }
    __syncthreads();
    const int p = s_piv;
    if (p >= N) { singular = true; break; }  // only when the column is NaN
    if (p != k) {
      for (int j = tid; j < N; j += nt) {
        const double t = A[(long)k * lda + j];
        A[(long)k * lda + j] = A[(long)p * lda + j];
        A[(long)p * lda + j] = t;
      }
      for (int j = tid; j < d; j += nt) {
        const double t = x[(long)k * d + j];
        x[(long)k * d + j] = x[(long)p * d + j];
        x[(long)p * d + j] = t;
      }
    }
    __syncthreads();
    const double piv = A[(long)k * lda + k];
    if (piv == 0.0) { singular = true; break; }
    for (int i = k + 1 + tid; i < N; i += nt) A[(long)i * lda + k] = __ddiv_rn(A[(long)i * lda + k], piv);
    __syncthreads();
    const int m = N - k - 1;
    for (long e = tid; e < (long)m * m; e += nt) {
      const int i = k + 1 + (int)(e / m), j = k + 1 + (int)(e - (e / m) * m);
      A[(long)i * lda + j] = __dsub_rn(A[(long)i * lda + j], mul(A[(long)i * lda + k], A[(long)k * lda + j]));
    }
    __syncthreads();
  }
  if (singular) {
    if (tid == 0) atomicExch(status, 1);
    return;
  }
  // forward substitution with the unit lower factor (the row interchanges were applied above)
  for (int k = 0; k < N - 1; ++k) {
    const int m = N - k - 1;
    for (int e = tid; e < m * d; e += nt) {
      const int i = k + 1 + e / d, j = e - (e / d) * d;
      x[(long)i * d + j] = fmad(-A[(long)i * lda + k], x[(long)k * d + j], x[(long)i * d + j]);
    }
    __syncthreads();
  }
  // backward substitution with the upper factor
  for (int k = N - 1; k >= 0; --k) {
    for (int j = tid; j < d; j += nt) x[(long)k * d + j] = __ddiv_rn(x[(long)k * d + j], A[(long)k * lda + k]);
    __syncthreads();
    for (int e = tid; e < k * d; e += nt) {
      const int i = e / d, j = e - i * d;
      x[(long)i * d + j] = fmad(-A[(long)i * lda + k], x[(long)k * d + j], x[(long)i * d + j]);
    }
    __syncthreads();
  }
  double *g = G_out + B.goff[b];
  for (long e = tid; e < (long)r * dd; e += nt) {
    const int t = (int)(e / dd), ij = (int)(e - (long)t * dd), i = ij / d, j = ij - i * d;
    const double v = x[e];
    g[e] = hermitize ? mul(0.5, add(v, x[(long)t * dd + j * d + i])) : v;
  }
}

// Per block: sum_x G_b(beta)[x][x] = sum_x sum_l K(1, om_l) (K^-1 G_b)_l[x][x], one lane per diagonal entry.
template <int RP>
__global__ void __launch_bounds__(128) trace_beta_kernel(DysonBasis B, const double *__restrict__ G, double *__restrict__ out) {
  extern __shared__ __align__(16) double smem[];
  double *sLU = smem;
  int *sPerm = reinterpret_cast<int *>(sLU + RP * RP + RP);
  __shared__ double part[128];
  const int b = blockIdx.x;
  for (int i = threadIdx.x; i < RP * RP + RP; i += blockDim.x) sLU[i] = B.LUp[i];
  for (int i = threadIdx.x; i < RP; i += blockDim.x) sPerm[i] = B.perm[i];
  __syncthreads();
  const int r = B.r, d = B.dims[b], dd = d * d;
  const double *g = G + B.goff[b];
  // the thread's partial sum lives in shared memory: a register carried across the loop with the
  // register-resident solve made the compiler spill the whole vector
  part[threadIdx.x] = 0.0;
  for (int xx = threadIdx.x; xx < d; xx += blockDim.x) {
    double x[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) {
      const int src = sPerm[i];
      x[i] = src >= 0 ? g[(long)src * dd + xx * d + xx] : 0.0;
    }
    lu_solve_reg<RP>(sLU, x);
    double v = 0.0;
#pragma unroll
    for (int l = 0; l < RP; ++l)
      if (l < r) v = add(v, mul(B.k1[l], x[l]));
    part[threadIdx.x] = add(part[threadIdx.x], v);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)blockDim.x; ++i) t = add(t, part[i]);
    out[b] = t;
  }
}

// G(tau_i) <- G(tau_i) exp(-tau_i deta), tau_i = beta t_i (energy_shift_ppgf, block_sparse_solver.py:436-441).
// G_b(tau_t) <- G_b(tau_t) * fac[t] for every block, fac[t] = exp(-tau_t deta) (energy_shift_ppgf of
// normalize_pseudo_particle_gf, python/triqs_xca/block_sparse_solver.py:436-442); the r factors are
// computed by the caller.
__global__ void energy_shift_kernel(DysonBasis B, double *__restrict__ G, const double *__restrict__ fac) {
  const int b = blockIdx.y;
  const int dd = B.dims[b] * B.dims[b];
  const long n = (long)B.r * dd;
  double *g = G + B.goff[b];
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const int t = (int)(e / dd);
    g[e] = mul(g[e], fac[t]);
  }
}

// Partial maxima of |a - b| over a packed slab (one per CTA; the host takes the max of the partials).
__global__ void __launch_bounds__(256) max_abs_diff_kernel(const double *__restrict__ a, const double *__restrict__ b, long n,
                                                           double *__restrict__ out) {
  __shared__ double red[256];
  double m = 0.0;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(a[e] - b[e]));
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// y <- alpha x + beta y (two rounded products, one rounded sum: mix * G_new + (1 - mix) * G).
__global__ void axpby_kernel(double alpha, const double *__restrict__ x, double beta, double *__restrict__ y, long n) {
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    y[e] = add(mul(alpha, x[e]), mul(beta, y[e]));
}

}  // namespace xca

namespace xca {

// convolve_ppsc (c++/triqs_xca/block_sparse.cpp:832-850): per block, H = convolve(beta, K^-1 G1_b, K^-1 G2_b,
// TIME_ORDERED) on the nodes, with the operation order of the CPU restatement: f = K^-1 G1, ft = W f,
// g = K^-1 G2, gt = W g; Q_l = ft_l g_l + f_l gt_l and P'_l = K(0, om_l) (f_l g_l) (fused multiply-adds over
// the inner index, the f gt term first); H(t_i) = fma(t_i, sum_l (beta K_il) P'_l, sum_l (beta K_il) Q_l).
// One CTA per block; work holds 6 r d^2 doubles per block at B.woff.
template <int RP>
__global__ void __launch_bounds__(256) convolve_ppsc_kernel(DysonBasis B, const double *__restrict__ G1, const double *__restrict__ G2,
                                                             double *__restrict__ H) {
  extern __shared__ __align__(16) double smem[];
  double *sLU = smem, *sW = sLU + RP * RP + RP;
  int *sPerm = reinterpret_cast<int *>(sW + RP * RP);
  stage_lu_w<RP>(B, sLU, sW, sPerm);
  const int b = blockIdx.x, r = B.r, d = B.dims[b], dd = d * d;
  double *f = B.work + B.woff[b], *ft = f + (long)r * dd, *g = ft + (long)r * dd, *gt = g + (long)r * dd;
  double *Q = gt + (long)r * dd, *P = Q + (long)r * dd;
  coefs_and_hilbert<RP, true>(sLU, sW, sPerm, r, dd, G1 + B.goff[b], f, ft);
  coefs_and_hilbert<RP, true>(sLU, sW, sPerm, r, dd, G2 + B.goff[b], g, gt);
  __syncthreads();
  for (int idx = threadIdx.x; idx < r * dd; idx += blockDim.x) {
    const int l = idx / dd, e = idx - l * dd, x = e / d, z = e - x * d;
    const double *fl = f + (long)l * dd + x * d, *ftl = ft + (long)l * dd + x * d;
    const double *gl = g + (long)l * dd + z, *gtl = gt + (long)l * dd + z;
    double sq = 0.0, sp = 0.0;
    for (int y = 0; y < d; ++y) {
      sq = fmad(ftl[y], gl[y * d], fmad(fl[y], gtl[y * d], sq));
      sp = fmad(fl[y], gl[y * d], sp);
    }
    Q[idx] = sq;
    P[idx] = mul(B.k0[l], sp);
  }
  __syncthreads();
  double *h = H + B.goff[b];
  for (int idx = threadIdx.x; idx < r * dd; idx += blockDim.x) {
    const int i = idx / dd, e = idx - i * dd;
    double h1 = 0.0, h2 = 0.0;
    for (int l = 0; l < r; ++l) {
      const double bk = B.BKp[l * RP + i];
      h1 = fmad(bk, Q[(long)l * dd + e], h1);
      h2 = fmad(bk, P[(long)l * dd + e], h2);
    }
    h[idx] = fmad(B.tabs[i], h2, h1);
  }
}

// expectation_value (c++/triqs_xca/block_sparse.cpp:797-818), per block b with a diagonal operator block O_b
// (op_off[b] >= 0): G_b(beta) by DLR evaluation (K^-1 per entry, then sum_l K(1, om_l) c_l from zero in
// ascending l), then out[b] = Tr[O_b G_b(beta)] = sum_x (sum_y O[x][y] G(beta)[y][x]) (fused multiply-adds
// over y, the x sums in order); out[b] = 0 for blocks without an operator block.  work: r d^2 per block.
template <int RP>
__global__ void __launch_bounds__(128) expectation_beta_kernel(DysonBasis B, const double *__restrict__ G, const double *__restrict__ ops,
                                                                const long *__restrict__ op_off, double *__restrict__ out) {
  extern __shared__ __align__(16) double smem[];
  double *sLU = smem;
  int *sPerm = reinterpret_cast<int *>(sLU + RP * RP + RP);
  for (int i = threadIdx.x; i < RP * RP + RP; i += blockDim.x) sLU[i] = B.LUp[i];
  for (int i = threadIdx.x; i < RP; i += blockDim.x) sPerm[i] = B.perm[i];
  __syncthreads();
  const int b = blockIdx.x, r = B.r, d = B.dims[b], dd = d * d;
  if (op_off[b] < 0) {
    if (threadIdx.x == 0) out[b] = 0.0;
    return;
  }
  const double *g = G + B.goff[b];
  double *gb = B.work + B.woff[b];
  for (int col = threadIdx.x; col < dd; col += blockDim.x) {
    double x[RP];
#pragma unroll
    for (int i = 0; i < RP; ++i) {
      const int src = sPerm[i];
      x[i] = src >= 0 ? g[(long)src * dd + col] : 0.0;
    }
    lu_solve_reg<RP>(sLU, x);
    double v = 0.0;
#pragma unroll
    for (int l = 0; l < RP; ++l)
      if (l < r) v = add(v, mul(B.k1[l], x[l]));
    gb[col] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double *O = ops + op_off[b];
    double tr = 0.0;
    for (int x = 0; x < d; ++x) {
      double s = 0.0;
      for (int y = 0; y < d; ++y) s = fmad(O[x * d + y], gb[y * d + x], s);
      tr = add(tr, s);
    }
    out[b] = tr;
  }
}

}  // namespace xca

namespace xca {

// ---------------------------------------------------------------------------------------------------------
// Blocked LU with partial pivoting and substitution for large Dyson systems (N = r d in the thousands for
// the five-orbital d shell).  Panels of LU_NB columns; every matrix element still receives the elimination
// updates a_ij <- a_ij - l_ik u_kj of the unblocked getrf in ascending k, each product and difference
// separately rounded, and every right-hand-side entry the fused multiply-adds of the substitutions in the
// order of the CPU restatement (forward k ascending, backward k descending with the division by U_kk), so
// the result equals the unblocked kernel's bit for bit; only the number of passes over the matrix changes.
// Every kernel takes the Fock-space block from blockIdx.z / blockIdx.x and returns at once for blocks
// whose system is smaller than the current panel.
constexpr int LU_NB = 32;

__device__ __forceinline__ long lu_dim(const DysonBasis &B, int b) { return (long)B.r * B.dims[b]; }

// Panel factorisation of columns [k0, k0 + LU_NB) over all rows: pivot search, full-row interchange (matrix
// and right-hand side), column scaling, rank-1 updates inside the panel.  One CTA per block.
__global__ void __launch_bounds__(1024) lu_panel_kernel(DysonBasis B, double *__restrict__ rhs, int k0, int *__restrict__ status) {
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv;
  const int b = blockIdx.x;
  const int N = (int)lu_dim(B, b), d = B.dims[b];
  if (k0 >= N) return;
  const int kend = min(k0 + LU_NB, N);
  double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  for (int k = k0; k < kend; ++k) {
    double bv = -1.0;
    int bi = N;
    for (int i = k + tid; i < N; i += nt) argmax_combine(bv, bi, fabs(A[(long)i * N + k]), i);
    for (int o = 16; o > 0; o >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
      argmax_combine(bv, bi, v2, i2);
    }
    if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
    __syncthreads();
    if (warp == 0) {
      bv = lane < (nt >> 5) ? red_v[lane] : -1.0;
      bi = lane < (nt >> 5) ? red_i[lane] : N;
      for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        argmax_combine(bv, bi, v2, i2);
      }
      if (lane == 0) s_piv = bi;
    }
    __syncthreads();
    const int p = s_piv;
    if (p >= N) {  // a column of NaN: flag and leave the block
      if (tid == 0) atomicExch(status, 1);
      return;
    }
    if (p != k) {
      for (int j = tid; j < N; j += nt) {
        const double t = A[(long)k * N + j];
        A[(long)k * N + j] = A[(long)p * N + j];
        A[(long)p * N + j] = t;
      }
      for (int j = tid; j < d; j += nt) {
        const double t = x[(long)k * d + j];
        x[(long)k * d + j] = x[(long)p * d + j];
        x[(long)p * d + j] = t;
      }
    }
    __syncthreads();
    const double piv = A[(long)k * N + k];
    if (piv == 0.0) {
      if (tid == 0) atomicExch(status, 1);
      return;
    }
    for (int i = k + 1 + tid; i < N; i += nt) A[(long)i * N + k] = __ddiv_rn(A[(long)i * N + k], piv);
    __syncthreads();
    const int w = kend - k - 1;
    if (w > 0)
      for (long e = tid; e < (long)(N - k - 1) * w; e += nt) {
        const int i = k + 1 + (int)(e / w), j = k + 1 + (int)(e - (e / w) * w);
        A[(long)i * N + j] = __dsub_rn(A[(long)i * N + j], mul(A[(long)i * N + k], A[(long)k * N + j]));
      }
    __syncthreads();
  }
}

// The panel factorisation of lu_panel_kernel with the panel -- rows [k0, N) x columns [k0, k0 + LU_NB) --
// held in shared memory (row stride LU_PS, so a warp reading one column hits distinct banks): the same pivot
// choices (largest |a_ik|, lowest row on ties) and the same separately rounded divisions and updates in the
// same order.  Interchanges only permute the entries of the other columns and of the right-hand side, so
// those are applied after the panel, pivot by pivot in order, one thread per column.  Launched with
// (n_max - k0) LU_PS doubles of dynamic shared memory, at most LU_PANEL_SMEM_MAX_BYTES.
constexpr int LU_PS = LU_NB + 1;
constexpr int LU_PANEL_SMEM_MAX_BYTES = 200 * 1024;

__global__ void __launch_bounds__(1024) lu_panel_smem_kernel(DysonBasis B, double *__restrict__ rhs, int k0, int *__restrict__ status) {
  extern __shared__ double P[];
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv[LU_NB];
  const int b = blockIdx.x;
  const int N = (int)lu_dim(B, b), d = B.dims[b];
  if (k0 >= N) return;
  const int M = N - k0, nb = min(LU_NB, M);
  double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
  if (M > nt) {  // one thread per panel row; the launcher keeps M within the block
    if (tid == 0) atomicExch(status, 1);
    return;
  }
  for (int e = tid; e < M * nb; e += nt) {
    const int i = e / nb, c = e - i * nb;
    P[i * LU_PS + c] = A[(long)(k0 + i) * N + k0 + c];
  }
  __syncthreads();
  // thread tid owns panel row i = tid: its candidate for the first pivot, reduced per warp
  const int i = tid;
  double bv = -1.0;
  int bi = M;
  if (i < M) argmax_combine(bv, bi, fabs(P[i * LU_PS]), i);
  for (int c = 0;; ++c) {
    for (int o = 16; o > 0; o >>= 1) {
      const double v2 = __shfl_xor_sync(0xffffffffu, bv, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
      argmax_combine(bv, bi, v2, i2);
    }
    if (lane == 0) { red_v[warp] = bv; red_i[warp] = bi; }
    __syncthreads();
    if (c == nb) break;
    // warp 0: the pivot of column c (largest |a_ic|, lowest row on ties), then the interchange of the
    // panel rows c and p
    if (warp == 0) {
      double v = lane < nw ? red_v[lane] : -1.0;
      int ix = lane < nw ? red_i[lane] : M;
      for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, ix, o);
        argmax_combine(v, ix, v2, i2);
      }
      if (ix < M && ix != c && lane < nb) {
        const double t = P[c * LU_PS + lane];
        P[c * LU_PS + lane] = P[ix * LU_PS + lane];
        P[ix * LU_PS + lane] = t;
      }
      if (lane == 0) s_piv[c] = ix;
    }
    __syncthreads();
    const int p = s_piv[c];
    if (p >= M) {  // a column of NaN: flag and leave the block
      if (tid == 0) atomicExch(status, 1);
      return;
    }
    const double piv = P[c * LU_PS + c];
    if (piv == 0.0) {
      if (tid == 0) atomicExch(status, 1);
      return;
    }
    // rows below the pivot: l_ic = a_ic / u_cc, then a_ij -= l_ic u_cj for the panel columns j > c, and the
    // row's candidate for the next pivot
    bv = -1.0;
    bi = M;
    if (i > c && i < M) {
      const double l = __ddiv_rn(P[i * LU_PS + c], piv);
      P[i * LU_PS + c] = l;
      for (int j = c + 1; j < nb; ++j) P[i * LU_PS + j] = __dsub_rn(P[i * LU_PS + j], mul(l, P[c * LU_PS + j]));
      if (c + 1 < nb) argmax_combine(bv, bi, fabs(P[i * LU_PS + c + 1]), i);
    }
  }
  for (int e = tid; e < M * nb; e += nt) {
    const int i = e / nb, c = e - i * nb;
    A[(long)(k0 + i) * N + k0 + c] = P[i * LU_PS + c];
  }
  // columns [0, k0) and [k0 + nb, N) of the matrix, then the d right-hand-side columns
  for (int j = tid; j < N - nb + d; j += nt) {
    double *col;
    long ld;
    if (j < N - nb) {
      col = A + (j < k0 ? j : j + nb);
      ld = N;
    } else {
      col = x + (j - (N - nb));
      ld = d;
    }
    for (int c = 0; c < nb; ++c) {
      const int p = s_piv[c];
      if (p != c) {
        const double t = col[(long)(k0 + c) * ld];
        col[(long)(k0 + c) * ld] = col[(long)(k0 + p) * ld];
        col[(long)(k0 + p) * ld] = t;
      }
    }
  }
}

// Panel rows right of the panel (U12): for every column j >= k0 + LU_NB, the panel's updates
// a_ij -= l_ik a_kj for k0 <= k < i < k0 + LU_NB in ascending k.  One thread per column.
__global__ void __launch_bounds__(128) lu_u12_kernel(DysonBasis B, int k0) {
  __shared__ double L[LU_NB][LU_NB + 1];
  const int b = blockIdx.z;
  const int N = (int)lu_dim(B, b);
  const int kend = min(k0 + LU_NB, N), nb = kend - k0;
  if (kend >= N) return;
  const double *A0 = B.mats + B.moff[b];
  for (int e = threadIdx.x; e < LU_NB * LU_NB; e += blockDim.x) {
    const int i = e / LU_NB, k = e - i * LU_NB;
    L[i][k] = (i < nb && k < nb) ? A0[(long)(k0 + i) * N + k0 + k] : 0.0;
  }
  __syncthreads();
  const int j = kend + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  double *A = B.mats + B.moff[b];
  double a[LU_NB];
#pragma unroll
  for (int i = 0; i < LU_NB; ++i) a[i] = i < nb ? A[(long)(k0 + i) * N + j] : 0.0;
#pragma unroll
  for (int k = 0; k < LU_NB; ++k)
#pragma unroll
    for (int i = k + 1; i < LU_NB; ++i)
      if (i < nb) a[i] = __dsub_rn(a[i], mul(L[i][k], a[k]));
#pragma unroll
  for (int i = 1; i < LU_NB; ++i)
    if (i < nb) A[(long)(k0 + i) * N + j] = a[i];
}

// Trailing update A22 -= L21 U12 for rows and columns >= k0 + LU_NB: 64 x 64 tiles, 256 threads with 4 x 4
// entries each; every entry takes the panel's updates in ascending k, separately rounded.
__global__ void __launch_bounds__(256) lu_trail_kernel(DysonBasis B, int k0) {
  __shared__ double Ls[64][LU_NB + 1];
  __shared__ double Us[LU_NB][64 + 1];
  const int b = blockIdx.z;
  const int N = (int)lu_dim(B, b);
  const int kend = min(k0 + LU_NB, N), nb = kend - k0;
  const int i0 = kend + blockIdx.y * 64, j0 = kend + blockIdx.x * 64;
  if (i0 >= N || j0 >= N) return;
  double *A = B.mats + B.moff[b];
  const int tid = threadIdx.x;
  for (int e = tid; e < 64 * LU_NB; e += 256) {
    const int i = e / LU_NB, k = e - i * LU_NB;
    Ls[i][k] = (i0 + i < N && k < nb) ? A[(long)(i0 + i) * N + k0 + k] : 0.0;
    const int kk = e / 64, jj = e - kk * 64;
    Us[kk][jj] = (j0 + jj < N && kk < nb) ? A[(long)(k0 + kk) * N + j0 + jj] : 0.0;
  }
  __syncthreads();
  const int ty = tid / 16, tx = tid - ty * 16;
  double acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = i0 + ty * 4 + a, j = j0 + tx * 4 + c;
      acc[a][c] = (i < N && j < N) ? A[(long)i * N + j] : 0.0;
    }
  for (int k = 0; k < nb; ++k) {
    double l[4], u[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) l[a] = Ls[ty * 4 + a][k];
#pragma unroll
    for (int c = 0; c < 4; ++c) u[c] = Us[k][tx * 4 + c];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][c] = __dsub_rn(acc[a][c], mul(l[a], u[c]));
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = i0 + ty * 4 + a, j = j0 + tx * 4 + c;
      if (i < N && j < N) A[(long)i * N + j] = acc[a][c];
    }
}

// Forward substitution with the unit lower factor, panel [k0, k0 + LU_NB): in-panel rows (one thread per
// right-hand-side column), then the rows below (64-row tiles).  x_ij <- fma(-L_ik, x_kj, x_ij), k ascending.
// The panel's diagonal block in shared memory (zero outside the nb x nb block), each column's nb entries in
// registers.
__global__ void __launch_bounds__(128) lu_fwd_panel_kernel(DysonBasis B, double *__restrict__ rhs, int k0) {
  __shared__ double L[LU_NB][LU_PS];
  const int b = blockIdx.x;
  const int N = (int)lu_dim(B, b), d = B.dims[b];
  if (k0 >= N) return;
  const int nb = min(LU_NB, N - k0);
  const double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  for (int e = threadIdx.x; e < LU_NB * LU_NB; e += blockDim.x) {
    const int i = e / LU_NB, k = e - i * LU_NB;
    L[i][k] = (i < nb && k < nb) ? A[(long)(k0 + i) * N + k0 + k] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < d; j += blockDim.x) {
    double xr[LU_NB];
#pragma unroll
    for (int i = 0; i < LU_NB; ++i) xr[i] = i < nb ? x[(long)(k0 + i) * d + j] : 0.0;
#pragma unroll
    for (int k = 0; k < LU_NB; ++k)
      if (k < nb) {
        const double xk = xr[k];
#pragma unroll
        for (int i = k + 1; i < LU_NB; ++i) xr[i] = fmad(-L[i][k], xk, xr[i]);
      }
#pragma unroll
    for (int i = 0; i < LU_NB; ++i)
      if (i < nb) x[(long)(k0 + i) * d + j] = xr[i];
  }
}

__global__ void __launch_bounds__(256) lu_fwd_trail_kernel(DysonBasis B, double *__restrict__ rhs, int k0) {
  __shared__ double Xs[LU_NB][129];
  const int b = blockIdx.z;
  const int N = (int)lu_dim(B, b), d = B.dims[b];
  const int kend = min(k0 + LU_NB, N), nb = kend - k0;
  const int i = kend + blockIdx.x * blockDim.y + threadIdx.y;
  const int j = blockIdx.y * 128 + threadIdx.x;
  if (kend >= N || blockIdx.y * 128 >= d) return;
  const double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  for (int e = threadIdx.y * blockDim.x + threadIdx.x; e < LU_NB * 128; e += blockDim.x * blockDim.y) {
    const int k = e / 128, jj = e - k * 128;
    Xs[k][jj] = (k < nb && blockIdx.y * 128 + jj < d) ? x[(long)(k0 + k) * d + blockIdx.y * 128 + jj] : 0.0;
  }
  __syncthreads();
  if (i >= N || j >= d) return;
  double v = x[(long)i * d + j];
  for (int k = 0; k < nb; ++k) v = fmad(-A[(long)i * N + k0 + k], Xs[k][threadIdx.x], v);
  x[(long)i * d + j] = v;
}

// Backward substitution with the upper factor, panel [k0, k0 + LU_NB) from the bottom: in-panel rows
// (x_kj <- x_kj / U_kk, then the rows above it in the panel), then the rows above the panel; k descending.
// The panel's diagonal block in shared memory, each column's nb entries in registers, as the forward panel.
__global__ void __launch_bounds__(128) lu_bwd_panel_kernel(DysonBasis B, double *__restrict__ rhs, int k0) {
  __shared__ double U[LU_NB][LU_PS];
  const int b = blockIdx.x;
  const int N = (int)lu_dim(B, b), d = B.dims[b];
  if (k0 >= N) return;
  const int nb = min(LU_NB, N - k0);
  const double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  for (int e = threadIdx.x; e < LU_NB * LU_NB; e += blockDim.x) {
    const int i = e / LU_NB, k = e - i * LU_NB;
    U[i][k] = (i < nb && k < nb) ? A[(long)(k0 + i) * N + k0 + k] : 0.0;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < d; j += blockDim.x) {
    double xr[LU_NB];
#pragma unroll
    for (int i = 0; i < LU_NB; ++i) xr[i] = i < nb ? x[(long)(k0 + i) * d + j] : 0.0;
#pragma unroll
    for (int k = LU_NB - 1; k >= 0; --k)
      if (k < nb) {
        const double xk = __ddiv_rn(xr[k], U[k][k]);
        xr[k] = xk;
#pragma unroll
        for (int i = 0; i < k; ++i) xr[i] = fmad(-U[i][k], xk, xr[i]);
      }
#pragma unroll
    for (int i = 0; i < LU_NB; ++i)
      if (i < nb) x[(long)(k0 + i) * d + j] = xr[i];
  }
}

__global__ void __launch_bounds__(256) lu_bwd_trail_kernel(DysonBasis B, double *__restrict__ rhs, int k0) {
  __shared__ double Xs[LU_NB][129];
  const int b = blockIdx.z;
  const int N = (int)lu_dim(B, b), d = B.dims[b];
  if (k0 >= N || k0 == 0 || blockIdx.y * 128 >= d) return;
  const int kend = min(k0 + LU_NB, N), nb = kend - k0;
  const int i = blockIdx.x * blockDim.y + threadIdx.y;
  const int j = blockIdx.y * 128 + threadIdx.x;
  const double *A = B.mats + B.moff[b];
  double *x = rhs + B.goff[b];
  for (int e = threadIdx.y * blockDim.x + threadIdx.x; e < LU_NB * 128; e += blockDim.x * blockDim.y) {
    const int k = e / 128, jj = e - k * 128;
    Xs[k][jj] = (k < nb && blockIdx.y * 128 + jj < d) ? x[(long)(k0 + k) * d + blockIdx.y * 128 + jj] : 0.0;
  }
  __syncthreads();
  if (i >= k0 || j >= d) return;
  double v = x[(long)i * d + j];
  for (int k = nb - 1; k >= 0; --k) v = fmad(-A[(long)i * N + k0 + k], Xs[k][threadIdx.x], v);
  x[(long)i * d + j] = v;
}

// G_out <- x, hermitized (G(t) + G(t)^T) / 2 when asked (solve_dyson, block_sparse_solver.py:582-586).
__global__ void lu_store_kernel(DysonBasis B, const double *__restrict__ rhs, double *__restrict__ G_out, int hermitize) {
  const int b = blockIdx.y;
  const int d = B.dims[b], dd = d * d;
  const double *x = rhs + B.goff[b];
  double *g = G_out + B.goff[b];
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < (long)B.r * dd; e += (long)gridDim.x * blockDim.x) {
    const int t = (int)(e / dd), ij = (int)(e - (long)t * dd), i = ij / d, j = ij - i * d;
    const double v = x[e];
    g[e] = hermitize ? mul(0.5, add(v, x[(long)t * dd + j * d + i])) : v;
  }
}

// Right-hand side x <- G0 for every block.
__global__ void lu_rhs_init_kernel(DysonBasis B, double *__restrict__ rhs) {
  const int b = blockIdx.y;
  const long n = (long)B.r * B.dims[b] * B.dims[b];
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    rhs[B.goff[b] + e] = B.g0[B.goff[b] + e];
}

}  // namespace xca
