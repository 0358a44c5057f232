// Launchers of the Dyson, trace and normalisation kernels (dyson_kernel.cuh), every padded rank.
#include <stdexcept>
#include <string>

#include "launch.hpp"
#include "dyson_kernel.cuh"

namespace xca {

static void check_launch(const char *what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Blocked LU and substitution of every block's system (the blocked kernels of dyson_kernel.cuh); n_max is
// the largest system dimension r d_b and d_max the largest block dimension.
static int launch_blocked_lu(cudaStream_t s, const DysonBasis &B, int n_max, int d_max, double *rhs, double *G, int hermitize,
                             int *status) {
  int launches = 0;
  dim3 gi(64, (unsigned)B.nb);
  lu_rhs_init_kernel<<<gi, 256, 0, s>>>(B, rhs);
  check_launch("lu_rhs_init_kernel");
  ++launches;
  // the attribute is set to the same maximum by every caller (contexts of different sizes may call this
  // concurrently from several host threads)
  if (cudaFuncSetAttribute(lu_panel_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, LU_PANEL_SMEM_MAX_BYTES) !=
      cudaSuccess)
    check_launch("lu_panel_smem_kernel attributes");
  for (int k0 = 0; k0 < n_max; k0 += LU_NB) {
    // the panel's rows [k0, N) in shared memory where they fit, else the panel in global memory
    const size_t psm = (size_t)(n_max - k0) * LU_PS * sizeof(double);
    if (psm <= (size_t)LU_PANEL_SMEM_MAX_BYTES) {
      lu_panel_smem_kernel<<<B.nb, 1024, psm, s>>>(B, rhs, k0, status);
      check_launch("lu_panel_smem_kernel");
    } else {
      lu_panel_kernel<<<B.nb, 1024, 0, s>>>(B, rhs, k0, status);
      check_launch("lu_panel_kernel");
    }
    const int rest = n_max - k0 - LU_NB;
    if (rest > 0) {
      lu_u12_kernel<<<dim3((unsigned)((rest + 127) / 128), 1, (unsigned)B.nb), 128, 0, s>>>(B, k0);
      check_launch("lu_u12_kernel");
      const unsigned t = (unsigned)((rest + 63) / 64);
      lu_trail_kernel<<<dim3(t, t, (unsigned)B.nb), 256, 0, s>>>(B, k0);
      check_launch("lu_trail_kernel");
      launches += 2;
    }
    ++launches;
  }
  const unsigned dcol = (unsigned)((d_max + 127) / 128);
  for (int k0 = 0; k0 < n_max; k0 += LU_NB) {
    lu_fwd_panel_kernel<<<B.nb, 128, 0, s>>>(B, rhs, k0);
    check_launch("lu_fwd_panel_kernel");
    const int rest = n_max - k0 - LU_NB;
    if (rest > 0) {
      lu_fwd_trail_kernel<<<dim3((unsigned)((rest + 1) / 2), dcol, (unsigned)B.nb), dim3(128, 2), 0, s>>>(B, rhs, k0);
      check_launch("lu_fwd_trail_kernel");
      ++launches;
    }
    ++launches;
  }
  const int last = ((n_max - 1) / LU_NB) * LU_NB;
  for (int k0 = last; k0 >= 0; k0 -= LU_NB) {
    // a block whose system is smaller than k0 starts at its own last panel: the panel kernels skip
    // k0 >= N, so every block is processed from its bottom panel upward
    lu_bwd_panel_kernel<<<B.nb, 128, 0, s>>>(B, rhs, k0);
    check_launch("lu_bwd_panel_kernel");
    if (k0 > 0) {
      lu_bwd_trail_kernel<<<dim3((unsigned)((k0 + 1) / 2), dcol, (unsigned)B.nb), dim3(128, 2), 0, s>>>(B, rhs, k0);
      check_launch("lu_bwd_trail_kernel");
      ++launches;
    }
    ++launches;
  }
  lu_store_kernel<<<dim3(64, (unsigned)B.nb), 256, 0, s>>>(B, rhs, G, hermitize);
  check_launch("lu_store_kernel");
  return launches + 1;
}

template <int RP>
int launch_dyson(cudaStream_t s, const DysonBasis &B, long n_conv_rows, const double *Sigma, double eta, int hermitize, double *rhs,
                 double *G, int *status, int n_max, int d_max, int blocked_min_n, const double *op) {
  const size_t sm = (2 * (size_t)RP * RP + RP + (RP + 1) / 2) * sizeof(double);
  if (cudaFuncSetAttribute(dyson_coef_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    check_launch("dyson_coef_kernel attributes");
  dyson_coef_kernel<RP><<<B.nb, 256, sm, s>>>(B, Sigma, eta, op);
  check_launch("dyson_coef_kernel");
  dim3 grid((unsigned)((n_conv_rows + 63) / 64), (unsigned)B.nb);
  dyson_convmat_kernel<RP><<<grid, 64, 0, s>>>(B);
  check_launch("dyson_convmat_kernel");
  if (n_max > blocked_min_n) return 2 + launch_blocked_lu(s, B, n_max, d_max, rhs, G, hermitize, status);
  // the largest block's matrix (row stride N + 1) and right-hand sides in shared memory when they fit
  const size_t lu_smem = ((size_t)n_max * (n_max + 1) + (size_t)n_max * d_max) * sizeof(double);
  if (n_max <= DYSON_SMEM_MAX_N && lu_smem <= DYSON_SMEM_MAX_BYTES) {
    // the attribute is the function's, shared by every context and thread: always the same bound, so that a
    // concurrent launch with a larger system is never left below its own size
    if (cudaFuncSetAttribute(dyson_lu_solve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DYSON_SMEM_MAX_BYTES) !=
        cudaSuccess)
      check_launch("dyson_lu_solve_kernel attributes");
    dyson_lu_solve_kernel<true><<<B.nb, 1024, lu_smem, s>>>(B, rhs, G, hermitize, status);
  } else {
    dyson_lu_solve_kernel<false><<<B.nb, 1024, 0, s>>>(B, rhs, G, hermitize, status);
  }
  check_launch("dyson_lu_solve_kernel");
  return 3;
}

template <int RP>
int launch_trace_beta(cudaStream_t s, const DysonBasis &B, const double *G, double *out) {
  const size_t sm = ((size_t)RP * RP + RP + (RP + 1) / 2) * sizeof(double);
  if (cudaFuncSetAttribute(trace_beta_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    check_launch("trace_beta_kernel attributes");
  trace_beta_kernel<RP><<<B.nb, 128, sm, s>>>(B, G, out);
  check_launch("trace_beta_kernel");
  return 1;
}

template <int RP>
int launch_convolve_ppsc(cudaStream_t s, const DysonBasis &B, const double *G1, const double *G2, double *H) {
  const size_t sm = (2 * (size_t)RP * RP + RP + (RP + 1) / 2) * sizeof(double);
  if (cudaFuncSetAttribute(convolve_ppsc_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    check_launch("convolve_ppsc_kernel attributes");
  convolve_ppsc_kernel<RP><<<B.nb, 256, sm, s>>>(B, G1, G2, H);
  check_launch("convolve_ppsc_kernel");
  return 1;
}

template <int RP>
int launch_expectation_beta(cudaStream_t s, const DysonBasis &B, const double *G, const double *ops, const long *op_off, double *out) {
  const size_t sm = ((size_t)RP * RP + RP + (RP + 1) / 2) * sizeof(double);
  if (cudaFuncSetAttribute(expectation_beta_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    check_launch("expectation_beta_kernel attributes");
  expectation_beta_kernel<RP><<<B.nb, 128, sm, s>>>(B, G, ops, op_off, out);
  check_launch("expectation_beta_kernel");
  return 1;
}

int launch_energy_shift(cudaStream_t s, const DysonBasis &B, double *G, const double *fac) {
  dim3 grid(64, (unsigned)B.nb);
  energy_shift_kernel<<<grid, 256, 0, s>>>(B, G, fac);
  check_launch("energy_shift_kernel");
  return 1;
}

int launch_max_abs_diff(cudaStream_t s, int blocks, const double *a, const double *b, long n, double *out) {
  max_abs_diff_kernel<<<blocks, 256, 0, s>>>(a, b, n, out);
  check_launch("max_abs_diff_kernel");
  return 1;
}

int launch_axpby(cudaStream_t s, double alpha, const double *x, double beta, double *y, long n) {
  const long grid = n / 256 + 1 < 1184 ? n / 256 + 1 : 1184;
  axpby_kernel<<<(int)grid, 256, 0, s>>>(alpha, x, beta, y, n);
  check_launch("axpby_kernel");
  return 1;
}

template int launch_dyson<32>(cudaStream_t, const DysonBasis &, long, const double *, double, int, double *, double *, int *, int,
                               int, int, const double *);
template int launch_dyson<48>(cudaStream_t, const DysonBasis &, long, const double *, double, int, double *, double *, int *, int,
                               int, int, const double *);
template int launch_dyson<64>(cudaStream_t, const DysonBasis &, long, const double *, double, int, double *, double *, int *, int,
                               int, int, const double *);
template int launch_convolve_ppsc<32>(cudaStream_t, const DysonBasis &, const double *, const double *, double *);
template int launch_convolve_ppsc<48>(cudaStream_t, const DysonBasis &, const double *, const double *, double *);
template int launch_convolve_ppsc<64>(cudaStream_t, const DysonBasis &, const double *, const double *, double *);
template int launch_expectation_beta<32>(cudaStream_t, const DysonBasis &, const double *, const double *, const long *, double *);
template int launch_expectation_beta<48>(cudaStream_t, const DysonBasis &, const double *, const double *, const long *, double *);
template int launch_expectation_beta<64>(cudaStream_t, const DysonBasis &, const double *, const double *, const long *, double *);
template int launch_trace_beta<32>(cudaStream_t, const DysonBasis &, const double *, double *);
template int launch_trace_beta<48>(cudaStream_t, const DysonBasis &, const double *, double *);
template int launch_trace_beta<64>(cudaStream_t, const DysonBasis &, const double *, double *);

}  // namespace xca
