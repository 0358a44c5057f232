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

template <int RP>
int launch_dyson(cudaStream_t s, const DysonBasis &B, long n_conv_rows, const double *Sigma, double eta, int hermitize, double *rhs,
                 double *G, int *status) {
  const size_t sm = (2 * (size_t)RP * RP + RP + (RP + 1) / 2) * sizeof(double);
  if (cudaFuncSetAttribute(dyson_coef_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
    check_launch("dyson_coef_kernel attributes");
  dyson_coef_kernel<RP><<<B.nb, 256, sm, s>>>(B, Sigma, eta);
  check_launch("dyson_coef_kernel");
  dim3 grid((unsigned)((n_conv_rows + 63) / 64), (unsigned)B.nb);
  dyson_convmat_kernel<RP><<<grid, 64, 0, s>>>(B);
  check_launch("dyson_convmat_kernel");
  dyson_lu_solve_kernel<<<B.nb, 1024, 0, s>>>(B, rhs, G, hermitize, status);
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

template int launch_dyson<32>(cudaStream_t, const DysonBasis &, long, const double *, double, int, double *, double *, int *);
template int launch_dyson<48>(cudaStream_t, const DysonBasis &, long, const double *, double, int, double *, double *, int *);
template int launch_dyson<64>(cudaStream_t, const DysonBasis &, long, const double *, double, int, double *, double *, int *);
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
