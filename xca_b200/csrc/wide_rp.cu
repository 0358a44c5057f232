// Launcher of the wide-chain Sigma kernel (sigma_wide.cuh) for one padded rank, XCA_RP, which the Makefile
// sets per object file.
#include <stdexcept>
#include <string>

#include "launch.hpp"
#include "sigma_wide.cuh"

#ifndef XCA_RP
#error "XCA_RP (padded DLR rank: 32, 48 or 64) must be defined"
#endif

namespace xca {

template <int RP>
int launch_sigma_wide(cudaStream_t s, int grid, const DevBasis &B, const ClassRec *classes, const WorkUnit *units, int n_units,
                      int *counter, const double *G, const SigmaOut &out, double *scratch, long slab, long cta_doubles) {
  const size_t sm = wide_smem_bytes<RP>();
  cudaError_t e = cudaFuncSetAttribute(sigma_wide_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) throw std::runtime_error(std::string("sigma_wide_kernel attributes: ") + cudaGetErrorString(e));
  e = cudaMemsetAsync(counter, 0, sizeof(int), s);
  if (e != cudaSuccess) throw std::runtime_error(std::string("wide unit counter reset: ") + cudaGetErrorString(e));
  sigma_wide_kernel<RP><<<grid, WIDE_THREADS, sm, s>>>(B, classes, units, n_units, counter, G, out, scratch, slab, cta_doubles);
  e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("sigma_wide_kernel: ") + cudaGetErrorString(e));
  return 1;
}

template int launch_sigma_wide<XCA_RP>(cudaStream_t, int, const DevBasis &, const ClassRec *, const WorkUnit *, int, int *,
                                       const double *, const SigmaOut &, double *, long, long);

}  // namespace xca
