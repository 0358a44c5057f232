// Launcher of the FP32 Sigma kernel (sigma_f32.cuh) for one padded rank, XCA_RP, which the Makefile sets
// (one translation unit per rank, compiled in parallel).
#include <algorithm>
#include <stdexcept>
#include <string>

#include "launch.hpp"
#include "sigma_f32.cuh"

#ifndef XCA_RP
#error "XCA_RP (padded DLR rank: 32, 48 or 64) must be defined"
#endif

namespace xca {

template <int RP>
int launch_sigma_f32(cudaStream_t s, int nsm, const DevBasis &B, const ClassRec *classes, const WorkUnit *units, int n_units, int *counter,
                     const double *G, const SigmaOut &out) {
  const size_t smem = f32_smem_bytes<RP>();
  cudaError_t e = cudaFuncSetAttribute(sigma_f32_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) throw std::runtime_error(std::string("sigma_f32_kernel attributes: ") + cudaGetErrorString(e));
  e = cudaMemsetAsync(counter, 0, sizeof(int), s);
  if (e != cudaSuccess) throw std::runtime_error(std::string("unit counter reset: ") + cudaGetErrorString(e));
  const int grid = std::max(1, std::min(2 * nsm, n_units));
  sigma_f32_kernel<RP><<<grid, F32_THREADS, smem, s>>>(B, classes, units, n_units, counter, G, out);
  e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("sigma_f32_kernel: ") + cudaGetErrorString(e));
  return 1;
}

template int launch_sigma_f32<XCA_RP>(cudaStream_t, int, const DevBasis &, const ClassRec *, const WorkUnit *, int, int *, const double *,
                                      const SigmaOut &);

}  // namespace xca
