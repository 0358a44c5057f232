// Launcher of the single-particle correlator kernel (spgf_kernel.cuh) for one padded rank, XCA_RP, which
// the Makefile sets per object file.
#include <stdexcept>
#include <string>

#include "launch.hpp"

#ifndef XCA_RP
#error "XCA_RP (padded DLR rank: 32, 48 or 64) must be defined"
#endif

namespace xca {

template <int RP>
int launch_correlator(cudaStream_t s, int grid, int warps_per_cta, const DevBasis &B, const CorrBasis &CB, const CorrClass *classes,
                      const CorrChain *chains, const CorrTerm *terms, const WorkUnit *units, int n_units, int *counter,
                      const double *G, double *g, double scale, int nmax, double *scratch, long warp_doubles) {
  const size_t sm = (4 * (size_t)RP * RP + RP + (RP + 1) / 2) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(correlator_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) throw std::runtime_error(std::string("correlator_kernel attributes: ") + cudaGetErrorString(e));
  correlator_kernel<RP><<<grid, 32 * warps_per_cta, sm, s>>>(B, CB, classes, chains, terms, units, n_units, counter, G, g, scale, nmax,
                                                             scratch, warp_doubles);
  e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("correlator_kernel: ") + cudaGetErrorString(e));
  return 1;
}

template int launch_correlator<XCA_RP>(cudaStream_t, int, int, const DevBasis &, const CorrBasis &, const CorrClass *,
                                       const CorrChain *, const CorrTerm *, const WorkUnit *, int, int *, const double *, double *,
                                       double, int, double *, long);

}  // namespace xca
