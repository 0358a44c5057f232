// Launchers of the Sigma panel kernels (sigma_panel.cuh) for one padded rank, XCA_RP, which the Makefile
// sets per object file.
#include <algorithm>
#include <stdexcept>
#include <string>

#include "launch.hpp"
#include "sigma_panel.cuh"

#ifndef XCA_RP
#error "XCA_RP (padded DLR rank: 32, 48 or 64) must be defined"
#endif

namespace xca {

static void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <int RP>
int panel_width() {
  return panel_nc<RP>();
}

template <int RP>
int launch_edge_tables(cudaStream_t s, int nsm, const DevBasis &B, const double *G, const int2 *chunks, int n_chunks) {
  const size_t smem = panel_smem_doubles<RP>() * sizeof(double);
  check(cudaFuncSetAttribute(edge_tables_panel_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
        "edge_tables_panel_kernel attributes");
  const int grid = std::max(1, std::min(n_chunks, nsm));
  edge_tables_panel_kernel<RP><<<grid, PANEL_THREADS, smem, s>>>(B, G, chunks, n_chunks);
  check(cudaGetLastError(), "edge_tables_panel_kernel");
  return 1;
}

template <int RP>
int launch_sigma_panel(cudaStream_t s, int nsm, const DevBasis &B, const ClassRec *classes, const WorkUnit *units, int n_units,
                       int *counter, const double *G, const SigmaOut &out) {
  const size_t smem = panel_smem_doubles<RP>() * sizeof(double);
  check(cudaFuncSetAttribute(sigma_panel_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
        "sigma_panel_kernel attributes");
  check(cudaMemsetAsync(counter, 0, sizeof(int), s), "unit counter reset");
  const int grid = std::max(1, std::min(nsm, n_units));
  sigma_panel_kernel<RP><<<grid, PANEL_THREADS, smem, s>>>(B, classes, units, n_units, counter, G, out);
  check(cudaGetLastError(), "sigma_panel_kernel");
  return 1;
}

template <int RP>
int launch_sigma_panel_batch(cudaStream_t s, int nsm, const SigmaJob *jobs, const WorkUnit *units, int n_units, int *counter) {
  const size_t smem = panel_smem_doubles<RP>() * sizeof(double);
  check(cudaFuncSetAttribute(sigma_panel_batch_kernel<RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
        "sigma_panel_batch_kernel attributes");
  check(cudaMemsetAsync(counter, 0, sizeof(int), s), "unit counter reset");
  const int grid = std::max(1, std::min(nsm, n_units));
  sigma_panel_batch_kernel<RP><<<grid, PANEL_THREADS, smem, s>>>(jobs, units, n_units, counter);
  check(cudaGetLastError(), "sigma_panel_batch_kernel");
  return 1;
}

template int launch_sigma_panel_batch<XCA_RP>(cudaStream_t, int, const SigmaJob *, const WorkUnit *, int, int *);
template int panel_width<XCA_RP>();
template int launch_edge_tables<XCA_RP>(cudaStream_t, int, const DevBasis &, const double *, const int2 *, int);
template int launch_sigma_panel<XCA_RP>(cudaStream_t, int, const DevBasis &, const ClassRec *, const WorkUnit *, int, int *,
                                        const double *, const SigmaOut &);

}  // namespace xca
