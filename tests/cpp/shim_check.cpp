// Exercises the C++ face (include/xca_b200.hpp) on the H = 0 one-fermion model with a one-pole
// hybridization (the model of test/c++/block_sparse_utils.cpp:17-42): prints Sigma of the NCA and OCA
// topologies, the order-1 single-particle correlator and the exception types of failing calls, one line
// each, for tests/test_cpp_shim.py to compare with the oracle.  Without a GPU it prints the exception
// the evaluator's constructor throws and exits 3.
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "xca_b200.hpp"

using namespace xca_b200;

int main(int argc, char **argv) {
  const double beta = 2.0, lam = 20.0, eps = 1e-10, pole = argc > 1 ? std::atof(argv[1]) : 0.0;
  block_sparse::BlockOpSymQuartet Fq;
  Fq.sym_set_labels = {0};
  Fq.dims = {1, 1};               // N = 0, N = 1
  Fq.F_index = {-1, 0};           // c maps N = 1 to N = 0
  Fq.Fd_index = {1, -1};          // c^dag maps N = 0 to N = 1
  Fq.F_data = {dcomplex(1.0, 0.0)};
  Fq.Fd_data = {dcomplex(1.0, 0.0)};
  try {
    block_sparse::DiagramEvaluator ev(beta, lam, eps, {pole}, {dcomplex(1.0, 0.0)}, Fq);
    // G0 of H = 0: G_b(tau) = -1/2 in both blocks
    BlockGf G(2, std::vector<dcomplex>(ev.r, dcomplex(-0.5, 0.0)));
    std::printf("rank %d\n", ev.r);
    for (const Topology &t : {Topology{{0, 1}}, Topology{{0, 2}, {1, 3}}}) {
      const BlockGf S = ev.compute_self_energy(G, t);
      std::printf("sigma%zu", t.size());
      for (const auto &blk : S)
        for (const auto &x : blk) std::printf(" %.17g", x.real());
      std::printf("\n");
    }
    const auto g = ev.compute_single_ptcle_gf(G, Topology{{0, 1}});
    std::printf("spgf1");
    for (const auto &x : g) std::printf(" %.17g", x.real());
    std::printf("\n");
    try {
      ev.compute_self_energy(G, Topology{{1, 0}});
      std::printf("no exception\n");
    } catch (const std::invalid_argument &) {
      std::printf("bad topology: invalid_argument\n");
    }
    try {
      ev.compute_self_energy(G, Topology{{0, 1}}, 1000000L);
      std::printf("no exception\n");
    } catch (const std::invalid_argument &) {
      std::printf("f_ix out of range: invalid_argument\n");
    } catch (const std::runtime_error &) {
      std::printf("f_ix out of range: runtime_error\n");
    }
  } catch (const std::runtime_error &e) {
    std::printf("runtime_error: %s\n", e.what());
    return 3;
  }
  return 0;
}
