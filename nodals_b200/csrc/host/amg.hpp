// Host construction of the pressure AMG hierarchies, built once at start-up
// from the initial (U = 0) rAU and kept as a setup snapshot, as the
// reference does (gpu/serial_cuda/PRESSURE_SOLVER_OPTIONS.md:93).
//
//   SA  smoothed aggregation:  g5_sa_host.hpp:1545-1580
//       greedy BFS aggregation  g2_host.hpp:84-86 (target 16, min 6, soft max 18)
//       damped-Jacobi smoothed transfer, row-normalised, <= 8 nnz/row
//       (g5_sa_host.hpp:81-108, 173-203, 491-502), Galerkin products
//       (g5_sa_host.hpp:525-546, 940-971)
//   CF  classical C/F split:     g8_cf_hierarchy_host.hpp:1584-1781
//       negative-coupling strength, PMIS with (degree, splitmix hash, index)
//       priorities (:90-106, :169-293), direct / extended+i interpolation
//       with top-pmax pruning (:625-785), Galerkin PtAP
// Terminal level: dense inverse by Cholesky (g2_host.hpp:137-138).
#pragma once
#include <string>
#include <vector>

#include "mesh.hpp"
#include "setup.hpp"

namespace nds {

struct Transfer {
  int nf = 0, nc = 0;
  std::vector<int64_t> row;
  std::vector<int32_t> col;
  std::vector<double> val;
};

struct Hierarchy {
  std::vector<std::vector<int32_t>> agg;  // SA: aggregate id per fine row, per transfer
  std::vector<Transfer> P;                // P[0]: fine -> A[0], P[l]: A[l-1] -> A[l]
  std::vector<CsrHost> A;                 // explicit coarse levels; last is terminal
  std::vector<double> fine_diag;
  double fine_lambda = 0.0;
  std::vector<double> level_lambda;       // per explicit level
  std::vector<double> terminal_inv;       // dense, row-major
  int terminal_n = 0;
};

struct AmgOptions {
  std::string hierarchy = "sa";  // sa | cf
  int terminal = 1000;
  int power_its = 16;            // 0: skip spectrum estimation
  double lambda_safety = 1.5;
  // SA
  int agg_target = 16, agg_min = 6, agg_softmax = 18, interp_max_nnz = 8;
  double sa_damping = 4.0 / 3.0;
  // CF
  double cf_theta = 0.25;
  int cf_pmax = 8;
  std::string cf_interp = "exti";  // direct | exti
  bool cf_aggressive_first = false;
};

Hierarchy build_hierarchy(const Mesh& m, const Setup& S, const std::vector<double>& rau, const AmgOptions& o);
// classical C/F hierarchy of any symmetric CSR with a positive diagonal (the
// reference's build_cf_hierarchy_from_csr, hybrid_hxt5b/hybrid_cf_overload.inc)
Hierarchy build_cf_hierarchy(CsrHost A, const AmgOptions& o);

// pieces exposed for tests
std::vector<int32_t> aggregate_graph(const std::vector<std::vector<int32_t>>& g, int target, int minsz, int softmax,
                                     int* nagg);
std::vector<double> dense_inverse_cholesky(const CsrHost& A);
double power_csr(const CsrHost& A, int its, double safety);

}  // namespace nds
