// Host-side setup of the steady P1+BF3/P0 SIMPLE problem on a pipe.
//
// Mirrors the reference start-up sequence (gpu/serial_cuda/h8_main_base.cu:1914-1938):
//   pipe geometry and boundary data        g4_host.hpp:37-49, 289-305
//   velocity unknown numbering             g3_host.hpp:29-55 (same as g2_host.hpp:52-66)
//   static diffusion CSR (nu, alpha = 1)   g3_host.hpp:286-485
//   greedy multicolouring of that graph     g3_host.hpp:614-652
//   per-cell plans (refs, row slots, J^-1) g4_host.hpp:115-175
//   static Dirichlet RHS, fixedDiv         g4_host.hpp:306-315
//   divergence coefficients B[c][a][d]     g2_host.hpp:67-76
//   initial rAU at U = 0                   g4_host.hpp:326-340, 422
//   fine pressure CSR topology             h2b_fine_csr.cuh:57-149
// Only the laminar configuration is modelled (no DG inlet, no weak wall).
#pragma once
#include <array>
#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace nds {

// stderr stage timings when NDS_SETUP_TIMING is set
class StageTimer {
 public:
  explicit StageTimer(const char* scope);
  void mark(const char* stage);

 private:
  const char* scope_;
  std::chrono::steady_clock::time_point t0_, last_;
  bool on_ = false;
};

struct PipeBC {
  int wall = -1, inlet = -1, outlet = -1;
  double cx = 0, cy = 0, z_in = 0, z_out = 0, R = 0, D = 0, L = 0;
  double bulk = 1, profile_scale = 1, nu = 0, re = 20;
  double inlet_area = 0, inlet_projected_area = 0, circle_area = 0;
  double hp_gradient = 0, hp_drop = 0;
  double inlet_normal[3] = {0, 0, -1};
  double inlet_velocity[3] = {0, 0, 1};
};

struct CsrHost {
  int n = 0;
  std::vector<int64_t> row;
  std::vector<int32_t> col;
  std::vector<double> val, diag;
  int64_t nnz() const { return row.empty() ? 0 : row.back(); }
};

// Velocity-DOF incidence + fine Schur CSR topology with the reference refresh map.
struct FineTopo {
  int n = 0, nv = 0;
  std::vector<int32_t> row, col, diag_pos;
  std::vector<int32_t> inc_off;      // free velocity dof -> incident (cell,basis)
  std::vector<uint32_t> packed;      // (cell << 3) | basis, ascending cell
  std::vector<int32_t> contrib_off;  // per pressure row: first directed contribution
  std::vector<uint8_t> slot;         // row-local CSR slot of each directed contribution
  uint32_t row_max = 0;
};

struct Setup {
  int nc = 0;          // cells = pressure unknowns
  int nv = 0;          // free velocity unknowns
  int n_vert = 0, n_face = 0;
  int n_fixed = 0;
  PipeBC pipe;
  // numbering
  std::vector<int32_t> g2free;       // entity (vertex | n_vert + face) -> free index or -1
  std::vector<int32_t> fixed_slot;   // entity -> fixed slot or -1
  std::vector<double> fixed_value;   // 3 * n_fixed
  // momentum operator topology + persistent diffusion numerics
  CsrHost mom;                       // values = diffusion K at nu (no relaxation)
  std::vector<int32_t> mom_diag_pos;
  // colouring
  int ncolors = 0;
  std::vector<int32_t> color, color_off, color_rows;
  // cells
  std::vector<int32_t> ref;          // 8 per cell: >=0 free dof, <0 -(fixed slot+1)
  std::vector<uint8_t> row_slot;     // 64 per cell: row-local slot of (a,b) or 255
  std::vector<double> det, h2, invJ; // invJ: 9 per cell, row-major J^-1
  std::vector<double> bco;           // 24 per cell: B[c][a][d]
  std::array<std::vector<double>, 3> static_rhs;
  std::vector<double> fixed_div, volume;
  // initial relaxed momentum data at U = 0
  std::vector<double> init_rau, init_delta;
  FineTopo fine;
};

struct SetupOptions {
  double re = 20.0, bulk = 1.0, alpha_u = 0.5, rau_scale = 1.0;
  bool supg = false;  // laminar SUPG terms in the setup snapshot
  double supg_tau_scale = 0.05, supg_magic = 9.0;
  std::string wall = "patch_0_0", inlet = "patch_2_0", outlet = "patch_1_0";
  int threads = 0;  // 0: all hardware threads
  // pipe centre and radius from the inlet patch's vertices instead of the
  // bounding box of the whole mesh (bent pipes, whose bounding box is not
  // the inlet disk's); the reference's rule is the bounding box
  bool geom_from_inlet = false;
};

Setup build_setup(const Mesh& m, const SetupOptions& o);

// B[c][a][d] from the cell Jacobian (g4_host.hpp:95-106 / g2_host.hpp:67-76)
double bcoeff(double det, const double* invJ, int a, int d);

// Host twins used for setup-time snapshots and for checks:
// A = K + C(U) with Dirichlet convection into conv (g4_host.hpp:326-340)
void host_assemble_central(const Setup& S, const std::array<std::vector<double>, 3>& U, std::vector<double>& aval,
                           std::array<std::vector<double>, 3>& conv);
// adds the implicit SUPG terms at U (g4_host.hpp:324-419): entries in
// ascending cell order after the convection, Dirichlet columns into conv
void host_add_supg(const Setup& S, const std::array<std::vector<double>, 3>& U, double tau_scale, double magic,
                   std::vector<double>& aval, std::array<std::vector<double>, 3>& conv);
// the implicit SUPG block S[a][b] of cell c at U (64 values, row-major)
void supg_cell_block(const Setup& S, int c, const std::array<std::vector<double>, 3>& U, double tau_scale, double magic,
                     double out[64]);
// row-L1 relaxation (g4_host.hpp:422): returns rAU; writes delta if non-null
std::vector<double> host_finalize_relax(const Setup& S, std::vector<double>& aval, double alpha_u,
                                        std::vector<double>* delta);
// exact fine Schur CSR values B diag(rau) B^T on the FineTopo pattern
CsrHost host_fine_csr(const Setup& S, const std::vector<double>& rau);

}  // namespace nds
