// Mixed hexahedron/tetrahedron Stokes operators (the reference's HXT gates,
// gpu/serial_cuda/hybrid_hxt2, hybrid_hxt3a, hybrid_hxt4a).
//
// Velocity: Q1 + six face bubbles ("BF2", 14 unknowns) on hexahedra, P1 +
// four cubic face bubbles (8 unknowns) on tetrahedra; one P0 pressure per
// cell.  Hexahedra and tetrahedra meet on quads, each covered by two tet
// faces; the two sides are coupled weakly by symmetric two-sided Nitsche
// terms (arithmetic flux average, penalty gamma nu / h with h = 2 V / A).
// The divergence of a cell uses its volume integral, with the trace on an
// interface triangle replaced by the average of the two sides' traces.
//
// The reference applies these operators matrix-free with atomic scatter;
// here they are assembled once on the host, row by row in a fixed order
// (the gate's operators do not change during its solve), so that the device
// only runs sparse products.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "amg.hpp"
#include "setup.hpp"

struct nds_hybrid_flow_options;

namespace nds {

struct HybridMesh {
  // nv nhex ntet nhexface ntetface nvel npressure ninterface
  // nwallhex ninhex nintet nouthex nouttet
  uint64_t count[13] = {};
  std::vector<double> xyz;                         // 3 * nv
  std::vector<std::array<int32_t, 8>> hexes;       // bottom quad, then top quad
  std::vector<std::array<int32_t, 4>> tets;
  std::vector<std::array<int32_t, 14>> hex_dofs;   // 8 vertices, 6 face bubbles
  std::vector<std::array<int32_t, 8>> tet_dofs;    // 4 vertices, 4 face bubbles
  std::vector<std::array<double, 82>> hex_geom;    // volume, h2, det J at 8 Gauss points, J^-1 (8 x 9)
  std::vector<std::array<double, 12>> tet_geom;    // volume, h2, det J, J^-1
  std::vector<std::array<int32_t, 9>> interface;   // hex cell/face/bubble, tet0 cell/face/bubble, tet1 ...
  std::vector<std::array<int32_t, 3>> wall_hex, in_hex, in_tet, out_hex, out_tet;  // cell, local face, bubble
  int nv() const { return (int)count[0]; }
  int nhex() const { return (int)count[1]; }
  int ntet() const { return (int)count[2]; }
  int nvel() const { return (int)count[5]; }
  int np() const { return nhex() + ntet(); }
};

// binary HXT1 with hex cells (hybrid_hxt1/hxt1_mesh.hpp:19-103)
HybridMesh read_hxt1_hybrid(const std::string& path);

struct InterfacePlan {
  int hex_cell, hex_face;
  int tet_cell[2], tet_face[2];
  int hex_tri_local[2][3];  // hex local vertex of each corner of the two triangles
  double normal[3];         // unit, from the hex into the tets
  double area_quad, area_tri[2];
  double inv_h_hex, inv_h_tet[2];  // A / (2 V)
};
std::vector<InterfacePlan> interface_plans(const HybridMesh& m);

struct HybridStokes {
  int nvel = 0, np = 0;
  // velocity operator: rows of fixed unknowns are identity rows
  std::vector<int32_t> a_row, a_col;
  std::vector<double> a_val;
  std::vector<double> diag_full, diag_rau;  // diag(A) and diag(A) without the Nitsche penalty
  std::vector<uint8_t> fixed;
  // divergence B (np rows, sorted columns) and its transpose (nvel rows)
  std::vector<int32_t> b_row, b_col;
  std::vector<double> bx, by, bz;
  std::vector<int32_t> bt_row, bt_col;
  std::vector<double> btx, bty, btz;
  std::vector<double> p_exact;  // manufactured pressure: axial linear, p_exact[0] = 0
};
HybridStokes build_hybrid_stokes(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double nu,
                                 double gamma);

// The production mixed-mesh SIMPLE of the reference (HXT4B,
// gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu): steady Navier-Stokes in a
// straight pipe (10 diameters) with a lagged central advective convection
// term assembled into the velocity CSR each iteration, multicolour
// Gauss-Seidel velocity sweeps, and a Jacobi-PCG pressure correction.
struct HybridFlow {
  int nvel = 0, np = 0, nhex = 0, ntet = 0;
  double radius = 0, length = 0, diameter = 0, nu = 0;
  int pin = 0;  // pressure gauge cell: the first outlet face's cell
  // velocity CSR of all unknowns (columns sorted), the constant part of its
  // values (diffusion + Nitsche) and the penalty-free diagonal of that part
  std::vector<int32_t> row, col, diag_pos;
  std::vector<double> base, diag_r_base;
  // entry k of the convection matrix = sum of local[src[q]] over q in
  // [src_off[k], src_off[k+1]): local holds 196 values per hex (row-major
  // a * 14 + b), then 64 per tet, in cell order
  std::vector<int32_t> src_off, src;
  // wall, inlet unknowns; initial state (parabolic axial velocity at every
  // vertex, the inlet bubbles corrected to the profile at the face centre)
  std::vector<uint8_t> fixed;
  std::vector<double> u0, u1, u2;
  // colours of the free unknowns: rows of colour c are colour_rows[colour_off[c] ..)
  std::vector<int32_t> colour_rows, colour_off;
  int max_colour = 0;
};
HybridFlow build_hybrid_flow(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double re, double bulk,
                             double gamma);
// the divergence operator alone (rows of HybridStokes::b_* and bt_*)
void build_hybrid_divergence(const HybridMesh& m, const std::vector<InterfacePlan>& plans, HybridStokes& H);
// Pressure matrix of the mixed-mesh SIMPLE for the AMG preconditioner
// (hybrid_hxt5b/hybrid_amg.cuh:63-125): S = B diag(rAU) B^T with the pin row
// replaced by the identity and the pin column dropped.  Row i holds i and
// every cell sharing a velocity unknown with it, sorted; each value is the
// merge of the two sorted B rows summed in extended precision.
struct HybridSchurCsr {
  CsrHost A;
  std::vector<int32_t> entry_row, diag_pos;
};
HybridSchurCsr hybrid_schur_csr(const HybridStokes& B, int pin, const std::vector<double>& rau);
// velocity operator without boundary conditions: nu-scaled diffusion of the
// hex (Q1+BF2) and tet (P1+BF3) cells, plus the Nitsche coupling of the
// interface when with_interface (CSR, columns sorted)
void hybrid_velocity_operator(const HybridMesh& m, const std::vector<InterfacePlan>& plans, double nu, double gamma,
                              bool with_interface, std::vector<int32_t>& row, std::vector<int32_t>& col,
                              std::vector<double>& val);
// pressure gauge cell of the pipe solvers: the first outlet face's cell
// (hybrid_hxt4b/hxt4b_main.cu:236)
int hybrid_pin(const HybridMesh& m);
// hierarchy options of a mixed-mesh run, checked as the reference's
// turbulent entry checks them (hxt5b_main.cu:76-86, 195-200); throws
// std::invalid_argument on a bad combination
AmgOptions hybrid_amg_options(const nds_hybrid_flow_options& o);
// axial velocity of the Hagen-Poiseuille profile
inline double pipe_profile(double x, double y, double R, double bulk) {
  const double r2 = x * x + y * y;
  const double v = 2.0 * bulk * (1.0 - r2 / (R * R));
  return v > 0 ? v : 0.0;
}

// least-squares axial pressure slope and area-weighted inlet/outlet pressure
// of a P0 field (hybrid_hxt4a/hxt4a_main.cu:339-357)
double hybrid_pressure_slope(const HybridMesh& m, const std::vector<double>& p);
double hybrid_boundary_pressure(const HybridMesh& m, const std::vector<double>& p, bool inlet);

// ASCII VTU of a mixed mesh (hybrid_hxt4b/hxt4b_main.cu:203-209): the hexes
// (VTK type 12, region 1) then the tets (type 10, region 2); vertex velocity
// (the first nv entries of each component), the P0 pressure per cell, and its
// volume-weighted vertex average (each cell gives a quarter or an eighth of
// its volume to every vertex).  Values are printed with 16 significant digits.
void write_hybrid_vtu(const HybridMesh& m, const std::string& path, const double* u0, const double* u1,
                      const double* u2, const double* p);

}  // namespace nds
