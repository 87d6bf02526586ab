// P1 + cubic face-bubble ("BF3") velocity element on the reference tetrahedron.
//
// Local basis (reference: gpu/serial_cuda/g3_host.hpp:73-84, g4_host.hpp:92-98):
//   phi_i     = lambda_i                       i = 0..3 (vertices)
//   phi_{4+i} = 27 lambda_j lambda_k lambda_l   {j,k,l} = {0..3} \ {i}
// i.e. bubble 4+i lives on the face opposite vertex i.  Integrals use the
// collapsed (Duffy) 5x5x5 product rule: Gauss-Jacobi in r with weight
// (1-r)^2, in s with weight (1-s), Gauss-Legendre in t, on [0,1], mapped by
//   lambda = ((1-r)(1-s)(1-t), r, (1-r)s, (1-r)(1-s)t).
// The node/weight tables are computed here from the Jacobi three-term
// recurrence by Newton's method (Golub & Welsch give the same rule).
#pragma once
#include <array>
#include <vector>

namespace nds {

struct QuadPoint {
  std::array<double, 4> lam;
  double w;
};

// n-point Gauss-Jacobi rule on [0,1] for weight (1-x)^alpha (beta = 0),
// nodes ascending.  alpha = 0 gives Gauss-Legendre.
void gauss_jacobi01(int n, int alpha, std::vector<double>& x, std::vector<double>& w);

// 125-point collapsed rule on the reference tetrahedron (weights sum to 1/6).
const std::vector<QuadPoint>& tet_rule_125();
// 64-point (4x4x4) collapsed rule of the SUPG terms, same construction
// (h7_momentum_assembly.cuh:100-226, g4_host.hpp:324-419), ordered r-major:
// point 16 ir + 4 is + it.
const std::vector<QuadPoint>& tet_rule_64();

// Reference tensors of the element:
//   D[a][b][j][k] = sum_q w_q dphi_a/dxi_j dphi_b/dxi_k            (diffusion)
//   T[a][m][b][j] = sum_q w_q phi_a phi_m dphi_b/dxi_j              (convection)
struct RefTensors {
  double D[8][8][3][3];
  double T[8][8][8][3];
};
const RefTensors& ref_tensors();

// values and reference gradients of the 8 basis functions at lam
void basis_eval(const std::array<double, 4>& lam, double phi[8], double grad[8][3]);

}  // namespace nds
