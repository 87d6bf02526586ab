// Output surface: VTU, Hagen-Poiseuille errors, pressure-drop fit.
#pragma once
#include <string>
#include <vector>

#include "mesh.hpp"
#include "setup.hpp"

namespace nds {

struct HpErrors {
  double h_eff = 0, u_l2 = 0, u_rel_l2 = 0, p_shifted_l2 = 0, p_shifted_rel_l2 = 0, pressure_shift = 0;
  double dp_fit = 0, dp_exact = 0, dp_rel_err = 0;
};

double pressure_drop_fit(const Mesh& m, const double* p);
HpErrors hp_errors(const Mesh& m, const Setup& S, const double* u0, const double* u1, const double* u2, const double* p);
// U0 cell average: 1/4 sum vertex + 9/40 sum face bubble (h12_vtu_output.hpp:10-24)
void cell_average_velocity(const Setup& S, const double* u0, const double* u1, const double* u2, std::vector<double>& out);
void write_vtu(const std::string& path, const Mesh& m, const Setup& S, const double* u0, const double* u1, const double* u2,
               const double* p, bool converged, int outer);

}  // namespace nds
