// Internal types shared by the host and device halves of the C ABI.
#pragma once
#include <map>
#include <string>
#include <vector>

#include "../../include/nodals_b200.h"
#include "host/amg.hpp"
#include "host/mesh.hpp"
#include "host/setup.hpp"

namespace nds {

void set_error(const std::string& e);
bool validate_options(const nds_options& o, std::string& why);
int effective_amg_power_its(const nds_options& o);

// Host setup bundle behind nds_problem*.
struct Problem {
  nds_options opt{};
  Mesh mesh;
  Setup setup;
  Hierarchy hier;
  int power_its = 0;
  // named read-only views for nds_problem_array
  std::map<std::string, nds_array> arrays;
  std::map<std::string, std::vector<double>> scalars;
  std::vector<int32_t> mesh_tets, mesh_opp;
  std::vector<double> supg_rule;  // 64 x (lambda0..3, weight) of the SUPG quadrature
  void index_arrays();
};

}  // namespace nds
