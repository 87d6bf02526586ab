// nodals_hxt4a_fp64: drop-in for the reference's HXT4A gate executable
// (gpu/serial_cuda/hybrid_hxt4a/hxt4a_main.cu:405-518): same flags (--mesh
// --nu --gamma --rau-scale --alpha-p --simple-tol --max-outer), same
// NODALS_HXT4A_* lines and HXT4A_PRECISION_STATUS, exit 0 on PASS, 3 on a
// failed accuracy check, 2 on an error.
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "../../include/nodals_b200.h"

int main(int argc, char** argv) {
  try {
    std::string mesh;
    double nu = 1.0, gamma = 50.0, rau_scale = 24.0, alpha_p = 1.0, simple_tol = 1e-3;
    int max_outer = 300;
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      auto next = [&]() {
        if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
        return std::string(argv[++i]);
      };
      if (a == "--mesh") mesh = next();
      else if (a == "--nu") nu = std::stod(next());
      else if (a == "--gamma") gamma = std::stod(next());
      else if (a == "--rau-scale") rau_scale = std::stod(next());
      else if (a == "--alpha-p") alpha_p = std::stod(next());
      else if (a == "--simple-tol") simple_tol = std::stod(next());
      else if (a == "--max-outer") max_outer = std::stoi(next());
      else throw std::runtime_error("unknown argument " + a);
    }
    if (mesh.empty()) throw std::runtime_error("--mesh required");
    nds_hybrid_report r{};
    if (nds_hybrid_stokes_gate(mesh.c_str(), nu, gamma, rau_scale, alpha_p, simple_tol, max_outer, 0, 1, &r) != NDS_OK)
      throw std::runtime_error(nds_last_error());
    std::printf("NODALS_HXT4A_TIMING loopMs=%.3f outer=%d status=PASS\n", r.loop_ms, r.outer_its);
    std::printf("HXT4A_PRECISION_STATUS=%s\n", r.pass ? "PASS" : "FAIL");
    return r.pass ? 0 : 3;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "HXT4A_ERROR precision=fp64: %s\n", e.what());
    std::fprintf(stderr, "HXT4A_PRECISION_STATUS=FAIL\n");
    return 2;
  }
}
