// nodals_hxt4b_fp64: drop-in for the reference's HXT4B mixed-mesh pipe
// SIMPLE executable (gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu:211-268):
// same flags and defaults, same NODALS_HXT4B_* lines and HXT4B_GATE_STATUS,
// exit 0 when the Hagen-Poiseuille checks pass, 3 when they fail, 2 on an
// error.  The VTU (--vtu, default HXT4B_Re20.vtu) is written after the
// NODALS_HXT4B_PHYSICS line, before NODALS_HXT4B_OUTPUT; a write failure
// exits 2 as in the reference, though after PHYSICS rather than before it.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nodals_b200.h"

int main(int argc, char** argv) {
  try {
    std::string mesh, vtu = "HXT4B_Re20.vtu", work = "sgs1";
    nds_hybrid_flow_options o;
    nds_hybrid_flow_defaults(&o);
    for (int i = 1; i < argc; ++i) {
      const std::string a = argv[i];
      auto next = [&]() {
        if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
        return std::string(argv[++i]);
      };
      if (a == "--mesh") mesh = next();
      else if (a == "--vtu") vtu = next();
      else if (a == "--re") o.re = std::stod(next());
      else if (a == "--bulk") o.bulk = std::stod(next());
      else if (a == "--gamma") o.gamma = std::stod(next());
      else if (a == "--alpha-u") o.alpha_u = std::stod(next());
      else if (a == "--alpha-p") o.alpha_p = std::stod(next());
      else if (a == "--rau-scale") o.rau_scale = std::stod(next());
      else if (a == "--simple-tol") o.simple_tol = std::stod(next());
      else if (a == "--max-outer") o.max_outer = std::stoi(next());
      else if (a == "--momentum-work") work = next();
      else if (a == "--mom-omega") o.mom_omega = std::stod(next());
      else if (a == "--mom-rtol") o.mom_rtol = std::stod(next());
      else if (a == "--mom-atol") o.mom_atol = std::stod(next());
      else if (a == "--p-rtol") o.p_rtol = std::stod(next());
      else if (a == "--p-atol") o.p_atol = std::stod(next());
      else if (a == "--p-max") o.p_max = std::stoi(next());
      else throw std::runtime_error("unknown argument " + a);
    }
    if (mesh.empty()) throw std::runtime_error("--mesh required");
    if (!(o.alpha_u > 0 && o.alpha_u <= 1 && o.alpha_p > 0)) throw std::runtime_error("bad relaxation");
    if (work == "fgs1") o.momentum_work = 0;
    else if (work == "altgs1") o.momentum_work = 1;
    else if (work == "sgs1") o.momentum_work = 2;
    else throw std::runtime_error("momentum-work must be fgs1, altgs1, or sgs1");
    std::printf("NODALS_HXT4B_KERNEL_POLICY convectionBlocks=CELL_LOCAL_THEN_GATHER gsRows=WARP_PER_ROW status=PASS\n");
    uint64_t counts[13];
    if (nds_hybrid_counts(mesh.c_str(), counts) != NDS_OK) throw std::runtime_error(nds_last_error());
    std::vector<double> u0(counts[5]), u1(counts[5]), u2(counts[5]), p(counts[6]);
    nds_hybrid_flow_report r{};
    if (nds_hybrid_flow_fields(mesh.c_str(), &o, 0, 1, &r, u0.data(), u1.data(), u2.data(), p.data()) != NDS_OK)
      throw std::runtime_error(nds_last_error());
    if (nds_hybrid_write_vtu(mesh.c_str(), vtu.c_str(), u0.data(), u1.data(), u2.data(), p.data()) != NDS_OK)
      throw std::runtime_error(nds_last_error());
    std::printf("NODALS_HXT4B_TIMING loopMs=%.3f outer=%d status=PASS\n", r.loop_ms, r.outer_its);
    std::printf("NODALS_HXT4B_OUTPUT vtu=%s status=PASS\n", vtu.c_str());
    std::printf("HXT4B_GATE_STATUS=%s\n", r.pass ? "PASS" : "FAIL");
    return r.pass ? 0 : 3;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "HXT4B_ERROR precision=fp64: %s\n", e.what());
    std::fprintf(stderr, "HXT4B_GATE_STATUS=FAIL\n");
    return 2;
  }
}
