// nodals_hxt4b_fp64: drop-in for the reference's HXT4B mixed-mesh pipe
// SIMPLE executable (gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu:211-268):
// same flags and defaults, same NODALS_HXT4B_* lines and HXT4B_GATE_STATUS,
// exit 0 when the Hagen-Poiseuille checks pass, 3 when they fail, 2 on an
// error.  Also takes the pressure preconditioner flags of the reference's
// turbulent entry (hxt5b_main.cu:57-86): --pressure-solver pcg_amg runs the
// classical AMG V-cycle instead of Jacobi inside the pressure PCG.  The VTU (--vtu, default HXT4B_Re20.vtu) is written after the
// NODALS_HXT4B_PHYSICS line, before NODALS_HXT4B_OUTPUT; a write failure
// exits 2 as in the reference, though after PHYSICS rather than before it.
#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nodals_b200.h"

int main(int argc, char** argv) {
  try {
    std::string mesh, vtu = "HXT4B_Re20.vtu", work = "sgs1";
    std::string psolver = "pcg_jacobi", interp = "exti", smoother = "cheb2", spectrum = "auto", order = "symmetric";
    nds_hybrid_flow_options o;
    nds_hybrid_flow_defaults(&o);
    auto need = [](const std::string& v, const char* want, const char* msg) {
      if (v != want) throw std::runtime_error(msg);
    };
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
      // the pressure preconditioner flags of the reference's turbulent entry
      // (hxt5b_main.cu:57-73); pcg_jacobi keeps the HXT4B solver
      else if (a == "--pressure-solver") psolver = next();
      else if (a == "--amg-hierarchy") need(next(), "cf", "--amg-hierarchy must be cf");
      else if (a == "--cf-coarsening") need(next(), "pmis", "--cf-coarsening must be pmis");
      else if (a == "--cf-strength") need(next(), "classical-negative", "--cf-strength must be classical-negative");
      else if (a == "--cf-theta") o.cf_theta = std::stod(next());
      else if (a == "--cf-interp") interp = next();
      else if (a == "--cf-pmax") o.cf_pmax = std::stoi(next());
      else if (a == "--cf-aggressive-first") o.cf_aggressive_first = std::stoi(next());
      else if (a == "--amg-terminal") o.amg_terminal = std::stoi(next());
      else if (a == "--amg-smoother") smoother = next();
      else if (a == "--amg-jacobi-omega") o.amg_jacobi_omega = std::stod(next());
      else if (a == "--amg-jacobi-fine-sweeps") o.amg_jacobi_fine_sweeps = std::stoi(next());
      else if (a == "--amg-jacobi-coarse-sweeps") o.amg_jacobi_coarse_sweeps = std::stoi(next());
      else if (a == "--amg-cheb-degree") o.amg_cheb_degree = std::stoi(next());
      else if (a == "--amg-power-its") o.amg_power_its = std::stoi(next());
      else if (a == "--amg-lambda-safety") o.amg_lambda_safety = std::stod(next());
      else if (a == "--amg-lambda-low-fraction") o.amg_lambda_low_fraction = std::stod(next());
      else if (a == "--amg-spectrum-policy") spectrum = next();
      else if (a == "--amg-mcgs-fine-sweeps") o.amg_mcgs_fine_sweeps = std::stoi(next());
      else if (a == "--amg-mcgs-coarse-sweeps") o.amg_mcgs_coarse_sweeps = std::stoi(next());
      else if (a == "--amg-mcgs-omega") o.amg_mcgs_omega = std::stod(next());
      else if (a == "--amg-mcgs-order") order = next();
      else if (a == "--amg-separate-post") o.amg_separate_post = std::stoi(next());
      else throw std::runtime_error("unknown argument " + a);
    }
    if (mesh.empty()) throw std::runtime_error("--mesh required");
    if (!(o.alpha_u > 0 && o.alpha_u <= 1 && o.alpha_p > 0)) throw std::runtime_error("bad relaxation");
    if (work == "fgs1") o.momentum_work = 0;
    else if (work == "altgs1") o.momentum_work = 1;
    else if (work == "sgs1") o.momentum_work = 2;
    else throw std::runtime_error("momentum-work must be fgs1, altgs1, or sgs1");
    auto pick = [](const std::string& v, std::initializer_list<const char*> names, const char* msg) {
      int k = 0;
      for (const char* n : names) {
        if (v == n) return k;
        ++k;
      }
      throw std::runtime_error(msg);
    };
    o.pressure_solver = pick(psolver, {"pcg_jacobi", "pcg_amg"}, "pressure solver must be pcg_amg or pcg_jacobi");
    o.cf_interp = pick(interp, {"direct", "exti"}, "CF interp must be direct or exti");
    o.amg_smoother = pick(smoother, {"cheb2", "jacobi", "l1jacobi", "mcgs"}, "unknown AMG smoother");
    o.amg_spectrum_policy = pick(spectrum, {"auto", "always", "off"}, "bad AMG spectrum policy");
    o.amg_mcgs_order = pick(order, {"symmetric", "forward", "backward"}, "bad MCGS order");
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
