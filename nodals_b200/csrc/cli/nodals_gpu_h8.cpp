// Drop-in executable for the reference's nodals_gpu_h8_fp64 / nodals_gpu_h8_fp32
// (gpu/serial_cuda/h8_main.cu, h8_main_base.cu:1748-2203).
//
// Same argv flags, same NODALS_GPU_* stdout markers consumed by
// scripts/nodals_gpu_case.py and the ANALYZE_*.py scripts, same exit codes:
// 0 pass, 35 fail / not converged, 90 exception.  The precision is taken from
// the executable name (..._fp32 -> FP32, otherwise FP64) or --precision.
// Turbulence closures (--mixing-length/--dg-inlet/--weak-wall) and SUPG are
// accepted only when disabled.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/nodals_b200.h"

namespace {

struct Fail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(int rc, const char* what) {
  if (rc != NDS_OK) throw Fail(std::string(what) + ": " + nds_last_error());
}

bool ends_with(const std::string& s, const std::string& t) {
  return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

// a regular file that starts with the HXT1 magic
bool is_hxt1(const std::string& path) {
  std::FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  char m[8] = {};
  const bool ok = std::fread(m, 1, 8, f) == 8 && std::memcmp(m, "HXT1BIN1", 8) == 0;
  std::fclose(f);
  return ok;
}

int run(int argc, char** argv) {
  nds_options o;
  nds_options_default(&o);
  std::string mesh, tag = "h8", vtu, krylov = "pcg", stageFile;
  std::string prog = argv[0];
  if (ends_with(prog, "_fp32")) o.precision = NDS_FP32;
  std::string runMode = "fixed10", momWork = "fgs1", smoother = "cheb2", hierarchy = "sa", interp = "direct",
              psolver = "pcg", coarsening = "pmis", strength = "classical-negative", spectrum = "auto",
              mcgsOrder = "symmetric", supgForm = "implicit", wallMode = "spalding";
  int supg = 0, mixlen = 0, dg = 0, weak = 0, supgQuad = 64;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto has = [&]() { return i + 1 < argc; };
    auto sv = [&]() { return std::string(argv[++i]); };
    auto dv = [&]() { return std::atof(argv[++i]); };
    auto iv = [&]() { return std::atoi(argv[++i]); };
    auto str = [&](char* dst) {
      std::string v = sv();
      std::snprintf(dst, 64, "%s", v.c_str());
    };
    if (!has()) throw Fail("H8 usage error");
    if (a == "--mesh") mesh = sv();
    else if (a == "--tag") tag = sv();
    else if (a == "--vtu-out") vtu = sv();
    else if (a == "--wall") str(o.wall);
    else if (a == "--inlet") str(o.inlet);
    else if (a == "--outlet") str(o.outlet);
    else if (a == "--re") o.re = dv();
    else if (a == "--bulk") o.bulk = dv();
    else if (a == "--mixing-length") mixlen = iv();
    else if (a == "--mixlen-scale") (void)dv();
    else if (a == "--dg-inlet") dg = iv();
    else if (a == "--weak-wall") weak = iv();
    else if (a == "--wall-traction-mode") wallMode = sv();
    else if (a == "--wall-reference-f") (void)dv();
    else if (a == "--wall-diag-csv") (void)sv();
    else if (a == "--supg") supg = iv();
    else if (a == "--supg-tau-scale") o.supg_tau_scale = dv();
    else if (a == "--supg-magic") o.supg_magic = dv();
    else if (a == "--supg-form") supgForm = sv();
    else if (a == "--supg-quad-points") supgQuad = iv();
    else if (a == "--simple-tol") o.simple_tol = dv();
    else if (a == "--max-outer") o.max_outer = iv();
    else if (a == "--alpha-u") o.alpha_u = dv();
    else if (a == "--alpha-p") o.alpha_p = dv();
    else if (a == "--rau-scale") o.rau_scale = dv();
    else if (a == "--mom-rtol") o.mom_rtol = dv();
    else if (a == "--mom-atol") o.mom_atol = dv();
    else if (a == "--mom-drop") o.mom_drop = dv();
    else if (a == "--mom-omega") o.mom_omega = dv();
    else if (a == "--mom-max") o.mom_max = iv();
    else if (a == "--p-rtol") o.p_rtol = dv();
    else if (a == "--p-atol") o.p_atol = dv();
    else if (a == "--p-max") o.p_max = iv();
    else if (a == "--snapshot-tol") o.snapshot_tol = dv();
    else if (a == "--fine-csr-refresh-every") o.fine_csr_refresh_every = iv();
    else if (a == "--amg-hierarchy") hierarchy = sv();
    else if (a == "--cf-theta") o.cf_theta = dv();
    else if (a == "--cf-pmax") o.cf_pmax = iv();
    else if (a == "--cf-interp") interp = sv();
    else if (a == "--cf-coarsening") coarsening = sv();
    else if (a == "--cf-strength") strength = sv();
    else if (a == "--cf-aggressive-first") o.cf_aggressive_first = iv();
    else if (a == "--amg-terminal") o.amg_terminal = iv();
    else if (a == "--amg-spectrum-policy") spectrum = sv();
    else if (a == "--amg-power-its") o.amg_power_its = iv();
    else if (a == "--amg-cheb-degree") o.amg_cheb_degree = iv();
    else if (a == "--amg-lambda-safety") o.amg_lambda_safety = dv();
    else if (a == "--amg-lambda-low-fraction") o.amg_lambda_low_fraction = dv();
    else if (a == "--pressure-solver") psolver = sv();
    else if (a == "--pressure-richardson-omega") o.p_richardson_omega = dv();
    else if (a == "--pressure-cheb-degree") o.p_cheb_degree = iv();
    else if (a == "--pressure-power-its") o.p_power_its = iv();
    else if (a == "--pressure-cheb-low-fraction") o.p_cheb_low_fraction = dv();
    else if (a == "--pressure-power-safety") o.p_power_safety = dv();
    else if (a == "--amg-smoother") smoother = sv();
    else if (a == "--amg-jacobi-omega") o.amg_jacobi_omega = dv();
    else if (a == "--amg-jacobi-fine-sweeps") o.amg_jacobi_fine_sweeps = iv();
    else if (a == "--amg-jacobi-coarse-sweeps") o.amg_jacobi_coarse_sweeps = iv();
    else if (a == "--amg-mcgs-omega") o.amg_mcgs_omega = dv();
    else if (a == "--amg-mcgs-fine-sweeps") o.amg_mcgs_fine_sweeps = iv();
    else if (a == "--amg-mcgs-coarse-sweeps") o.amg_mcgs_coarse_sweeps = iv();
    else if (a == "--amg-mcgs-order") mcgsOrder = sv();
    else if (a == "--momentum-work") momWork = sv();
    else if (a == "--run-mode") runMode = sv();
    else if (a == "--precision") {
      const std::string p = sv();
      if (p == "fp64") o.precision = NDS_FP64;
      else if (p == "fp32") o.precision = NDS_FP32;
      else if (p == "amg_fp32") o.precision = NDS_AMG_FP32;
      else if (p == "mixed") o.precision = NDS_MIXED;
      else throw Fail("--precision must be fp64, fp32, amg_fp32 or mixed");
    } else if (a == "--device") o.device = iv();
    // controls of the mixed-precision pressure solve (no reference counterpart)
    else if (a == "--p-krylov") krylov = sv();
    else if (a == "--p-restart") o.p_restart = iv();
    else if (a == "--p-inner-rtol") o.p_inner_rtol = dv();
    else if (a == "--p-refine-max") o.p_refine_max = iv();
    else if (a == "--p-guess") o.p_guess = iv();
    else if (a == "--p-guess-fresh") o.p_guess_fresh = iv();
    else if (a == "--amg-half") o.amg_half = iv();
    else if (a == "--learned-stage") stageFile = sv();
    else throw Fail("H8 usage error");
  }
  if (mesh.empty()) throw Fail("--mesh required");
  if (mixlen || dg || weak) throw Fail("RANS closures (--mixing-length/--dg-inlet/--weak-wall) are not part of this solver");
  o.supg = supg != 0 ? 1 : 0;
  if (o.supg) {  // laminar SUPG entry checks (h8_supg_main_cli.inc:92-95)
    if (!(o.supg_tau_scale > 0.0)) throw Fail("H8 SUPG tau scale must be positive");
    if (!(o.supg_magic > 0.0)) throw Fail("H8 SUPG magic must be positive");
    if (supgForm != "implicit") throw Fail("H8 GPU SUPG currently supports form=implicit");
    if (supgQuad != 64) throw Fail("H8 GPU SUPG currently supports quad-points=64");
  }
  (void)wallMode;
  auto pick = [](const std::string& v, std::initializer_list<const char*> names, const char* err) {
    int k = 0;
    for (const char* n : names) {
      if (v == n) return k;
      ++k;
    }
    throw Fail(err);
  };
  o.run_mode = pick(runMode, {"fixed10", "converge"}, "H8 run-mode must be fixed10 or converge");
  o.momentum_work = pick(momWork, {"fgs1", "altgs1", "sgs1"}, "H8 momentum-work must be fgs1, altgs1 or sgs1");
  o.amg_smoother = pick(smoother, {"cheb2", "jacobi", "l1jacobi", "mcgs"}, "H8 amg-smoother must be cheb2, jacobi, l1jacobi or mcgs");
  o.amg_hierarchy = pick(hierarchy, {"sa", "cf"}, "H8 amg-hierarchy must be sa or cf");
  o.cf_interp = pick(interp, {"direct", "exti"}, "H8 cf-interp must be direct or exti");
  o.pressure_solver = pick(psolver, {"pcg", "richardson", "cheb"}, "G12 pressure-solver must be pcg, richardson or cheb");
  o.amg_spectrum_policy = pick(spectrum, {"auto", "always", "off"}, "H8 amg-spectrum-policy must be auto, always or off");
  o.amg_mcgs_order = pick(mcgsOrder, {"symmetric", "forward", "backward"}, "H8 amg-mcgs-order must be symmetric, forward or backward");
  if (coarsening != "pmis") throw Fail("H8 cf-coarsening currently supports pmis");
  if (strength != "classical-negative") throw Fail("H8 cf-strength currently supports classical-negative");
  o.p_krylov = pick(krylov, {"pcg", "fgmres"}, "--p-krylov must be pcg or fgmres");
  o.learned = stageFile.empty() ? 0 : 1;
  const char* prec = o.precision == NDS_FP32       ? "fp32"
                     : o.precision == NDS_AMG_FP32 ? "amg_fp32"
                     : o.precision == NDS_MIXED    ? "mixed"
                                                   : "fp64";

  const auto t0 = std::chrono::steady_clock::now();
  nds_mesh* M = nullptr;
  if (ends_with(mesh, ".msh")) ck(nds_mesh_read_msh2(mesh.c_str(), &M), "mesh");
  else if (is_hxt1(mesh)) ck(nds_mesh_read_hxt1(mesh.c_str(), &M), "mesh");
  else ck(nds_mesh_read_polymesh(mesh.c_str(), &M), "mesh");
  nds_problem* P = nullptr;
  ck(nds_problem_create(M, &o, &P), "setup");
  nds_mesh_destroy(M);
  int nc = 0, nv = 0, ncolors = 0, levels = 0;
  nds_problem_counts(P, &nc, &nv, &ncolors, &levels);
  const double setup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  nds_solver* S = nullptr;
  ck(nds_solver_create(P, &S), "device setup");
  if (!stageFile.empty()) {
    // learned stage parameters: NDS_MPNN_NPARAM float32 values
    std::vector<float> prm(NDS_MPNN_NPARAM);
    FILE* f = std::fopen(stageFile.c_str(), "rb");
    const size_t got = f ? std::fread(prm.data(), sizeof(float), prm.size(), f) : 0;
    if (f) std::fclose(f);
    if (got != prm.size()) throw Fail("--learned-stage: cannot read " + std::to_string(prm.size()) + " parameters");
    ck(nds_solver_load_stage(S, prm.data(), (int)prm.size()), "learned stage");
  }
  const double upload_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - setup_s;
  std::printf("NODALS_GPU_H8_CONFIG tag=%s precision=%s device=B200 cells=%d runMode=%s momentumWork=%s "
              "momentumResidualPolicy=%s physicalOperator=exact_current_CSR alphaU=%.8g alphaP=%.8g simpleTol=%.3e "
              "maxOuter=%d momentumOmega=%.8g pressureRtol=%.3e pressureAtol=%.3e pressureMaxIts=%d reductions=FP64 "
              "state=%s operator=%s amg=%s\n",
              tag.c_str(), prec, nc, runMode.c_str(), momWork.c_str(),
              o.run_mode == NDS_RUN_FIXED10 ? "NONE" : "CONVERGENCE_ONLY_PRE_SWEEP", o.alpha_u, o.alpha_p,
              o.simple_tol, o.max_outer, o.mom_omega, o.p_rtol, o.p_atol, o.p_max, prec, prec, prec);
  std::printf("NODALS_GPU_H8_SETUP tag=%s cells=%d freeVel=%d colors=%d hierarchyLevels=%d hierarchy=%s smoother=%s "
              "pressureSolver=%s hostSetupSeconds=%.6f deviceSetupSeconds=%.6f status=PASS\n",
              tag.c_str(), nc, nv, ncolors, levels, hierarchy.c_str(), smoother.c_str(), psolver.c_str(), setup_s,
              upload_s);
  if (o.supg)
    std::printf("NODALS_GPU_H8_SUPG tag=%s enabled=1 form=%s quadPoints=%d tauScale=%.8g magic=%.8g "
                "setupSnapshotIncludesSUPG=1 status=PASS\n",
                tag.c_str(), supgForm.c_str(), supgQuad, o.supg_tau_scale, o.supg_magic);
  std::fflush(stdout);

  bool converged = false, pressureAll = true, finiteAll = true;
  int finalIt = 0;
  long long sumP = 0;
  int audits = 0;
  double contRel = 1.0, lastAudit[3] = {NAN, NAN, NAN};
  double tA = 0, tM = 0, tC = 0, tP = 0, tU = 0;
  const auto w0 = std::chrono::steady_clock::now();
  for (int it = 1; it <= o.max_outer; ++it) {
    nds_iter_report r{};
    const int rc = nds_simple_step(S, &r);
    if (rc != NDS_OK) throw Fail(std::string("SIMPLE iteration ") + std::to_string(it) + ": " + nds_last_error());
    finalIt = it;
    contRel = r.rel_cont;
    sumP += r.p_its;
    tA += r.ms_assembly;
    tM += r.ms_momentum;
    tC += r.ms_continuity;
    tP += r.ms_pressure;
    tU += r.ms_update;
    finiteAll = finiteAll && std::isfinite(r.rel_cont) && std::isfinite(r.p_rel);
    if (r.audited) {
      ++audits;
      for (int d = 0; d < 3; ++d) lastAudit[d] = r.audit_rel[d];
    }
    converged = r.converged != 0;
    const char* dir = o.momentum_work == NDS_MOM_FGS1 ? "FWD"
                      : o.momentum_work == NDS_MOM_SGS1 ? "FWD+BWD"
                      : (it & 1) ? "FWD" : "BWD";
    if (it <= 10 || it % 25 == 0 || r.audited || converged)
      std::printf("NODALS_GPU_H8_SIMPLE tag=%s it=%d relCont=%.12e momentumWork=%s momentumDirection=%s residualAudit=%s "
                  "auditInitRel=[%.3e,%.3e,%.3e] pCG=%d pTrueRel=%.3e allMomentumMet=%d converged=%d status=%s\n",
                  tag.c_str(), it, r.rel_cont, momWork.c_str(), dir, r.audited ? "DONE" : "SKIPPED",
                  r.audited ? r.audit_rel[0] : NAN, r.audited ? r.audit_rel[1] : NAN, r.audited ? r.audit_rel[2] : NAN,
                  r.p_its, r.p_rel, r.all_momentum_met, (int)converged, (pressureAll && finiteAll) ? "PASS" : "FAIL");
    if (o.run_mode == NDS_RUN_CONVERGE && converged) break;
  }
  const double wallMs = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
  std::vector<double> u0((size_t)nv), u1((size_t)nv), u2((size_t)nv), p((size_t)nc);
  ck(nds_get_fields(S, u0.data(), u1.data(), u2.data(), p.data()), "fields");
  if (!vtu.empty()) {
    ck(nds_write_vtu(P, vtu.c_str(), u0.data(), u1.data(), u2.data(), p.data(), converged ? 1 : 0, finalIt), "vtu");
    std::printf("NODALS_GPU_RANS_VTU path=%s cells=%d cellVelocity=U0 cellPressure=p_P0 outerIts=%d converged=%d status=PASS\n",
                vtu.c_str(), nc, finalIt, (int)converged);
  }
  nds_hp_errors E{};
  ck(nds_compute_hp_errors(P, u0.data(), u1.data(), u2.data(), p.data(), &E), "hp errors");
  std::printf("NODALS_GPU_H8_HP_ERROR tag=%s cells=%d hEff=%.12e U_L2=%.12e U_relL2=%.12e P_shifted_L2=%.12e "
              "P_shifted_relL2=%.12e pressureShift=%.12e pressureDropFit=%.12e exactPressureDrop=%.12e "
              "pressureDropRelErr=%.12e quadrature=duffy5_125 finalStateD2H=AFTER_LOOP status=%s\n",
              tag.c_str(), nc, E.h_eff, E.u_l2, E.u_rel_l2, E.p_shifted_l2, E.p_shifted_rel_l2, E.pressure_shift,
              E.dp_fit, E.dp_exact, E.dp_rel_err, converged ? "PASS" : "UNCONVERGED");
  const double n = finalIt ? (double)finalIt : 1.0;
  if (o.run_mode == NDS_RUN_FIXED10) {
    std::printf("NODALS_GPU_H8_FIXED10 tag=%s cells=%d fixedOuter=%d momentumWork=%s finalRelCont=%.12e "
                "avgPressureIts=%.6f pressureDropFit=%.12e exactPressureDrop=%.12e pressureDropRelErr=%.12e loopMs=%.3f "
                "avgSimpleMs=%.6f assemblyAvgMs=%.6f momentumAvgMs=%.6f continuityAvgMs=%.6f pressureAvgMs=%.6f "
                "pressureUpdateAvgMs=%.6f status=%s\n",
                tag.c_str(), nc, finalIt, momWork.c_str(), contRel, sumP / n, E.dp_fit, E.dp_exact, E.dp_rel_err, wallMs,
                wallMs / n, tA / n, tM / n, tC / n, tP / n, tU / n,
                (pressureAll && finiteAll && finalIt == 10) ? "PASS" : "FAIL");
  } else {
    std::printf("NODALS_GPU_H8_FULLCONV tag=%s cells=%d momentumWork=%s simpleTol=%.3e outerIts=%d converged=%d "
                "finalRelCont=%.12e convergenceAuditCalls=%d finalAuditInitRel=[%.3e,%.3e,%.3e] avgPressureIts=%.6f "
                "pressureDropFit=%.12e exactPressureDrop=%.12e pressureDropRelErr=%.12e loopMs=%.3f avgSimpleMs=%.6f "
                "assemblyAvgMs=%.6f momentumAvgMs=%.6f continuityAvgMs=%.6f pressureAvgMs=%.6f pressureUpdateAvgMs=%.6f "
                "status=%s\n",
                tag.c_str(), nc, momWork.c_str(), o.simple_tol, finalIt, (int)converged, contRel, audits, lastAudit[0],
                lastAudit[1], lastAudit[2], sumP / n, E.dp_fit, E.dp_exact, E.dp_rel_err, wallMs, wallMs / n, tA / n,
                tM / n, tC / n, tP / n, tU / n, converged ? "PASS" : "FAIL");
  }
  const bool pass = o.run_mode == NDS_RUN_FIXED10 ? (finalIt == 10 && pressureAll && finiteAll) : converged;
  std::printf("NODALS_GPU_RESULT gate=H8 tag=%s cells=%d precision=%s runMode=%s momentumWork=%s outer=%d simpleTol=%.3e "
              "fineCsrRefreshEvery=1 physicalOperator=current_exact_CSR pressureAll=%s finite=%s noPetsc=1 noMPI=1 "
              "status=%s\n",
              tag.c_str(), nc, prec, runMode.c_str(), momWork.c_str(), finalIt, o.simple_tol,
              pressureAll ? "PASS" : "FAIL", finiteAll ? "PASS" : "FAIL", pass ? "PASS" : "FAIL");
  nds_solver_destroy(S);
  nds_problem_destroy(P);
  return pass ? 0 : 35;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "NODALS_GPU_H8_EXCEPTION what=%s\n", e.what());
    return 90;
  }
}
