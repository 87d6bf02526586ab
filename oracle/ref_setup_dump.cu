// Test-only checker: runs the REFERENCE's own host setup builders (compiled
// from the reference tree in place, see oracle/Makefile) on a polyMesh and
// writes every setup array to a flat binary record file.  The tests compare
// the product's host setup (nodals_b200/csrc/host) against these arrays:
// integer arrays bit-exact, floating arrays to round-off.
//
// Calls, in the order the reference solver makes them at start-up
// (gpu/serial_cuda/h8_main_base.cu:1914-1938):
//   load_foam_tet_mesh            foam_mesh_g2.hpp:55
//   build_g4_setup                g4_host.hpp:289
//   host_assemble_central_g4 /
//   host_finalize_relax_g4        g4_host.hpp:326,422   (U = 0, initial rAU)
//   build_h2_fine_csr_host        h2b_fine_csr.cuh:445
//   build_sa_hierarchy            g5_sa_host.hpp:1545
//   build_cf_hierarchy            g8_cf_hierarchy_host.hpp:1584
// No CUDA runtime call is made: this binary runs on a CPU-only machine.
#define main h8_base_main   // the reference solver entry point is not used here
#include "h8_main_base.cu"    // brings every reference header (host builders + kernels)
#undef main

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct Writer {
  FILE* f = nullptr;
  explicit Writer(const std::string& p) {
    f = std::fopen(p.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot open dump output " + p);
    std::fwrite("NDSDUMP1", 1, 8, f);
  }
  ~Writer() { if (f) std::fclose(f); }
  void rec(const std::string& name, const char* dt, const void* data, long long count, int esize) {
    char nm[48] = {0};
    std::strncpy(nm, name.c_str(), 47);
    char d[8] = {0};
    std::strncpy(d, dt, 7);
    std::fwrite(nm, 1, 48, f);
    std::fwrite(d, 1, 8, f);
    std::fwrite(&count, sizeof(count), 1, f);
    if (count) std::fwrite(data, (size_t)esize, (size_t)count, f);
  }
  template <class T> void vec(const std::string& n, const std::vector<T>& v);
};
template <> void Writer::vec(const std::string& n, const std::vector<double>& v) { rec(n, "f64", v.data(), (long long)v.size(), 8); }
template <> void Writer::vec(const std::string& n, const std::vector<std::int32_t>& v) { rec(n, "i32", v.data(), (long long)v.size(), 4); }
template <> void Writer::vec(const std::string& n, const std::vector<std::int64_t>& v) { rec(n, "i64", v.data(), (long long)v.size(), 8); }
template <> void Writer::vec(const std::string& n, const std::vector<std::uint32_t>& v) { rec(n, "u32", v.data(), (long long)v.size(), 4); }
template <> void Writer::vec(const std::string& n, const std::vector<std::uint8_t>& v) { rec(n, "u8", v.data(), (long long)v.size(), 1); }

void scalar_f64(Writer& w, const std::string& n, double x) { std::vector<double> v{x}; w.vec(n, v); }
void scalar_i64(Writer& w, const std::string& n, long long x) { std::vector<std::int64_t> v{x}; w.vec(n, v); }

}  // namespace

int main(int argc, char** argv) {
  try {
    std::string mesh, out, hierarchy = "sa", interp = "exti";
    std::string wall = "patch_0_0", inlet = "patch_2_0", outlet = "patch_1_0";
    double re = 20, bulk = 1, alphaU = 0.5, theta = 0.25, safety = 1.5, lowFrac = 0.05, rauScale = 1.0;
    int pmax = 8, terminal = 1000, powerIts = 16, aggressive = 0, supg = 0;
    double supgTau = 0.05, supgMagic = 9.0;
    for (int i = 1; i < argc; ++i) {
      std::string a = argv[i];
      auto nx = [&]() -> std::string { if (i + 1 >= argc) throw std::runtime_error("missing value for " + a); return argv[++i]; };
      if (a == "--mesh") mesh = nx();
      else if (a == "--out") out = nx();
      else if (a == "--re") re = std::atof(nx().c_str());
      else if (a == "--bulk") bulk = std::atof(nx().c_str());
      else if (a == "--alpha-u") alphaU = std::atof(nx().c_str());
      else if (a == "--rau-scale") rauScale = std::atof(nx().c_str());
      else if (a == "--amg-hierarchy") hierarchy = nx();
      else if (a == "--cf-theta") theta = std::atof(nx().c_str());
      else if (a == "--cf-pmax") pmax = std::atoi(nx().c_str());
      else if (a == "--cf-interp") interp = nx();
      else if (a == "--cf-aggressive-first") aggressive = std::atoi(nx().c_str());
      else if (a == "--amg-terminal") terminal = std::atoi(nx().c_str());
      else if (a == "--power-its") powerIts = std::atoi(nx().c_str());
      else if (a == "--lambda-safety") safety = std::atof(nx().c_str());
      else if (a == "--lambda-low-fraction") lowFrac = std::atof(nx().c_str());
      else if (a == "--wall") wall = nx();
      else if (a == "--inlet") inlet = nx();
      else if (a == "--outlet") outlet = nx();
      else if (a == "--supg") supg = std::atoi(nx().c_str());
      else if (a == "--supg-tau-scale") supgTau = std::atof(nx().c_str());
      else if (a == "--supg-magic") supgMagic = std::atof(nx().c_str());
      else throw std::runtime_error("usage: unknown flag " + a);
    }
    if (mesh.empty() || out.empty()) throw std::runtime_error("--mesh and --out are required");

    auto M = load_foam_tet_mesh(mesh);
    auto S = build_g4_setup(M, re, bulk, wall, inlet, outlet, false, false);
    std::array<std::vector<double>, 3> U0;
    for (auto& u : U0) u.assign((std::size_t)S.topo.n, 0.0);
    std::vector<double> hostA, initDelta;
    std::array<std::vector<double>, 3> hostConv;
    host_assemble_central_g4(S, U0, hostA, hostConv);
    // the SUPG entry adds its host SUPG twin before relaxing (h8_supg_main_setup.inc:6-7)
    if (supg) host_add_supg64_g4(S, U0, supgTau, supgMagic, hostA, hostConv);
    auto initRau = host_finalize_relax_g4(S, hostA, alphaU, &initDelta);
    if (rauScale != 1.0) for (double& q : initRau) q *= rauScale;
    S.pressure.rAU = initRau;
    auto FH = build_h2_fine_csr_host(S);
    SAHierarchyHost H;
    if (hierarchy == "sa")
      H = build_sa_hierarchy(M, S.pressure, 16, 6, 18, terminal, 8, powerIts, safety, lowFrac, 4.0 / 3.0);
    else
      H = build_cf_hierarchy(S, FH, theta, pmax, interp, aggressive != 0, terminal, powerIts, safety, lowFrac);

    Writer w(out);
    // mesh as the reference reads it
    std::vector<std::int32_t> tets, opp;
    for (auto& t : M.tets) for (int i = 0; i < 4; ++i) tets.push_back(t[i]);
    for (auto& t : M.opp_face) for (int i = 0; i < 4; ++i) opp.push_back(t[i]);
    w.vec("mesh.tets", tets);
    w.vec("mesh.opp_face", opp);
    w.vec("mesh.face_patch", M.face_patch);
    // pipe
    scalar_f64(w, "pipe.nu", S.pipe.nu);
    scalar_f64(w, "pipe.R", S.pipe.R);
    scalar_f64(w, "pipe.L", S.pipe.L);
    scalar_f64(w, "pipe.profileScale", S.pipe.profileScale);
    scalar_f64(w, "pipe.hpDrop", S.pipe.hpDrop);
    // DOF numbering and Dirichlet data
    w.vec("g2free", S.momMask.g2free);
    std::vector<std::int32_t> fslot = S.fixedSlot;
    w.vec("fixedSlot", fslot);
    std::vector<double> fval;
    for (auto& q : S.fixedValue) for (int d = 0; d < 3; ++d) fval.push_back(q[d]);
    w.vec("fixedValue", fval);
    // momentum CSR (diffusion at nu, alpha_u = 1) and coloring
    w.vec("mom.row", S.topo.row);
    w.vec("mom.col", S.topo.col);
    w.vec("mom.val", S.topo.val);
    std::vector<std::int32_t> color = S.coloring.color;
    w.vec("color", color);
    w.vec("color.offset", S.coloring.offset);
    w.vec("color.rows", S.coloring.rows);
    // cell plans
    std::vector<std::int32_t> ref;
    std::vector<std::uint8_t> slot;
    std::vector<double> det, invJ;
    for (auto& cp : S.cells) {
      for (int a = 0; a < 8; ++a) ref.push_back(cp.ref[a]);
      for (int k = 0; k < 64; ++k) slot.push_back(cp.rowSlot[k]);
      det.push_back(cp.det);
      for (int k = 0; k < 9; ++k) invJ.push_back(cp.invJ[k]);
    }
    w.vec("cell.ref", ref);
    w.vec("cell.rowSlot", slot);
    w.vec("cell.det", det);
    w.vec("cell.invJ", invJ);
    std::vector<double> bco;
    for (std::size_t c = 0; c < S.cells.size(); ++c)
      for (int a = 0; a < 8; ++a)
        for (int d = 0; d < 3; ++d) bco.push_back(coeff(S.pressure.cells[c], a, d));
    w.vec("cell.bcoeff", bco);
    for (int d = 0; d < 3; ++d) w.vec("staticRhs" + std::to_string(d), S.staticRhs[(std::size_t)d]);
    w.vec("fixedDiv", S.fixedDiv);
    w.vec("initRau", initRau);
    w.vec("initDelta", initDelta);
    // fine pressure CSR topology and refresh map
    w.vec("fine.row", FH.row);
    w.vec("fine.col", FH.col);
    w.vec("fine.diagPos", FH.diagPos);
    w.vec("fine.incOff", FH.incOff);
    w.vec("fine.packed", FH.packed);
    w.vec("fine.contribOff", FH.contribOff);
    w.vec("fine.slot", FH.slot);
    // AMG hierarchy
    scalar_i64(w, "amg.levels", (long long)H.csr.size());
    w.vec("amg.fineDiag", H.fineDiag);
    scalar_f64(w, "amg.fineLambda", H.fineLambda);
    w.vec("amg.levelLambda", H.levelLambda);
    for (std::size_t l = 0; l < H.agg.size(); ++l) w.vec("amg.agg" + std::to_string(l), H.agg[l].id);
    for (std::size_t l = 0; l < H.P.size(); ++l) {
      const std::string p = "amg.P" + std::to_string(l) + ".";
      scalar_i64(w, p + "nCoarse", H.P[l].nCoarse);
      w.vec(p + "row", H.P[l].row);
      w.vec(p + "col", H.P[l].col);
      w.vec(p + "val", H.P[l].val);
    }
    for (std::size_t l = 0; l < H.csr.size(); ++l) {
      const std::string p = "amg.A" + std::to_string(l) + ".";
      w.vec(p + "row", H.csr[l].row);
      w.vec(p + "col", H.csr[l].col);
      w.vec(p + "val", H.csr[l].val);
      w.vec(p + "diag", H.csr[l].diag);
    }
    w.vec("amg.terminal_inv", H.terminal_inv);
    {
      const auto& CT = central_tensor_g4();
      const auto& DT = diffusion_tensor_g3();
      std::vector<double> ct(&CT.t[0][0][0][0], &CT.t[0][0][0][0] + 8 * 8 * 8 * 3);
      std::vector<double> dt(&DT.t[0][0][0][0], &DT.t[0][0][0][0] + 8 * 8 * 3 * 3);
      w.vec("centT", ct);
      w.vec("diffT", dt);
    }
    std::printf("NDS_REF_SETUP_DUMP cells=%zu freeVel=%d momNnz=%zu colors=%d fineNnz=%zu levels=%zu status=PASS\n",
                M.tets.size(), S.topo.n, S.topo.val.size(), S.coloring.ncolors, FH.col.size(), H.csr.size());
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "NDS_REF_SETUP_DUMP_ERROR %s\n", e.what());
    return 90;
  }
}
