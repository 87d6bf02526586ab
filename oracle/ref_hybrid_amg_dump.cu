// Test-only checker: runs the REFERENCE's own host builders of the mixed-mesh
// pressure preconditioner (compiled from the reference tree in place, see
// oracle/Makefile) and writes what they build to a flat record file
// (NDSDUMP1, the format of ref_setup_dump).
//
// Calls, as the reference's HXT5B start-up makes them
// (gpu/serial_cuda/hybrid_hxt5b/hxt5b_main.cu:88-90, 192, 202-204):
//   nodals_hxt1::load                      hybrid_hxt1/hxt1_mesh.hpp
//   hxt3a::build_if / hxt3a::build_b       hybrid_hxt3a/hxt3a_main.cu
//   hxt4c::build_hybrid_fine_host          hybrid_hxt5b/hybrid_amg.cuh:63
//   nodals_gpu::build_cf_hierarchy_from_csr hybrid_hxt5b/hybrid_cf_overload.inc:5
// with the HXT4B pressure pin (hybrid_hxt4b/hxt4b_main.cu:236) and an rAU
// vector read from a file of nvel doubles.  No CUDA runtime call is made
// unless --apply is given: then the reference's device preconditioner
// (hxt4c::HybridAMG, hybrid_amg.cuh:353-533) is built from that hierarchy,
// refreshed from rAU on the device and applied once to the np doubles of the
// --apply file, and the result is written to --z-out (needs a CUDA device).
#define HXT4B_EMBED_MAIN hxt4b_embedded_main
#include "hybrid_hxt4b/hxt4b_main.cu"
#undef HXT4B_EMBED_MAIN
#include "hybrid_hxt5b/hybrid_amg.cuh"

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
  void f64(const std::string& n, const std::vector<double>& v) { rec(n, "f64", v.data(), (long long)v.size(), 8); }
  void i32(const std::string& n, const std::vector<std::int32_t>& v) { rec(n, "i32", v.data(), (long long)v.size(), 4); }
  void i64(const std::string& n, const std::vector<std::int64_t>& v) { rec(n, "i64", v.data(), (long long)v.size(), 8); }
};

}  // namespace

int main(int argc, char** argv) {
  try {
    std::string mesh, rauPath, out, interp = "exti", applyPath, zPath;
    hxt4c::AMGOptions AO;
    AO.smoother = "cheb2";
    AO.chebDegree = 4;
    double theta = 0.25, safety = 1.5, lowFrac = 0.05;
    int pmax = 8, terminal = 1000, powerIts = 16, aggressive = 0;
    for (int i = 1; i < argc; ++i) {
      std::string a = argv[i];
      auto nx = [&]() -> std::string { if (i + 1 >= argc) throw std::runtime_error("missing value for " + a); return argv[++i]; };
      if (a == "--mesh") mesh = nx();
      else if (a == "--rau") rauPath = nx();
      else if (a == "--out") out = nx();
      else if (a == "--cf-theta") theta = std::atof(nx().c_str());
      else if (a == "--cf-pmax") pmax = std::atoi(nx().c_str());
      else if (a == "--cf-interp") interp = nx();
      else if (a == "--cf-aggressive-first") aggressive = std::atoi(nx().c_str());
      else if (a == "--amg-terminal") terminal = std::atoi(nx().c_str());
      else if (a == "--amg-power-its") powerIts = std::atoi(nx().c_str());
      else if (a == "--apply") applyPath = nx();
      else if (a == "--z-out") zPath = nx();
      else if (a == "--amg-smoother") AO.smoother = nx();
      else if (a == "--amg-cheb-degree") AO.chebDegree = std::atoi(nx().c_str());
      else if (a == "--amg-jacobi-omega") AO.jacobiOmega = std::atof(nx().c_str());
      else if (a == "--amg-jacobi-fine-sweeps") AO.jacobiFineSweeps = std::atoi(nx().c_str());
      else if (a == "--amg-jacobi-coarse-sweeps") AO.jacobiCoarseSweeps = std::atoi(nx().c_str());
      else if (a == "--amg-mcgs-omega") AO.mcgsOmega = std::atof(nx().c_str());
      else throw std::runtime_error("unknown arg " + a);
    }
    if (mesh.empty() || rauPath.empty() || out.empty()) throw std::runtime_error("--mesh, --rau and --out required");
    HostMesh M = nodals_hxt1::load(mesh);
    auto I3 = hxt3a::build_if(M);
    auto B = hxt3a::build_b(M, I3);
    const int nh = (int)M.h.nhex;
    int pin = 0;
    if (!M.outHex.empty()) pin = M.outHex[0].cell;
    else if (!M.outTet.empty()) pin = nh + M.outTet[0].cell;
    std::vector<double> rau((std::size_t)B.nv);
    {
      FILE* f = std::fopen(rauPath.c_str(), "rb");
      if (!f) throw std::runtime_error("cannot open " + rauPath);
      const size_t got = std::fread(rau.data(), sizeof(double), rau.size(), f);
      std::fclose(f);
      if (got != rau.size()) throw std::runtime_error("rAU file holds fewer than nvel doubles");
    }
    auto F = hxt4c::build_hybrid_fine_host(B, pin, rau);
    auto H = nodals_gpu::build_cf_hierarchy_from_csr(F.A, theta, pmax, interp, aggressive != 0, terminal, powerIts,
                                                     safety, lowFrac);
    Writer w(out);
    w.i64("pin", std::vector<std::int64_t>{pin});
    w.i64("b.row", B.row);
    w.i32("b.col", B.col);
    w.f64("b.bx", B.bx);
    w.f64("b.by", B.by);
    w.f64("b.bz", B.bz);
    w.i64("fine.row", F.A.row);
    w.i32("fine.col", F.A.col);
    w.f64("fine.val", F.A.val);
    w.f64("fine.diag", F.A.diag);
    w.i32("fine.entryRow", F.entryRow);
    w.i32("fine.diagPos", F.diagPos);
    w.i64("amg.levels", std::vector<std::int64_t>{(std::int64_t)H.csr.size()});
    w.f64("amg.fineLambda", std::vector<double>{H.fineLambda});
    w.f64("amg.levelLambda", H.levelLambda);
    for (std::size_t l = 0; l < H.P.size(); ++l) {
      const std::string p = "amg.P" + std::to_string(l) + ".";
      w.i64(p + "nCoarse", std::vector<std::int64_t>{H.P[l].nCoarse});
      w.i64(p + "row", H.P[l].row);
      w.i32(p + "col", H.P[l].col);
      w.f64(p + "val", H.P[l].val);
    }
    for (std::size_t l = 0; l < H.csr.size(); ++l) {
      const std::string p = "amg.A" + std::to_string(l) + ".";
      w.i64(p + "row", H.csr[l].row);
      w.i32(p + "col", H.csr[l].col);
      w.f64(p + "val", H.csr[l].val);
      w.f64(p + "diag", H.csr[l].diag);
    }
    w.f64("amg.terminal_inv", H.terminal_inv);
    if (!applyPath.empty()) {
      AO.lambdaLowFraction = lowFrac;
      std::vector<double> b((std::size_t)B.np), z((std::size_t)B.np);
      FILE* f = std::fopen(applyPath.c_str(), "rb");
      if (!f) throw std::runtime_error("cannot open " + applyPath);
      const size_t got = std::fread(b.data(), sizeof(double), b.size(), f);
      std::fclose(f);
      if (got != b.size()) throw std::runtime_error("--apply file holds fewer than np doubles");
      hxt4a::BDevice<double> Bd(B);
      hxt4c::HybridAMG<double> PC(F, H, pin, AO);
      hxt4c::Buf<double> dr, db, dz;
      dr.upload(rau);
      db.upload(b);
      dz.alloc(b.size());
      PC.refresh(Bd, dr.p);
      PC.apply(db.p, dz.p);
      HXT1_CUDA(cudaDeviceSynchronize());
      dz.download(z);
      FILE* g = std::fopen(zPath.c_str(), "wb");
      if (!g) throw std::runtime_error("cannot open " + zPath);
      std::fwrite(z.data(), sizeof(double), z.size(), g);
      std::fclose(g);
    }
    std::printf("NDS_REF_HYBRID_AMG_DUMP np=%d nv=%d pin=%d fineNnz=%zu levels=%zu status=PASS\n", B.np, B.nv, pin,
                F.A.val.size(), H.csr.size());
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "NDS_REF_HYBRID_AMG_DUMP_ERROR %s\n", e.what());
    return 90;
  }
}
