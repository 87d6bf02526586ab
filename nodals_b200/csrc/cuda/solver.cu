// Device SIMPLE solver: upload of the host setup, the pressure AMG V-cycle,
// the outer pressure solvers, one SIMPLE iteration, and the C ABI entry
// points nds_solver_*.  Numerics follow gpu/serial_cuda/h8_main_base.cu:
//   G4AMG::apply / explicit_vcycle        :544-564
//   smoothers cheb2 / jacobi / l1jacobi / mcgs  :425-542
//   pressure_pcg / richardson / cheb_poly  :569-611, :670-726
//   pressure_precond_power                 :613-668
//   g5_gpu_spectrum_refresh                :873-906
//   SIMPLE iteration                       :2046-2119
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../capi_internal.hpp"
#include "../host/fem.hpp"
#include "common.cuh"
#include "kernels.cuh"
#include "krylov.cuh"
#include "mpnn.hpp"

namespace nds {

unsigned long long g_launches = 0;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t m) {
    release();
    n = m;
    if (m) NDS_CUDA(cudaMalloc((void**)&p, m * sizeof(T)));
  }
  template <class U>
  void upload(const std::vector<U>& h) {
    if constexpr (std::is_same<U, T>::value) {
      alloc(h.size());
      if (n) NDS_CUDA(cudaMemcpy(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice));
    } else {
      std::vector<T> t(h.begin(), h.end());
      alloc(t.size());
      if (n) NDS_CUDA(cudaMemcpy(p, t.data(), n * sizeof(T), cudaMemcpyHostToDevice));
    }
  }
  void zero(cudaStream_t s) {
    if (n) NDS_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  size_t bytes() const { return n * sizeof(T); }
};

// Optional per-category CUDA-event timing of kernel launches on the solver's
// stream (the analogue of the reference's H0Profiler, h8_main_base.cu:58-99).
// fine_spmv: the physical fine operator (Krylov A p, power iterations);
// fine_spmv_amg: the fine-level operator inside the V-cycle
// fine_spmv_half: the V-cycle's fine-level operator in FP16 (amg_half)
enum ProfCat { P_FINE_SPMV = 0, P_COARSE_SPMV, P_REFRESH, P_ASSEMBLE, P_GS, P_CONTINUITY, P_TRANSFER, P_TERMINAL,
               P_VECTOR, P_FINE_AMG, P_FINE_HALF, P_NCAT };
static const char* const kProfNames[P_NCAT] = {"fine_spmv", "coarse_spmv", "fine_refresh", "mom_assemble", "mom_gs",
                                               "continuity", "transfer", "terminal_dense", "vector_reduce",
                                               "fine_spmv_amg", "fine_spmv_half"};
struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> ev;
  std::vector<int> cat;
  int used = 0;
  double total[P_NCAT] = {};
  long long calls[P_NCAT] = {};
  ~Profiler() {
    for (auto e : ev) cudaEventDestroy(e);
  }
  int begin(cudaStream_t s, int c) {
    if (!on) return -1;
    if (2 * (size_t)used + 2 > ev.size()) {
      const size_t n = ev.size();
      ev.resize(n + 512);
      cat.resize(ev.size() / 2);
      for (size_t i = n; i < ev.size(); ++i) NDS_CUDA(cudaEventCreate(&ev[i]));
    }
    const int id = used++;
    cat[(size_t)id] = c;
    NDS_CUDA(cudaEventRecord(ev[2 * (size_t)id], s));
    return id;
  }
  void end(cudaStream_t s, int id) {
    if (id >= 0) NDS_CUDA(cudaEventRecord(ev[2 * (size_t)id + 1], s));
  }
  void collect() {
    if (!used) return;
    NDS_CUDA(cudaEventSynchronize(ev[2 * (size_t)used - 1]));
    for (int i = 0; i < used; ++i) {
      float ms = 0;
      NDS_CUDA(cudaEventElapsedTime(&ms, ev[2 * (size_t)i], ev[2 * (size_t)i + 1]));
      total[cat[(size_t)i]] += ms;
      ++calls[cat[(size_t)i]];
    }
    used = 0;
  }
  void reset() {
    used = 0;
    for (int c = 0; c < P_NCAT; ++c) { total[c] = 0; calls[c] = 0; }
  }
};
struct ProfScope {
  Profiler& p;
  cudaStream_t s;
  int id;
  ProfScope(Profiler& pp, cudaStream_t ss, int c) : p(pp), s(ss), id(pp.begin(ss, c)) {}
  ~ProfScope() { p.end(s, id); }
};

struct ISolver {
  virtual ~ISolver() = default;
  virtual void reset() = 0;
  virtual void step(nds_iter_report* rep) = 0;
  virtual void solve(nds_solve_report* rep) = 0;
  virtual void get_fields(double* u0, double* u1, double* u2, double* p) = 0;
  virtual void set_fields(const double* u0, const double* u1, const double* u2, const double* p) = 0;
  // set_fields(in), step, get_fields(out), with the read-back overlapped
  // with the step where the state type and the output memory allow it
  virtual void step_io(const double* const in[4], double* const out[4], nds_iter_report* rep) = 0;
  // device cell-plan arrays read by nds_continuity_noalloc; false unless the
  // state type is double
  virtual bool cell_arrays(const int32_t** ref, const double** bco, const double** fixed_div, int* nc,
                           int* device) const = 0;
  // learned pressure stage (precision mixed, FGMRES)
  virtual void load_stage(const float* host_params) = 0;
  virtual void stage_graph(int32_t* nbr, float* ew, float* dscale) = 0;
  virtual void pressure_pair(float* rhs, float* x) = 0;
  virtual void stage_counts(long long* applied, long long* fallbacks) = 0;
  virtual void apply_operator(const float* x, float* y) = 0;
  Profiler prof;
};

struct SolveFailure : std::runtime_error {
  int code;
  SolveFailure(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

namespace {

// Exceptions cannot leave an OpenMP region: the first message is kept and
// rethrown after the region.
struct OmpErr {
  bool bad = false;
  std::string msg;
  template <class F>
  void run(F&& f) {
    try {
      f();
    } catch (const std::exception& e) {
#pragma omp critical(nds_solver_omp_error)
      if (!bad) {
        bad = true;
        msg = e.what();
      }
    }
  }
  void rethrow() const {
    if (bad) throw std::runtime_error(msg);
  }
};

std::vector<int32_t> to_i32(const std::vector<int64_t>& v, const char* what) {
  std::vector<int32_t> o(v.size());
  for (size_t i = 0; i < v.size(); ++i) {
    if (v[i] > INT32_MAX) throw std::runtime_error(std::string(what) + " exceeds int32 offsets");
    o[i] = (int32_t)v[i];
  }
  return o;
}

// greedy colouring of a CSR graph in row order (h8_main_base.cu:125-180)
void greedy_color(int n, const std::vector<int32_t>& row, const std::vector<int32_t>& col, std::vector<int32_t>& rows_out,
                  std::vector<int>& off_out) {
  std::vector<int32_t> color((size_t)n, -1);
  std::vector<int> mark(64, -1);
  int nc = 0;
  for (int i = 0; i < n; ++i) {
    for (int k = row[(size_t)i]; k < row[(size_t)i + 1]; ++k) {
      const int j = col[(size_t)k];
      if (j == i) continue;
      const int cj = color[(size_t)j];
      if (cj >= 0) {
        if ((size_t)cj >= mark.size()) mark.resize((size_t)cj + 2, -1);
        mark[(size_t)cj] = i;
      }
    }
    int c = 0;
    while ((size_t)c < mark.size() && mark[(size_t)c] == i) ++c;
    if ((size_t)c >= mark.size()) mark.resize((size_t)c + 2, -1);
    color[(size_t)i] = c;
    nc = std::max(nc, c + 1);
  }
  off_out.assign((size_t)nc + 1, 0);
  for (int i = 0; i < n; ++i) ++off_out[(size_t)color[(size_t)i] + 1];
  for (int c = 0; c < nc; ++c) off_out[(size_t)c + 1] += off_out[(size_t)c];
  rows_out.resize((size_t)n);
  std::vector<int> next(off_out.begin(), off_out.end() - 1);
  for (int i = 0; i < n; ++i) rows_out[(size_t)next[(size_t)color[(size_t)i]]++] = i;
}

// Jacobi scaling and edge weights of the learned stage's graph from the
// current FP32 operator: dscale_i = 1 / sqrt(a_ii), e_ij = a_ij dscale_i dscale_j
// (a_ij read at its SELL offset off[4 i + k]; 0 for a boundary slot)
__global__ void stage_dscale(int n, const float* __restrict__ diag, float* __restrict__ dscale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dscale[i] = diag[i] > 0.f ? rsqrtf(diag[i]) : 0.f;
}
__global__ void stage_edges(int n, const int32_t* __restrict__ nbr, const int32_t* __restrict__ off,
                            const float* __restrict__ val, const float* __restrict__ dscale, float* __restrict__ ew) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 4 * n) return;
  const int i = t >> 2, j = nbr[t];
  ew[t] = j >= 0 ? val[off[t]] * dscale[i] * dscale[j] : 0.f;
}
// after t = v - A z1: keep (t, z1) when ||t|| < ||v||, else fall back to the
// plain V-cycle (t = v, z1 = 0); counters: [0] applications, [1] fallbacks
__global__ void stage_select(int n, const float* __restrict__ v, float* __restrict__ t, float* __restrict__ z1,
                             const double* __restrict__ sc, int tt_slot, int vv_slot,
                             unsigned long long* __restrict__ cnt) {
  const bool bad = !(sc[tt_slot] < sc[vv_slot]);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    cnt[0] += 1;
    if (bad) cnt[1] += 1;
  }
  if (!bad) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    t[i] = v[i];
    z1[i] = 0.f;
  }
}
template <class Tin>
__global__ void to_float(int n, const Tin* __restrict__ a, float* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

double cheb_root(double hi, double lo, int k, int degree) {
  const double centre = .5 * (hi + lo), radius = .5 * (hi - lo), pi = 3.141592653589793238462643383279502884;
  return centre - radius * std::cos(pi * (2.0 * (double)k + 1.0) / (2.0 * (double)degree));
}

}  // namespace

// T: state, momentum and pressure-operator precision (and the outer Krylov
// vectors); TA: precision of the AMG V-cycle (levels, transfers, smoothers,
// fine-level copy of the operator).  T == TA for the FP64 and FP32 modes;
// the mixed mode runs an FP32 V-cycle inside FP64 PCG.
template <class T, class TA>
class Solver final : public ISolver {
 public:
  static constexpr bool kSame = std::is_same<T, TA>::value;
  struct Level {  // explicit AMG level
    int n = 0;
    DBuf<int32_t> row, col, crows;
    std::vector<int> coff;
    DBuf<TA> val, diag, l1, b, x, r, tmp, corr, pong;
    // amg_half: FP16 copy of the level's CSR values, scaled by 1 / hinv,
    // and its columns as 16-bit deltas to the row when they all fit
    DBuf<__half> hval;
    DBuf<int16_t> hcol;
    double hinv = 1.0;
  };
  struct Xfer {  // P (fine rows, ELL k-major) and R = P^T (coarse rows, CSR)
    int nf = 0, nc = 0, pw = 0;
    DBuf<int32_t> pcol, rrow, rcol;
    DBuf<TA> pval, rval;
  };

  Solver(const Problem& P) : P_(P), o_(P.opt) {
    NDS_CUDA(cudaSetDevice(o_.device));
    NDS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    NDS_CUDA(cudaStreamCreateWithFlags(&st2_, cudaStreamNonBlocking));
    NDS_CUDA(cudaStreamCreateWithFlags(&st_io_, cudaStreamNonBlocking));
    NDS_CUDA(cudaEventCreateWithFlags(&ev_io_, cudaEventDisableTiming));
    for (auto& e : ev_side_) NDS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : ev_) NDS_CUDA(cudaEventCreate(&e));
    upload();
  }
  ~Solver() override {
    for (auto& e : ev_)
      if (e) cudaEventDestroy(e);
    if (hsc_) cudaFreeHost(hsc_);
    if (hflags_) cudaFreeHost(hflags_);
    for (auto& e : ev_side_)
      if (e) cudaEventDestroy(e);
    if (ev_io_) cudaEventDestroy(ev_io_);
    if (st_io_) cudaStreamDestroy(st_io_);
    if (st2_) cudaStreamDestroy(st2_);
    if (st_) cudaStreamDestroy(st_);
  }

  // ------------------------------------------------------------------ setup
  void upload() {
    const Setup& S = P_.setup;
    const Hierarchy& H = P_.hier;
    StageTimer tm("device_upload");
    nc_ = S.nc;
    nv_ = S.nv;
    {
      // The momentum matrix is stored colour by colour: the Gauss-Seidel
      // pass of one colour then streams one contiguous block.  Each row
      // starts on a 32-byte boundary and is padded to a whole number of
      // 32-byte sectors (pad entries: column = the row itself, value 0), so
      // the assembly, which visits the rows in their natural order, writes
      // whole sectors.  The assembly and the audit address row i through
      // its span; the pads add zeros, so every value and sum is the one of
      // the natural order.  NDS_MOM_NATURAL_ORDER=1 keeps the natural CSR.
      const bool natural = std::getenv("NDS_MOM_NATURAL_ORDER") != nullptr;
      const int64_t pad = natural ? 1 : (int64_t)(32 / sizeof(T));
      int64_t nz = natural ? S.mom.row[(size_t)nv_] : 0;
      std::vector<int64_t> pos(natural ? 0 : (size_t)nv_);
      for (int q = 0; q < nv_ && !natural; ++q) {
        const int i = S.color_rows[(size_t)q];
        const int64_t len = S.mom.row[(size_t)i + 1] - S.mom.row[(size_t)i];
        pos[(size_t)i] = nz;
        nz += (len + pad - 1) / pad * pad;
      }
      if (nz > (int64_t)INT32_MAX) throw std::runtime_error("momentum CSR exceeds int32 offsets");
      std::vector<int32_t> col((size_t)nz), dpos((size_t)nv_);
      std::vector<int2> span((size_t)nv_);
      std::vector<T> kv((size_t)nz, T(0));
#pragma omp parallel for schedule(static)
      for (int i = 0; i < nv_; ++i) {
        const int64_t rb = S.mom.row[(size_t)i], re = S.mom.row[(size_t)i + 1];
        const int64_t cb = natural ? rb : pos[(size_t)i];
        const int64_t ce = natural ? re : cb + (re - rb + pad - 1) / pad * pad;
        span[(size_t)i] = make_int2((int)cb, (int)ce);
        dpos[(size_t)i] = (int32_t)(cb + (S.mom_diag_pos[(size_t)i] - rb));
        for (int64_t k = rb; k < re; ++k) {
          col[(size_t)(cb + (k - rb))] = S.mom.col[(size_t)k];
          kv[(size_t)(cb + (k - rb))] = (T)S.mom.val[(size_t)k];
        }
        for (int64_t k = cb + (re - rb); k < ce; ++k) col[(size_t)k] = i;
      }
      std::vector<int2> gspan((size_t)nv_);
#pragma omp parallel for schedule(static)
      for (int q = 0; q < nv_; ++q) gspan[(size_t)q] = span[(size_t)S.color_rows[(size_t)q]];
      mspan_.upload(span);
      gspan_.upload(gspan);
      mcol_.upload(col);
      mdpos_.upload(dpos);
      K_.upload(kv);
      A_.alloc((size_t)nz);
    }
    diag_.alloc((size_t)nv_);
    delta_.alloc((size_t)nv_);
    rau_.upload(S.init_rau);
    rau_pc_.upload(S.init_rau);
    inc_off_.upload(S.fine.inc_off);
    inc_.upload(S.fine.packed);
    ref_.upload(S.ref);
    slot_.upload(S.row_slot);
    det_.upload(S.det);
    invJ_.upload(S.invJ);
    bco_.upload(S.bco);
    fixed_.upload(S.fixed_value);
    fixed_div_.upload(S.fixed_div);
    for (int d = 0; d < 3; ++d) {
      s_[d].upload(S.static_rhs[(size_t)d]);
      b_[d].alloc((size_t)nv_);
      v_[d].alloc((size_t)nv_);
    }
    u3_.alloc((size_t)kVelComponents * nv_);
    NDS_CUDA(cudaMemset(u3_.p, 0, u3_.bytes()));
    p_.alloc((size_t)nc_);
    color_rows_.upload(S.color_rows);
    color_off_ = S.color_off;
    {
      const RefTensors& RT = ref_tensors();
      std::vector<double> t(1536);
      std::memcpy(t.data(), &RT.T[0][0][0][0], sizeof(double) * 1536);
      centT_.upload(t);
    }
    row_cap_ = 8;
    for (int i = 0; i < nv_; ++i) row_cap_ = std::max<int>(row_cap_, (int)(S.mom.row[(size_t)i + 1] - S.mom.row[(size_t)i]));
    row_cap_ = (row_cap_ + 7) / 8 * 8;
    mom_smem_ = (size_t)(kBlock / 8) * row_cap_ * sizeof(T);
    if (mom_smem_ > 200 * 1024) throw std::runtime_error("momentum row too long for the shared-memory assembly buffer");
    NDS_CUDA(cudaFuncSetAttribute(k::mom_assemble<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mom_smem_));
    NDS_CUDA(cudaFuncSetAttribute(k::mom_assemble<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(mom_smem_ + 1536 * sizeof(T))));
    // The two-pass assembly by default: the cell pass writes each cell's
    // convection block row by row into the incidence slots of the velocity
    // rows (8 values per incidence, contiguous per row), the row pass
    // streams them.  NDS_FUSED_ASSEMBLY=1 (not with SUPG) evaluates the
    // convection rows inside the row pass instead.
    fused_assembly_ = !o_.supg && std::getenv("NDS_FUSED_ASSEMBLY") != nullptr;
    if (!fused_assembly_) {
      const size_t nz = S.fine.packed.size();
      std::vector<int32_t> zpos(8 * (size_t)nc_, -1);
      std::vector<uint8_t> slotz(8 * nz), fixz(nz, 0);
      std::vector<T> bz(3 * nz);
#pragma omp parallel for schedule(static)
      for (size_t z = 0; z < nz; ++z) {
        const uint32_t pa = S.fine.packed[z];
        const size_t c = pa >> 3, a = pa & 7u;
        zpos[8 * c + a] = (int32_t)z;
        for (int d = 0; d < 3; ++d) bz[3 * z + (size_t)d] = (T)S.bco[24 * c + 3 * a + (size_t)d];
        for (int b = 0; b < 8; ++b) {
          slotz[8 * z + (size_t)b] = S.row_slot[64 * c + 8 * a + (size_t)b];
          if (S.ref[8 * c + (size_t)b] < 0) fixz[z] |= (uint8_t)(1u << b);
        }
      }
      zpos_.upload(zpos);
      slotz_.upload(slotz);
      fixz_.upload(fixz);
      bz_.upload(bz);
      pz_.alloc(nz);
      cconv_.alloc(8 * nz);
    }

    if (o_.supg) {
      h2_.upload(S.h2);
      std::vector<double> rule;
      for (const auto& q : tet_rule_64()) {
        for (int k = 0; k < 4; ++k) rule.push_back(q.lam[(size_t)k]);
        rule.push_back(q.w);
      }
      supg_rule_.upload(rule);
    }

    tm.mark("momentum_and_cells");
    // fine Schur refresh contributions, regrouped by destination slot in the
    // reference's order and laid out in runs (one run per fine entry, the
    // longest first) that never straddle a 32-contribution chunk of the row: a run that would
    // cross a chunk boundary starts the next chunk, the gap is filled with
    // pad entries.  Per contribution: the code word cs (basis a bits 0-2,
    // position in its run bits 3-5, run tail bit 6, slot bits 7-15; pads are
    // 0xFFFF) and the packed incidence (c2 << 3 | b) for the geometry.
    const FineTopo& F = S.fine;
    {
      std::vector<int32_t> plen((size_t)nc_ + 1, 0);
      std::vector<int32_t> poff((size_t)nc_ + 1, 0);
      OmpErr oerr;
      // pass 1: counts per slot and padded row lengths.  A row's runs are
      // laid out longest first (stable in slot order), so the few long runs
      // share a chunk and the chunks of short runs need few chain steps;
      // the order of the contributions inside a run is unchanged.
      std::vector<uint8_t> cnt(F.col.size(), 0);
      auto run_order = [&](int rb, int len, std::vector<int32_t>& ord) {
        ord.clear();
        for (int sl = 0; sl < len; ++sl)
          if (cnt[(size_t)rb + sl]) ord.push_back(sl);
        std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) {
          return cnt[(size_t)rb + x] > cnt[(size_t)rb + y];
        });
      };
#pragma omp parallel
      {
        std::vector<int32_t> ord;
#pragma omp for schedule(dynamic, 1024)
        for (int c = 0; c < nc_; ++c) {
          oerr.run([&] {
            const int rb = F.row[(size_t)c], len = F.row[(size_t)c + 1] - rb;
            for (int q = F.contrib_off[(size_t)c]; q < F.contrib_off[(size_t)c + 1]; ++q) {
              // the code word holds a position in the run in three bits
              if (cnt[(size_t)rb + F.slot[(size_t)q]] == 8)
                throw std::runtime_error("more than 8 contributions to one fine entry");
              ++cnt[(size_t)rb + F.slot[(size_t)q]];
            }
            if (cnt[(size_t)F.diag_pos[(size_t)c]] == 0)
              throw std::runtime_error("fine Schur row without a diagonal contribution");
            run_order(rb, len, ord);
            int L = 0;
            for (const int32_t sl : ord) {
              const int n = cnt[(size_t)rb + sl];
              if ((L & 31) + n > 32) L = (L + 31) & ~31;
              L += n;
            }
            plen[(size_t)c + 1] = L;
          });
        }
      }
      oerr.rethrow();
      for (int c = 0; c < nc_; ++c) poff[(size_t)c + 1] = poff[(size_t)c] + plen[(size_t)c + 1];
      const size_t nq = (size_t)poff[(size_t)nc_];
      std::vector<uint16_t> cs(nq, 0xFFFF);
      std::vector<uint32_t> cpk(nq, 0);
      // pass 2: stable placement (the order of (a, incidence)) into the runs
#pragma omp parallel
      {
        std::vector<int32_t> start, fill, ord;
#pragma omp for schedule(dynamic, 1024)
        for (int c = 0; c < nc_; ++c) {
          const int rb = F.row[(size_t)c], len = F.row[(size_t)c + 1] - rb;
          start.assign((size_t)len, 0);
          fill.assign((size_t)len, 0);
          run_order(rb, len, ord);
          int L = 0;
          for (const int32_t sl : ord) {
            const int n = cnt[(size_t)rb + sl];
            if ((L & 31) + n > 32) L = (L + 31) & ~31;
            start[(size_t)sl] = L;
            L += n;
          }
          const size_t o = (size_t)poff[(size_t)c];
          int q = F.contrib_off[(size_t)c];
          for (int a = 0; a < 8; ++a) {
            const int g = S.ref[8 * (size_t)c + a];
            if (g < 0) continue;
            for (int k = F.inc_off[(size_t)g]; k < F.inc_off[(size_t)g + 1]; ++k, ++q) {
              const int sl = F.slot[(size_t)q], n = cnt[(size_t)rb + sl];
              const int pos = fill[(size_t)sl]++;
              const size_t at = o + (size_t)(start[(size_t)sl] + pos);
              cpk[at] = F.packed[(size_t)k];
              cs[at] = (uint16_t)(((unsigned)sl << 7) | ((pos == n - 1) ? 64u : 0u) | ((unsigned)pos << 3) | (unsigned)a);
            }
          }
        }
      }
      fcoff_.upload(poff);
      fcs_.upload(cs);
      DBuf<uint32_t> cpk_d;
      cpk_d.upload(cpk);
      fgeo_.alloc(nq);
      k::refresh_geometry<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, fcoff_.p, cpk_d.p, fcs_.p, bco_.p, fgeo_.p);
      NDS_LAUNCH();
      NDS_CUDA(cudaStreamSynchronize(st_));
    }
    {
      tm.mark("refresh_contributions");
      // SELL-32x4 layout of the fine pattern (entry k of row 32 s + l at
      // base[s] + 128 (k/4) + 4 l + k%4, rows padded to a multiple of 4)
      const int ns = (nc_ + 31) / 32;
      std::vector<int32_t> width((size_t)ns, 0), base((size_t)ns + 1, 0), dslot((size_t)nc_);
      for (int c = 0; c < nc_; ++c) {
        const int len = F.row[(size_t)c + 1] - F.row[(size_t)c];
        width[(size_t)(c >> 5)] = std::max(width[(size_t)(c >> 5)], len);
        dslot[(size_t)c] = F.diag_pos[(size_t)c] - F.row[(size_t)c];
      }
      auto padded = [&](int q) { return (width[(size_t)q] + 3) & ~3; };
      auto offset = [&](int q, int l, int k) {
        return (size_t)base[(size_t)q] + 128 * (size_t)(k >> 2) + 4 * (size_t)l + (size_t)(k & 3);
      };
      for (int q = 0; q < ns; ++q) {
        const int64_t nb = (int64_t)base[(size_t)q] + 32LL * padded(q);
        if (nb > INT32_MAX) throw std::runtime_error("SELL fine operator exceeds int32 offsets");
        base[(size_t)q + 1] = (int32_t)nb;
      }
      // padding entries point at their own row; lanes past the last row of
      // the final slice point at row 0 (never read by a live thread)
      std::vector<int32_t> scol((size_t)base[(size_t)ns]);
#pragma omp parallel for schedule(static)
      for (int q = 0; q < ns; ++q)
        for (int l = 0; l < 32; ++l) {
          const int c = 32 * q + l;
          const int rb = c < nc_ ? F.row[(size_t)c] : 0, len = c < nc_ ? F.row[(size_t)c + 1] - rb : 0;
          for (int kk = 0; kk < padded(q); ++kk) scol[offset(q, l, kk)] = kk < len ? F.col[(size_t)rb + kk] : (c < nc_ ? c : 0);
        }
      swidth_.upload(width);
      int wmax = 0;
      for (int q = 0; q < ns; ++q) wmax = std::max(wmax, padded(q));
      refresh_smem_ = (size_t)33 * wmax * sizeof(T);
      if (refresh_smem_ > 200 * 1024) throw std::runtime_error("fine Schur row too long for the refresh slice buffer");
      NDS_CUDA(cudaFuncSetAttribute(k::sell_refresh<T, TA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)refresh_smem_));
      sbase_.upload(base);
      fdslot_.upload(dslot);
      fval_.alloc(scol.size());
      NDS_CUDA(cudaMemset(fval_.p, 0, fval_.bytes()));
      if (!kSame) {
        fvalA_.alloc(scol.size());
        NDS_CUDA(cudaMemset(fvalA_.p, 0, fvalA_.bytes()));
      }
      // 16-bit column deltas when the ordering keeps every |column - row| < 2^15
      int too_far = 0;
      std::vector<int16_t> dcol(scol.size());
#pragma omp parallel for schedule(static) reduction(| : too_far)
      for (int q = 0; q < ns; ++q)
        for (int l = 0; l < 32; ++l) {
          const int row = 32 * q + l;
          for (int kk = 0; kk < padded(q); ++kk) {
            const size_t o = offset(q, l, kk);
            const int d = row < nc_ ? scol[o] - row : 0;
            if (d < -32767 || d > 32767) too_far = 1;
            else dcol[o] = (int16_t)d;
          }
        }
      const bool fits = too_far == 0;
      if (fits && !std::getenv("NDS_SELL_COL32")) {
        sdcol_.upload(dcol);
        sell_ = k::Sell{nc_, sbase_.p, swidth_.p, nullptr, sdcol_.p};
      } else {
        scol_.upload(scol);
        sell_ = k::Sell{nc_, sbase_.p, swidth_.p, scol_.p, nullptr};
      }
      sell_nnz_ = (long long)scol.size();
    }
    tm.mark("sell_layout");
    fdiag_.upload(H.fine_diag);
    const bool l1 = o_.amg_smoother == NDS_SM_L1JACOBI;
    if (l1) fl1_.alloc((size_t)nc_);
    if (o_.amg_smoother == NDS_SM_MCGS) {
      std::vector<int32_t> rows;
      greedy_color(nc_, F.row, F.col, rows, fine_coff_);
      fine_crows_.upload(rows);
    }
    for (auto* b : {&x_, &r_, &z_, &pp_, &q_, &rhs_}) b->alloc((size_t)nc_);
    for (auto* b : {&fr_, &ftmp_, &fcorr_, &frhs_, &fpong_}) b->alloc((size_t)nc_);
    if (!kSame) {
      rA_.alloc((size_t)nc_);
      zA_.alloc((size_t)nc_);
    }

    // AMG levels and transfers
    L_.resize(H.A.size());
    for (size_t l = 0; l < H.A.size(); ++l) {
      const CsrHost& A = H.A[l];
      Level& Lv = L_[l];
      Lv.n = A.n;
      Lv.row.upload(to_i32(A.row, "AMG level CSR"));
      Lv.col.upload(A.col);
      Lv.val.upload(A.val);
      Lv.diag.upload(A.diag);
      std::vector<double> l1h((size_t)A.n);
#pragma omp parallel for schedule(static)
      for (int i = 0; i < A.n; ++i) {
        double ss = 0.0;
        for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) ss += std::abs(A.val[(size_t)k]);
        l1h[(size_t)i] = ss;
      }
      Lv.l1.upload(l1h);
      for (auto* b : {&Lv.b, &Lv.x, &Lv.r, &Lv.tmp, &Lv.corr, &Lv.pong}) b->alloc((size_t)A.n);
      // the mixed path's V-cycle reads FP16 copies of the explicit levels
      // (the terminal level goes through its dense inverse)
      if (!kSame && o_.precision == NDS_MIXED && o_.amg_half && l + 1 < H.A.size()) level_to_half(Lv, A);
      if (o_.amg_smoother == NDS_SM_MCGS && l + 1 < H.A.size()) {
        std::vector<int32_t> rows;
        std::vector<int32_t> r32 = to_i32(A.row, "AMG level CSR");
        greedy_color(A.n, r32, A.col, rows, Lv.coff);
        Lv.crows.upload(rows);
      }
    }
    X_.resize(H.P.size());
    for (size_t l = 0; l < H.P.size(); ++l) {
      const Transfer& Ph = H.P[l];
      Xfer& X = X_[l];
      X.nf = Ph.nf;
      X.nc = Ph.nc;
      {
        // P in ELL, entry k of fine row i at k nf + i (coalesced across rows);
        // padding entries carry value 0 and coarse column 0
        int pw = 0;
        for (int i = 0; i < Ph.nf; ++i) pw = std::max<int>(pw, (int)(Ph.row[(size_t)i + 1] - Ph.row[(size_t)i]));
        std::vector<int32_t> ec((size_t)pw * Ph.nf, 0);
        std::vector<double> ev((size_t)pw * Ph.nf, 0.0);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < Ph.nf; ++i)
          for (int64_t q = Ph.row[(size_t)i]; q < Ph.row[(size_t)i + 1]; ++q) {
            const size_t o = (size_t)(q - Ph.row[(size_t)i]) * Ph.nf + i;
            ec[o] = Ph.col[(size_t)q];
            ev[o] = Ph.val[(size_t)q];
          }
        X.pw = pw;
        X.pcol.upload(ec);
        X.pval.upload(ev);
      }
      // R = P^T, entries of each coarse row in ascending fine row
      std::vector<int32_t> rr((size_t)Ph.nc + 1, 0), rc(Ph.col.size());
      std::vector<double> rv(Ph.col.size());
      for (int32_t c : Ph.col) ++rr[(size_t)c + 1];
      for (int c = 0; c < Ph.nc; ++c) rr[(size_t)c + 1] += rr[(size_t)c];
      std::vector<int32_t> pos(rr.begin(), rr.end() - 1);
      for (int i = 0; i < Ph.nf; ++i)
        for (int64_t k = Ph.row[(size_t)i]; k < Ph.row[(size_t)i + 1]; ++k) {
          const int c = Ph.col[(size_t)k];
          rc[(size_t)pos[(size_t)c]] = i;
          rv[(size_t)pos[(size_t)c]++] = Ph.val[(size_t)k];
        }
      X.rrow.upload(rr);
      X.rcol.upload(rc);
      X.rval.upload(rv);
    }
    tinv_.upload(H.terminal_inv);
    fine_lambda_ = H.fine_lambda;
    level_lambda_ = H.level_lambda;
    level_lambda_.resize(L_.size(), 0.0);

    part_.alloc((size_t)kMaxPartBlocks * 8);
    sc_.alloc(kScalars);
    flags_.alloc(1);
    ctl_.alloc(4);
    NDS_CUDA(cudaMallocHost((void**)&hsc_, sizeof(double) * kScalars));
    NDS_CUDA(cudaMallocHost((void**)&hflags_, sizeof(int) * 8));
    NDS_CUDA(cudaMemsetAsync(flags_.p, 0, sizeof(int), st_));

    if constexpr (!kSame) {
      mixed_ = o_.precision == NDS_MIXED;
      if (mixed_) alloc_mixed();
    }
    // setup-time state: fine CSR refreshed with the initial rAU
    tm.mark("levels_and_transfers");
    refresh_fine(rau_.p);
    if (mixed_ && o_.amg_half) {
      // FP16 copy: scale by a power of two that puts the largest setup-time
      // diagonal at 2^11 (the diagonal dominates its row; 2^4 headroom below
      // the FP16 maximum for later growth of rAU, values beyond saturate)
      std::vector<TA> d((size_t)nc_);
      NDS_CUDA(cudaMemcpyAsync(d.data(), fdiag_.p, sizeof(TA) * d.size(), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
      double dmax = 0.0;
      for (TA v : d) dmax = std::max(dmax, std::abs((double)v));
      if (!(dmax > 0.0) || !std::isfinite(dmax)) throw std::runtime_error("FP16 operator copy: no positive diagonal");
      hscale_ = std::ldexp(1.0, (int)std::floor(std::log2(2048.0 / dmax)));
      fvalH_.alloc(fval_.n);
      refresh_fine(rau_.p);
    }
    if (P_.power_its > 0) {
      fine_lambda_ = power_fine(P_.power_its, o_.amg_lambda_safety);
      for (size_t l = 0; l + 1 < L_.size(); ++l) level_lambda_[l] = power_level(L_[l], P_.power_its, o_.amg_lambda_safety);
    } else {
      fine_lambda_ = 1.0;
      for (auto& v : level_lambda_) v = 1.0;
    }
    if (o_.pressure_solver == NDS_P_CHEB) p_cheb_lambda_ = precond_power(o_.p_power_its, o_.p_power_safety);
    NDS_CUDA(cudaStreamSynchronize(st_));
    tm.mark("refresh_and_spectrum");
    reset();
  }

  // ------------------------------------------------------------------ helpers
  static constexpr int kMaxPartBlocks = 1184;  // 8 x 148 SMs
  static constexpr int kScalars = 128;
  enum { S_RHO = 0, S_PQ = 1, S_ALPHA = 2, S_RN2 = 3, S_RHON = 4, S_BETA = 5, S_R0 = 6, S_TARGET = 7, S_TMP = 8,
         S_TMP2 = 9, S_CONT2 = 10, S_WN = 11,
         S_AUDIT = 16, S_ST_T = 20, S_ST_V = 21,
         S_GUESS = 24,  // 44 slots: Galerkin matrix (upper triangle) and right-hand side of the guess
         S_COEF = 72 };  // 8 slots: guess coefficients

  // CUDA graphs of fixed launch sequences (no host decisions inside)
  struct Graph {
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels = 0;
    ~Graph() {
      if (exec) cudaGraphExecDestroy(exec);
    }
  };
  template <class F>
  void capture(Graph& g, F&& body) {
    const bool was = prof.on;
    prof.on = false;
    const unsigned long long l0 = g_launches;
    NDS_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    try {
      body();
    } catch (...) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(st_, &junk);
      if (junk) cudaGraphDestroy(junk);
      prof.on = was;
      throw;
    }
    cudaGraph_t graph = nullptr;
    NDS_CUDA(cudaStreamEndCapture(st_, &graph));
    const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    NDS_CUDA(e);
    g.kernels = g_launches - l0;
    g_launches = l0;
    prof.on = was;
  }
  void replay(Graph& g) {
    NDS_CUDA(cudaGraphLaunch(g.exec, st_));
    g_launches += g.kernels;
  }
  bool use_graphs_ = std::getenv("NDS_NO_GRAPHS") == nullptr;
  Graph g_amg_, g_pcg2_;
  // the whole PCG iteration loop as one graph: a conditional while node whose
  // body is one iteration and ends with pcg_check, which sets the condition
  struct LoopGraph {
    cudaGraphExec_t exec = nullptr;
    unsigned long long body_kernels = 0;
    bool failed = false;
    ~LoopGraph() {
      if (exec) cudaGraphExecDestroy(exec);
    }
  };
  LoopGraph g_loop_;
  bool build_pcg_loop() {
    const bool was = prof.on;
    prof.on = false;
    cudaGraph_t graph = nullptr;
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle h{};
    cudaGraphNodeParams cp{};
    cudaGraphNode_t node{};
    if (ok) ok = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
    }
    const unsigned long long l0 = g_launches;
    if (ok) ok = cudaStreamBeginCaptureToGraph(st_, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      bool body_ok = true;
      try {
        pcg_loop_body(h);
      } catch (...) {
        body_ok = false;
      }
      ok = cudaStreamEndCapture(st_, nullptr) == cudaSuccess && body_ok;
    }
    g_loop_.body_kernels = g_launches - l0;
    g_launches = l0;
    if (ok) ok = cudaGraphInstantiate(&g_loop_.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
      if (g_loop_.exec) cudaGraphExecDestroy(g_loop_.exec);
      g_loop_.exec = nullptr;
      g_loop_.failed = true;
      cudaGetLastError();  // the fallback path runs instead
    }
    prof.on = was;
    return ok;
  }
  // z = M b with b, z in the state precision (casts around the V-cycle in
  // the mixed mode)
  void amg_T(const T* b, T* z) {
    if constexpr (kSame) {
      amg_apply(b, z);
    } else if (o_.amg_smoother != NDS_SM_MCGS) {
      // the cast also takes the fine pre-smoother's diagonal step
      const PolyPlan pl = fine_plan();
      k::cast_jacobi<T, TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, b, rA_.p, TA(pl.w0), pl.den0,
                                                               poly_first(pl, zA_.p, fpong_.p));
      NDS_LAUNCH();
      amg_apply(rA_.p, zA_.p, true);
      k::cast_copy<TA, T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, zA_.p, z);
      NDS_LAUNCH();
    } else {
      k::cast_copy<T, TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, b, rA_.p);
      NDS_LAUNCH();
      amg_apply(rA_.p, zA_.p);
      k::cast_copy<TA, T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, zA_.p, z);
      NDS_LAUNCH();
    }
  }
  // z = M r on the solver's fixed PCG buffers, replayed from a graph
  void amg_rz() {
    if (!use_graphs_) return amg_T(r_.p, z_.p);
    if (!g_amg_.exec) capture(g_amg_, [&] { amg_T(r_.p, z_.p); });
    replay(g_amg_);
  }

  int red_grid(long long n, int per = kBlock) const { return std::min(grid_for(n, per), kMaxPartBlocks); }
  template <int NV>
  void reduce_to(int nblocks, int slot) {
    k::reduce_partials<NV><<<1, kBlock, 0, st_>>>(part_.p, nblocks, sc_.p + slot);
    NDS_LAUNCH();
  }
  // reduction of one value into sc[slot], then the PCG scalar step STEP
  template <int STEP>
  void reduce_pcg(int nblocks, int slot, int max_its = 0, cudaGraphConditionalHandle h = {}, int in_graph = 1) {
    const k::PcgScalars ps{sc_.p, flags_.p, ctl_.p, S_RN2, S_R0, S_TARGET, max_its, h, in_graph};
    k::reduce_pcg<STEP><<<1, kBlock, 0, st_>>>(part_.p, nblocks, sc_.p + slot, ps);
    NDS_LAUNCH();
  }
  void fetch(int first, int count) {
    NDS_CUDA(cudaMemcpyAsync(hsc_ + first, sc_.p + first, sizeof(double) * count, cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaStreamSynchronize(st_));
  }
  template <class V>
  double dot_fetch(const V* x, const V* y, int n, int slot) {
    const int g = red_grid(n);
    k::dot<V><<<g, kBlock, 0, st_>>>(n, x, y, part_.p);
    NDS_LAUNCH();
    reduce_to<1>(g, slot);
    fetch(slot, 1);
    return hsc_[slot];
  }
  template <class V>
  void dot_dev(const V* x, const V* y, int n, int slot) {
    const int g = red_grid(n);
    k::dot<V><<<g, kBlock, 0, st_>>>(n, x, y, part_.p);
    NDS_LAUNCH();
    reduce_to<1>(g, slot);
  }

  // operator view: the fine Schur matrix in SELL-32, AMG levels in CSR
  template <class V>
  struct OpView {
    int n;
    bool sell;
    k::Sell s;
    const int32_t* rp;
    const int32_t* ci;
    const V* v;
    int cat;                     // profiler category
    const __half* vh = nullptr;  // FP16 copy of the values, scaled by 1 / vinv
    double vinv = 1.0;
    const int16_t* ch = nullptr;  // CSR levels with vh: columns as deltas to the row
  };
  template <int MODE, class V>
  void sell_launch(const OpView<V>& A, int grid, const V* x, const V* b, const V* den, double w, V* y, V* y2) {
    if constexpr (std::is_same<V, float>::value) {
      if (A.vh) {
        if (A.s.dcol)
          k::sell_spmv<V, MODE, true, __half><<<grid, kBlock, 0, st_>>>(A.s, A.vh, x, b, den, V(w), y, y2, part_.p,
                                                                          V(A.vinv));
        else
          k::sell_spmv<V, MODE, false, __half><<<grid, kBlock, 0, st_>>>(A.s, A.vh, x, b, den, V(w), y, y2, part_.p,
                                                                           V(A.vinv));
        return;
      }
    }
    if (A.s.dcol)
      k::sell_spmv<V, MODE, true><<<grid, kBlock, 0, st_>>>(A.s, A.v, x, b, den, V(w), y, y2, part_.p);
    else
      k::sell_spmv<V, MODE, false><<<grid, kBlock, 0, st_>>>(A.s, A.v, x, b, den, V(w), y, y2, part_.p);
  }
  // physical operator (precision T) and the AMG's fine operator (precision TA)
  OpView<T> fine_op() const { return {nc_, true, sell_, nullptr, nullptr, fval_.p, P_FINE_SPMV}; }
  OpView<TA> fine_opA() const {
    if constexpr (kSame) return {nc_, true, sell_, nullptr, nullptr, fval_.p, P_FINE_AMG};
    else return {nc_, true, sell_, nullptr, nullptr, fvalA_.p, P_FINE_AMG};
  }
  // the fine operator of the V-cycle: the FP16 copy when amg_half is on
  OpView<TA> fine_opV() const {
    OpView<TA> A = fine_opA();
    if (fvalH_.p) {
      A.vh = fvalH_.p;
      A.vinv = 1.0 / hscale_;
      A.cat = P_FINE_HALF;
    }
    return A;
  }
  OpView<TA> level_op(const Level& A) const {
    OpView<TA> V{A.n, false, k::Sell{}, A.row.p, A.col.p, A.val.p, P_COARSE_SPMV};
    if (A.hval.p) {
      V.vh = A.hval.p;
      V.vinv = A.hinv;
      V.ch = A.hcol.p;
    }
    return V;
  }
  // FP16 copy of an explicit level's CSR values (a setup snapshot), scaled by
  // the power of two that puts its largest diagonal at 2^11
  void level_to_half(Level& Lv, const CsrHost& A) {
    double dmax = 0.0;
    for (double d : A.diag) dmax = std::max(dmax, std::abs(d));
    if (!(dmax > 0.0) || !std::isfinite(dmax)) throw std::runtime_error("FP16 level copy: no positive diagonal");
    const double scale = std::ldexp(1.0, (int)std::floor(std::log2(2048.0 / dmax)));
    std::vector<__half> hv(A.val.size());
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < hv.size(); ++k)
      hv[k] = __float2half((float)std::min(std::max(A.val[k] * scale, -65504.0), 65504.0));
    Lv.hval.alloc(hv.size());
    NDS_CUDA(cudaMemcpy(Lv.hval.p, hv.data(), hv.size() * sizeof(__half), cudaMemcpyHostToDevice));
    Lv.hinv = 1.0 / scale;
    std::vector<int16_t> dc(A.col.size());
    int too_far = 0;
#pragma omp parallel for schedule(static) reduction(| : too_far)
    for (int i = 0; i < A.n; ++i)
      for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
        const int d = A.col[(size_t)k] - i;
        if (d < -32767 || d > 32767) too_far = 1;
        else dc[(size_t)k] = (int16_t)d;
      }
    const bool fits = too_far == 0;
    if (fits && !std::getenv("NDS_SELL_COL32")) Lv.hcol.upload(dc);
  }
  // launch f with the lanes per row of the FP16 level kernels
  template <class V, class F>
  void level_half_launch(const OpView<V>& A, F&& f) {
    if (level_lanes_ == 8) f(std::integral_constant<int, 8>{});
    else if (level_lanes_ == 16) f(std::integral_constant<int, 16>{});
    else f(std::integral_constant<int, 32>{});
  }
  template <class V>
  void op_spmv(const OpView<V>& A, const V* x, V* y) {
    ProfScope ps(prof, st_, A.cat);
    if (A.sell) sell_launch<k::SELL_Y, V>(A, grid_for(A.n), x, nullptr, nullptr, 0.0, y, nullptr);
    else if (A.vh && A.ch && std::is_same<V, float>::value)
      level_half_launch(A, [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::spmv<V, __half, int16_t, GL><<<grid_for((long long)A.n * GL), kBlock, 0, st_>>>(A.n, A.rp, A.ch, A.vh, x,
                                                                                             y, V(A.vinv));
      });
    else if (A.vh && std::is_same<V, float>::value)
      level_half_launch(A, [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::spmv<V, __half, int32_t, GL><<<grid_for((long long)A.n * GL), kBlock, 0, st_>>>(A.n, A.rp, A.ci, A.vh, x,
                                                                                             y, V(A.vinv));
      });
    else k::spmv<V><<<grid_for((long long)A.n * k::kRowLanes), kBlock, 0, st_>>>(A.n, A.rp, A.ci, A.v, x, y);
    NDS_LAUNCH();
  }
  // r = b - A x; r2 = r, or (den given) the first Jacobi step w r / den
  template <class V>
  void op_resid(const OpView<V>& A, const V* x, const V* b, V* r, V* r2 = nullptr, const V* den = nullptr,
                double w = 0.0) {
    ProfScope ps(prof, st_, A.cat);
    if (A.sell) sell_launch<k::SELL_RESID, V>(A, grid_for(A.n), x, b, den, w, r, r2);
    else if (A.vh && A.ch && std::is_same<V, float>::value)
      level_half_launch(A, [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::spmv_resid<V, __half, int16_t, GL><<<grid_for((long long)A.n * GL), kBlock, 0, st_>>>(
            A.n, A.rp, A.ch, A.vh, x, b, r, r2, den, V(w), V(A.vinv));
      });
    else if (A.vh && std::is_same<V, float>::value)
      level_half_launch(A, [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::spmv_resid<V, __half, int32_t, GL><<<grid_for((long long)A.n * GL), kBlock, 0, st_>>>(
            A.n, A.rp, A.ci, A.vh, x, b, r, r2, den, V(w), V(A.vinv));
      });
    else
      k::spmv_resid<V><<<grid_for((long long)A.n * k::kRowLanes), kBlock, 0, st_>>>(A.n, A.rp, A.ci, A.v, x, b, r, r2, den, V(w));
    NDS_LAUNCH();
  }
  // xout = xin + w (b - A xin) / den, or (add_to given) add_to += that
  template <class V>
  void op_smooth(const OpView<V>& A, const V* xin, const V* b, const V* den, double w, V* xout, V* add_to = nullptr) {
    ProfScope ps(prof, st_, A.cat);
    if (A.sell) sell_launch<k::SELL_SMOOTH, V>(A, grid_for(A.n), xin, b, den, w, xout, add_to);
    else if (A.vh && A.ch && std::is_same<V, float>::value)
      level_half_launch(A, [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::spmv_smooth<V, __half, int16_t, GL><<<grid_for((long long)A.n * GL), kBlock, 0, st_>>>(
            A.n, A.rp, A.ch, A.vh, xin, b, den, V(w), xout, add_to, V(A.vinv));
      });
    else if (A.vh && std::is_same<V, float>::value)
      level_half_launch(A, [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::spmv_smooth<V, __half, int32_t, GL><<<grid_for((long long)A.n * GL), kBlock, 0, st_>>>(
            A.n, A.rp, A.ci, A.vh, xin, b, den, V(w), xout, add_to, V(A.vinv));
      });
    else
      k::spmv_smooth<V><<<grid_for((long long)A.n * k::kRowLanes), kBlock, 0, st_>>>(A.n, A.rp, A.ci, A.v, xin, b, den, V(w), xout,
                                                                          add_to);
    NDS_LAUNCH();
  }
  template <class V>
  void vcopy(int n, const V* a, V* b) {
    k::copy<V><<<grid_for(n), kBlock, 0, st_>>>(n, a, b);
    NDS_LAUNCH();
  }
  template <class V>
  void vaxpy(int n, double a, const V* x, V* y) {
    k::axpy<V><<<grid_for(n), kBlock, 0, st_>>>(n, V(a), x, y);
    NDS_LAUNCH();
  }

  // fine Schur operator
  void refresh_fine(const T* rau, cudaStream_t s = nullptr) {
    if (!s) s = st_;
    ProfScope ps(prof, s, P_REFRESH);
    k::sell_refresh<T, TA><<<(nc_ + 31) / 32, k::kRefreshBlock, refresh_smem_, s>>>(
        nc_, fcoff_.p, fcs_.p, fgeo_.p, ref_.p, rau, fdslot_.p, sbase_.p, swidth_.p, fval_.p,
        kSame ? nullptr : fvalA_.p, fdiag_.p, fl1_.p, fvalH_.p, (float)hscale_);
    NDS_LAUNCH();
  }
  void fine_apply(const T* x, T* y) { op_spmv(fine_op(), x, y); }

  // ------------------------------------------------------------- smoothers
  // x = S(b) from a zero initial guess.  Jacobi-type steps write to a second
  // buffer (xin is read by every row), then the result is copied back.
  // Polynomial (Chebyshev or damped-Jacobi) smoother from a zero guess:
  // x = S(b).  One diagonal step, then m Jacobi-type steps ping-ponging
  // between two buffers; the first buffer is chosen by the parity of m so
  // that the last step writes x (no copy-back).
  struct PolyPlan {
    int m;            // Jacobi-type steps after the diagonal one
    double w0;        // weight of the diagonal step
    const TA* den0;   // its denominator
  };
  PolyPlan poly_plan(double lambda, bool cheb, const TA* diag, const TA* den_jac, int sweeps) const {
    if (cheb) {
      const int deg = o_.amg_cheb_degree;
      const double lo = o_.amg_lambda_low_fraction * lambda;
      if (!(lambda > lo && lo > 0)) throw SolveFailure(NDS_E_BREAKDOWN, "Chebyshev smoother interval invalid");
      return {deg - 1, 1.0 / cheb_root(lambda, lo, 0, deg), diag};
    }
    return {sweeps - 1, o_.amg_jacobi_omega, den_jac};
  }
  static TA* poly_first(const PolyPlan& pl, TA* x, TA* pong) { return (pl.m % 2 == 0) ? x : pong; }
  // first_done: the diagonal step is already in poly_first(x, pong) (written
  // by the residual kernel); add_to: the result is added to add_to instead
  // of stored in x.
  void poly_smooth(const OpView<TA>& A, const TA* diag, const TA* b, TA* x, TA* pong, double lambda, bool cheb,
                   const TA* den_jac, int sweeps, bool first_done = false, TA* add_to = nullptr) {
    const int n = A.n;
    const PolyPlan pl = poly_plan(lambda, cheb, diag, den_jac, sweeps);
    TA* cur = poly_first(pl, x, pong);
    TA* nxt = (pl.m % 2 == 0) ? pong : x;
    if (!first_done) {
      k::jacobi_zero<TA><<<grid_for(n), kBlock, 0, st_>>>(n, TA(pl.w0), b, pl.den0, cur);
      NDS_LAUNCH();
    }
    const double lo = cheb ? o_.amg_lambda_low_fraction * lambda : 0.0;
    for (int kk = 1; kk <= pl.m; ++kk) {
      const double w = cheb ? 1.0 / cheb_root(lambda, lo, kk, o_.amg_cheb_degree) : o_.amg_jacobi_omega;
      op_smooth(A, cur, b, cheb ? diag : den_jac, w, nxt, kk == pl.m ? add_to : nullptr);
      std::swap(cur, nxt);
    }
    if (pl.m == 0 && add_to) vaxpy(n, 1.0, (const TA*)x, add_to);
  }
  void mcgs(const OpView<TA>& A, const TA* diag, const TA* b, TA* x, const DBuf<int32_t>& crows,
            const std::vector<int>& coff, int sweeps) {
    const int n = A.n;
    NDS_CUDA(cudaMemsetAsync(x, 0, sizeof(TA) * (size_t)n, st_));
    const int ncol = (int)coff.size() - 1;
    auto pass = [&](bool reverse) {
      for (int qq = 0; qq < ncol; ++qq) {
        const int c = reverse ? ncol - 1 - qq : qq;
        const int cnt = coff[(size_t)c + 1] - coff[(size_t)c];
        if (cnt <= 0) continue;
        if (A.sell && A.s.dcol)
          k::sell_gs_color<TA, true><<<grid_for(cnt), kBlock, 0, st_>>>(cnt, crows.p + coff[(size_t)c], A.s, A.v, diag, b,
                                                                     x, TA(o_.amg_mcgs_omega));
        else if (A.sell)
          k::sell_gs_color<TA, false><<<grid_for(cnt), kBlock, 0, st_>>>(cnt, crows.p + coff[(size_t)c], A.s, A.v, diag,
                                                                      b, x, TA(o_.amg_mcgs_omega));
        else
          k::amg_gs_color<TA><<<grid_for((long long)cnt * 32), kBlock, 0, st_>>>(cnt, crows.p + coff[(size_t)c], A.rp, A.ci,
                                                                                A.v, diag, b, x, TA(o_.amg_mcgs_omega));
        NDS_LAUNCH();
      }
    };
    for (int s = 0; s < sweeps; ++s) {
      if (o_.amg_mcgs_order == NDS_MCGS_FORWARD) pass(false);
      else if (o_.amg_mcgs_order == NDS_MCGS_BACKWARD) pass(true);
      else { pass(false); pass(true); }
    }
  }
  // first_done: the diagonal step of the polynomial smoother is already in
  // place (taken by the kernel that produced b); never set for MCGS
  void smooth_fine(const TA* b, TA* x, bool first_done = false) {
    const int sm = o_.amg_smoother;
    if (sm == NDS_SM_MCGS) {
      mcgs(fine_opV(), fdiag_.p, b, x, fine_crows_, fine_coff_, o_.amg_mcgs_fine_sweeps);
      return;
    }
    const TA* den = sm == NDS_SM_L1JACOBI ? fl1_.p : fdiag_.p;
    poly_smooth(fine_opV(), fdiag_.p, b, x, fpong_.p, fine_lambda_, sm == NDS_SM_CHEB2, den, o_.amg_jacobi_fine_sweeps,
                first_done);
  }
  void smooth_level(Level& A, const TA* b, TA* x, double lambda, bool first_done = false) {
    const int sm = o_.amg_smoother;
    if (sm == NDS_SM_MCGS) {
      mcgs(level_op(A), A.diag.p, b, x, A.crows, A.coff, o_.amg_mcgs_coarse_sweeps);
      return;
    }
    const TA* den = sm == NDS_SM_L1JACOBI ? A.l1.p : A.diag.p;
    poly_smooth(level_op(A), A.diag.p, b, x, A.pong.p, lambda, sm == NDS_SM_CHEB2, den, o_.amg_jacobi_coarse_sweeps,
                first_done);
  }
  // plan of the pre-smoother of level l (polynomial smoothers only)
  PolyPlan level_plan(int l) const {
    const Level& A = L_[(size_t)l];
    const int sm = o_.amg_smoother;
    const TA* den = sm == NDS_SM_L1JACOBI ? A.l1.p : A.diag.p;
    return poly_plan(level_lambda_[(size_t)l], sm == NDS_SM_CHEB2, A.diag.p, den, o_.amg_jacobi_coarse_sweeps);
  }
  PolyPlan fine_plan() const {
    const int sm = o_.amg_smoother;
    const TA* den = sm == NDS_SM_L1JACOBI ? fl1_.p : fdiag_.p;
    return poly_plan(fine_lambda_, sm == NDS_SM_CHEB2, fdiag_.p, den, o_.amg_jacobi_fine_sweeps);
  }
  // whether the pre-smoother of level l can take its diagonal step in the
  // restriction that feeds it (a polynomial smoother, not the terminal level)
  bool fuse_pre(int l) const { return o_.amg_smoother != NDS_SM_MCGS && l < (int)L_.size() - 1; }
  // lanes per coarse row of the restriction (the FP16 levels' count on the
  // mixed FP16 path, a warp otherwise)
  int restrict_lanes() const { return mixed_ && o_.amg_half ? level_lanes_ : 32; }
  // c = R f; with level >= 0 also the diagonal step of that level's
  // pre-smoother (see fuse_pre)
  void restrict_to(const Xfer& X, const TA* f, TA* c, int level = -1) {
    ProfScope ps(prof, st_, P_TRANSFER);
    const TA* den0 = nullptr;
    TA* x1 = nullptr;
    double w0 = 0.0;
    if (level >= 0) {
      Level& C = L_[(size_t)level];
      const PolyPlan pl = level_plan(level);
      den0 = pl.den0;
      w0 = pl.w0;
      x1 = poly_first(pl, C.x.p, C.pong.p);
    }
    if (restrict_lanes() != 32) {
      auto run = [&](auto gl) {
        constexpr int GL = decltype(gl)::value;
        k::restrict_rows<TA, GL><<<grid_for((long long)X.nc * GL), kBlock, 0, st_>>>(X.nc, X.rrow.p, X.rcol.p,
                                                                                    X.rval.p, f, c, den0, TA(w0), x1);
      };
      if (restrict_lanes() == 8) run(std::integral_constant<int, 8>{});
      else run(std::integral_constant<int, 16>{});
    } else {
      k::restrict_rows<TA><<<grid_for((long long)X.nc * k::kRowLanes), kBlock, 0, st_>>>(
          X.nc, X.rrow.p, X.rcol.p, X.rval.p, f, c, den0, TA(w0), x1);
    }
    NDS_LAUNCH();
  }
  void prolong(const Xfer& X, const TA* c, TA* f) {
    ProfScope ps(prof, st_, P_TRANSFER);
    k::prolong_add<TA><<<grid_for(X.nf), kBlock, 0, st_>>>(X.nf, X.pw, X.pcol.p, X.pval.p, c, f);
    NDS_LAUNCH();
  }

  // -------------------------------------------------------------- V-cycle
  // pre_done: the diagonal step of this level's pre-smoother is already in
  // place (taken by the restriction that produced b)
  void vcycle(int l, const TA* b, TA* x, bool pre_done = false) {
    Level& A = L_[(size_t)l];
    if (l == (int)L_.size() - 1) {
      ProfScope ps(prof, st_, P_TERMINAL);
      k::dense_mv<TA><<<grid_for((long long)A.n * 32), kBlock, 0, st_>>>(A.n, tinv_.p, b, x);
      NDS_LAUNCH();
      return;
    }
    smooth_level(A, b, x, level_lambda_[(size_t)l], pre_done);
    op_resid(level_op(A), x, b, A.r.p);
    Level& C = L_[(size_t)l + 1];
    const bool fuse = fuse_pre(l + 1);
    restrict_to(X_[(size_t)l + 1], A.r.p, C.b.p, fuse ? l + 1 : -1);
    vcycle(l + 1, C.b.p, C.x.p, fuse);
    prolong(X_[(size_t)l + 1], C.x.p, x);
    // r = b - A x into b (b is no longer needed), then the post-smoother
    // solves A corr = r and x += corr
    const double lam = level_lambda_[(size_t)l];
    const int sm = o_.amg_smoother;
    if (sm == NDS_SM_MCGS) {
      op_resid(level_op(A), x, b, A.r.p, A.b.p);
      smooth_level(A, A.b.p, A.corr.p, lam);
      vaxpy(A.n, 1.0, A.corr.p, x);
      return;
    }
    // the residual kernel also takes the smoother's diagonal step, and the
    // last smoothing step adds the correction to x
    const bool cheb = sm == NDS_SM_CHEB2;
    const TA* den = sm == NDS_SM_L1JACOBI ? A.l1.p : A.diag.p;
    const PolyPlan pl = poly_plan(lam, cheb, A.diag.p, den, o_.amg_jacobi_coarse_sweeps);
    op_resid(level_op(A), x, b, A.b.p, poly_first(pl, A.corr.p, A.pong.p), pl.den0, pl.w0);
    poly_smooth(level_op(A), A.diag.p, A.b.p, A.corr.p, A.pong.p, lam, cheb, den, o_.amg_jacobi_coarse_sweeps, true, x);
  }
  // pre_done: the fine pre-smoother's diagonal step is already in place
  void amg_apply(const TA* b, TA* z, bool pre_done = false) {
    smooth_fine(b, z, pre_done);
    op_resid(fine_opV(), z, b, fr_.p);
    Level& C = L_[0];
    const bool fuse = fuse_pre(0);
    restrict_to(X_[0], fr_.p, C.b.p, fuse ? 0 : -1);
    vcycle(0, C.b.p, C.x.p, fuse);
    prolong(X_[0], C.x.p, z);
    const int sm = o_.amg_smoother;
    if (sm == NDS_SM_MCGS) {
      op_resid(fine_opV(), z, b, fr_.p, frhs_.p);
      smooth_fine(frhs_.p, fcorr_.p);
      vaxpy(nc_, 1.0, fcorr_.p, z);
      return;
    }
    // post-smoothing as on the levels: residual with the diagonal step, last
    // step added to z
    const bool cheb = sm == NDS_SM_CHEB2;
    const TA* den = sm == NDS_SM_L1JACOBI ? fl1_.p : fdiag_.p;
    const PolyPlan pl = poly_plan(fine_lambda_, cheb, fdiag_.p, den, o_.amg_jacobi_fine_sweeps);
    op_resid(fine_opV(), z, b, frhs_.p, poly_first(pl, fcorr_.p, fpong_.p), pl.den0, pl.w0);
    poly_smooth(fine_opV(), fdiag_.p, frhs_.p, fcorr_.p, fpong_.p, fine_lambda_, cheb, den, o_.amg_jacobi_fine_sweeps,
                true, z);
  }

  // ------------------------------------------------------ spectrum estimates
  double power_fine(int its, double safety) {
    TA* v = fcorr_.p;
    TA* u = frhs_.p;
    TA* au = ftmp_.p;
    TA* w = fr_.p;
    k::power_init<TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, v);
    NDS_LAUNCH();
    const double vn = std::sqrt(dot_fetch((const TA*)v, (const TA*)v, nc_, S_TMP));
    k::scale<TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, TA(1.0 / vn), v);
    NDS_LAUNCH();
    double ray = 0.0;
    for (int it = 0; it < its; ++it) {
      k::div_sqrt<TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, v, fdiag_.p, u);
      op_spmv(fine_opV(), (const TA*)u, au);
      k::div_sqrt<TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, au, fdiag_.p, w);
      NDS_LAUNCH();
      const double num = dot_fetch((const TA*)v, (const TA*)w, nc_, S_TMP),
                   den = dot_fetch((const TA*)v, (const TA*)v, nc_, S_TMP2);
      ray = num / std::max(den, 1e-300);
      const double wn = std::sqrt(dot_fetch((const TA*)w, (const TA*)w, nc_, S_TMP));
      if (!(ray > 0.0) || !(wn > 0.0) || !std::isfinite(ray) || !std::isfinite(wn))
        throw SolveFailure(NDS_E_BREAKDOWN, "fine GPU power iteration failed");
      vcopy(nc_, (const TA*)w, v);
      k::scale<TA><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, TA(1.0 / wn), v);
      NDS_LAUNCH();
    }
    return safety * ray;
  }
  double power_level(Level& A, int its, double safety) {
    const int n = A.n;
    k::power_init<TA><<<grid_for(n), kBlock, 0, st_>>>(n, A.corr.p);
    NDS_LAUNCH();
    const double vn = std::sqrt(dot_fetch((const TA*)A.corr.p, (const TA*)A.corr.p, n, S_TMP));
    k::scale<TA><<<grid_for(n), kBlock, 0, st_>>>(n, TA(1.0 / vn), A.corr.p);
    NDS_LAUNCH();
    double ray = 0.0;
    for (int it = 0; it < its; ++it) {
      k::div_sqrt<TA><<<grid_for(n), kBlock, 0, st_>>>(n, A.corr.p, A.diag.p, A.b.p);
      op_spmv(level_op(A), (const TA*)A.b.p, A.tmp.p);
      k::div_sqrt<TA><<<grid_for(n), kBlock, 0, st_>>>(n, A.tmp.p, A.diag.p, A.r.p);
      NDS_LAUNCH();
      const double num = dot_fetch((const TA*)A.corr.p, (const TA*)A.r.p, n, S_TMP),
                   den = dot_fetch((const TA*)A.corr.p, (const TA*)A.corr.p, n, S_TMP2);
      ray = num / std::max(den, 1e-300);
      const double wn = std::sqrt(dot_fetch((const TA*)A.r.p, (const TA*)A.r.p, n, S_TMP));
      if (!(ray > 0.0) || !(wn > 0.0) || !std::isfinite(ray) || !std::isfinite(wn))
        throw SolveFailure(NDS_E_BREAKDOWN, "coarse GPU power iteration failed");
      vcopy(n, (const TA*)A.r.p, A.corr.p);
      k::scale<TA><<<grid_for(n), kBlock, 0, st_>>>(n, TA(1.0 / wn), A.corr.p);
      NDS_LAUNCH();
    }
    return safety * ray;
  }
  // lambda_max(M^-1 A) for the outer Chebyshev solver
  double precond_power(int its, double safety) {
    k::power_init<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, pp_.p);
    NDS_LAUNCH();
    const double vn = std::sqrt(dot_fetch(pp_.p, pp_.p, nc_, S_TMP));
    k::scale<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, T(1.0 / vn), pp_.p);
    NDS_LAUNCH();
    double est = 0.0;
    for (int kk = 0; kk < its; ++kk) {
      fine_apply(pp_.p, q_.p);
      amg_T(q_.p, z_.p);
      const double zn = std::sqrt(dot_fetch(z_.p, z_.p, nc_, S_TMP));
      const double ray = dot_fetch(pp_.p, z_.p, nc_, S_TMP2);
      if (!(zn > 0.0) || !std::isfinite(zn) || !std::isfinite(ray)) throw SolveFailure(NDS_E_BREAKDOWN, "preconditioned power failed");
      est = std::max(est, std::max(std::abs(ray), zn));
      vcopy(nc_, z_.p, pp_.p);
      k::scale<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, T(1.0 / zn), pp_.p);
      NDS_LAUNCH();
    }
    const double hi = safety * est;
    if (!(hi > 0.0) || !std::isfinite(hi)) throw SolveFailure(NDS_E_BREAKDOWN, "preconditioned lambda invalid");
    return hi;
  }

  // ------------------------------------------------------ pressure solvers
  struct PRes {
    int its = 0;
    double rel = 1;
    bool ok = false;
  };
  void check_flags() {
    int f = 0;
    NDS_CUDA(cudaMemcpyAsync(&f, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaStreamSynchronize(st_));
    if (f & 1) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG pAp nonpositive");
    if (f & 2) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG rho nonpositive");
  }
  // ||r0|| and the zero solution
  double p_start(const T* rhs) {
    x_.zero(st_);
    vcopy(nc_, rhs, r_.p);
    const double r0 = std::sqrt(dot_fetch(r_.p, r_.p, nc_, S_TMP));
    if (!std::isfinite(r0)) throw SolveFailure(NDS_E_BREAKDOWN, "pressure initial norm nonfinite");
    return r0;
  }
  // one PCG iteration, first half: q = A p, pq = p.q, alpha = rho/pq,
  // x += alpha p, r -= alpha q, rn2 = r.r; then rn2 and the flags to the host
  void pcg_half1() {
    const int g = red_grid(nc_);
    {
      ProfScope ps(prof, st_, P_FINE_SPMV);
      sell_launch<k::SELL_DOT, T>(fine_op(), g, pp_.p, nullptr, nullptr, 0.0, q_.p, nullptr);
      NDS_LAUNCH();
    }
    reduce_to<1>(g, S_PQ);
    k::pcg_alpha<<<1, 1, 0, st_>>>(sc_.p, flags_.p);
    NDS_LAUNCH();
    k::xr_update<T><<<g, kBlock, 0, st_>>>(nc_, 0.0, sc_.p + S_ALPHA, pp_.p, q_.p, x_.p, r_.p, part_.p);
    NDS_LAUNCH();
    reduce_to<1>(g, S_RN2);
    NDS_CUDA(cudaMemcpyAsync(hsc_ + S_RN2, sc_.p + S_RN2, sizeof(double), cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaMemcpyAsync(hflags_, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
  }
  // second half: z = M r, rho_new = r.z, beta = rho_new/rho, p = z + beta p
  void pcg_half2() {
    amg_T(r_.p, z_.p);
    dot_dev(r_.p, z_.p, nc_, S_RHON);
    k::pcg_beta<<<1, 1, 0, st_>>>(sc_.p, flags_.p);
    NDS_LAUNCH();
    k::p_update<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, sc_.p + S_BETA, z_.p, pp_.p);
    NDS_LAUNCH();
  }
  // one pass of the device loop: z = M r; rho (first pass: p = z); q = A p;
  // alpha; x, r update; ||r||^2; check
  void pcg_loop_body(cudaGraphConditionalHandle h) {
    amg_T(r_.p, z_.p);
    const int g = red_grid(nc_);
    k::dot<T><<<g, kBlock, 0, st_>>>(nc_, r_.p, z_.p, part_.p);
    NDS_LAUNCH();
    reduce_pcg<k::PCG_RHO>(g, S_RHON);
    k::p_update_dev<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, sc_.p + S_BETA, ctl_.p, z_.p, pp_.p);
    NDS_LAUNCH();
    sell_launch<k::SELL_DOT, T>(fine_op(), g, pp_.p, nullptr, nullptr, 0.0, q_.p, nullptr);
    NDS_LAUNCH();
    reduce_pcg<k::PCG_ALPHA>(g, S_PQ);
    k::xr_update<T><<<g, kBlock, 0, st_>>>(nc_, 0.0, sc_.p + S_ALPHA, pp_.p, q_.p, x_.p, r_.p, part_.p);
    NDS_LAUNCH();
    reduce_pcg<k::PCG_CHECK>(g, S_RN2, o_.p_max, h);
  }
  // PCG with the iteration loop on the device: two host synchronisations per
  // solve (initial norm, final state) instead of one per iteration.  Same
  // arithmetic and stopping rule as pcg_host.
  PRes pcg_device(double r0) {
    const double target = std::max(o_.p_atol, o_.p_rtol * r0);
    hsc_[S_R0] = r0;
    hsc_[S_TARGET] = target;
    NDS_CUDA(cudaMemcpyAsync(sc_.p + S_R0, hsc_ + S_R0, 2 * sizeof(double), cudaMemcpyHostToDevice, st_));
    const int init[4] = {0, 0, 1, o_.p_max};
    std::memcpy(hflags_ + 4, init, sizeof(init));
    NDS_CUDA(cudaMemcpyAsync(ctl_.p, hflags_ + 4, 4 * sizeof(int), cudaMemcpyHostToDevice, st_));
    NDS_CUDA(cudaMemsetAsync(flags_.p, 0, sizeof(int), st_));
    NDS_CUDA(cudaGraphLaunch(g_loop_.exec, st_));
    NDS_CUDA(cudaMemcpyAsync(hflags_ + 4, ctl_.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaMemcpyAsync(hflags_, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaMemcpyAsync(hsc_ + S_RN2, sc_.p + S_RN2, sizeof(double), cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaStreamSynchronize(st_));
    const int its = hflags_[4], f = hflags_[0];
    g_launches += (unsigned long long)its * g_loop_.body_kernels;
    if (f & 8) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG initial rho nonpositive");
    if (f & 1) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG pAp nonpositive");
    if (f & 2) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG rho nonpositive");
    PRes R;
    R.its = its;
    R.rel = std::sqrt(hsc_[S_RN2]) / std::max(r0, 1e-300);
    if ((f & 4) || !std::isfinite(R.rel)) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG residual nonfinite");
    R.ok = hflags_[5] != 0;
    return R;
  }
  PRes pcg(const T* rhs) {
    const double r0 = p_start(rhs);
    start_readback();
    if (r0 <= o_.p_atol) return {0, 0.0, true};
    // device loop unless the category profiler needs per-kernel events (or
    // graphs are off / the conditional graph could not be built)
    if (use_graphs_ && !prof.on && !g_loop_.failed && o_.p_max >= 1) {
      if (g_loop_.exec || build_pcg_loop()) return pcg_device(r0);
    }
    return pcg_host(r0);
  }
  PRes pcg_host(double r0) {
    amg_rz();
    vcopy(nc_, z_.p, pp_.p);
    dot_dev(r_.p, z_.p, nc_, S_RHO);
    fetch(S_RHO, 1);
    if (!(hsc_[S_RHO] > 0) || !std::isfinite(hsc_[S_RHO])) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG initial rho nonpositive");
    NDS_CUDA(cudaMemsetAsync(flags_.p, 0, sizeof(int), st_));
    const double target = std::max(o_.p_atol, o_.p_rtol * r0);
    // the first half stays a direct launch sequence, so the fine SpMV of the
    // Krylov step is timed live by the profiler; the AMG half is a graph
    if (use_graphs_ && !g_pcg2_.exec) capture(g_pcg2_, [&] { pcg_half2(); });
    PRes R;
    for (int kk = 0; kk < o_.p_max; ++kk) {
      pcg_half1();
      NDS_CUDA(cudaStreamSynchronize(st_));
      if (*hflags_ & 1) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG pAp nonpositive");
      if (*hflags_ & 2) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG rho nonpositive");
      const double rn = std::sqrt(hsc_[S_RN2]);
      R.its = kk + 1;
      R.rel = rn / std::max(r0, 1e-300);
      if (!std::isfinite(R.rel)) throw SolveFailure(NDS_E_BREAKDOWN, "pressure PCG residual nonfinite");
      if (rn <= target) {
        R.ok = true;
        break;
      }
      if (use_graphs_) replay(g_pcg2_);
      else pcg_half2();
    }
    check_flags();
    return R;
  }
  // Richardson (omega fixed) and outer Chebyshev (omega = 1/root_k)
  PRes stationary(const T* rhs, bool cheb) {
    const double r0 = p_start(rhs);
    start_readback();
    if (r0 <= o_.p_atol) return {0, 0.0, true};
    const double target = std::max(o_.p_atol, o_.p_rtol * r0);
    double centre = 0, radius = 0;
    if (cheb) {
      const double lo = o_.p_cheb_low_fraction * p_cheb_lambda_;
      centre = .5 * (p_cheb_lambda_ + lo);
      radius = .5 * (p_cheb_lambda_ - lo);
    }
    const double pi = 3.141592653589793238462643383279502884;
    PRes R;
    for (int kk = 0; kk < o_.p_max; ++kk) {
      double omega = o_.p_richardson_omega;
      if (cheb) {
        const int ri = kk % o_.p_cheb_degree;
        omega = 1.0 / (centre - radius * std::cos(pi * (2.0 * (double)ri + 1.0) / (2.0 * (double)o_.p_cheb_degree)));
      }
      amg_rz();
      fine_apply(z_.p, q_.p);
      const int g = red_grid(nc_);
      k::xr_update<T><<<g, kBlock, 0, st_>>>(nc_, omega, nullptr, z_.p, q_.p, x_.p, r_.p, part_.p);
      NDS_LAUNCH();
      reduce_to<1>(g, S_RN2);
      fetch(S_RN2, 1);
      const double rn = std::sqrt(hsc_[S_RN2]);
      R.its = kk + 1;
      R.rel = rn / std::max(r0, 1e-300);
      if (!std::isfinite(R.rel)) throw SolveFailure(NDS_E_BREAKDOWN, "pressure stationary residual nonfinite");
      if (rn <= target) {
        R.ok = true;
        break;
      }
    }
    return R;
  }

  // ------------------------------------------- mixed-precision pressure solve
  // (precision NDS_MIXED: Solver<double, float>).  No reference counterpart.
  // FP64 defect correction around FP32 inner Krylov solves:
  //   target = max(atol, rtol ||b||); x = Galerkin guess (or 0); r = b - A x
  //   while ||r|| > target:  solve A d = r / ||r|| in FP32 (PCG or FGMRES,
  //   FP32 operator copy and V-cycle) to max(inner_rtol, target / (2 ||r||));
  //   x += ||r|| d;  r = b - A x in FP64 on the FP64 operator.
  // The stopping rule is the reference's ||r|| <= max(atol, rtol ||r0||)
  // with r0 = b (its zero initial guess), checked on the FP64 residual.
  void alloc_mixed() {
    const size_t n = (size_t)nc_;
    for (auto* b : {&xf_, &rf_, &zf_, &pf_, &qf_}) b->alloc(n);
    fg_m_ = o_.p_krylov == NDS_KRYLOV_FGMRES ? o_.p_restart : 0;
    if (fg_m_ > 0) {
      fgV_.alloc((size_t)(fg_m_ + 1) * n);
      fgZ_.alloc((size_t)fg_m_ * n);
      fg_.alloc((size_t)k::FgLayout{fg_m_}.size());
      fg_.zero(st_);
    }
    fgpart_.alloc((size_t)kMaxPartBlocks * std::max(fg_m_ + 1, 48));
    if (o_.p_guess > 0) {
      gY_.alloc((size_t)o_.p_guess * n);
      gW_.alloc((size_t)o_.p_guess * n);
      if (o_.p_guess_fresh) gYf_.alloc((size_t)o_.p_guess * n);
    }
  }
  // the preconditioner of the inner solves: z = M v (FP32).  With the
  // learned stage: z1 = N(v), t = v - A z1; the V-cycle then solves for t and
  // z = z1 + V(t) -- or, when the stage did not reduce the residual
  // (||t|| >= ||v||), z = V(v) (the plain preconditioner as fallback).
  // the inner PCG takes the fine pre-smoother's first step in the kernels
  // that produce r (plain V-cycle with a polynomial smoother only)
  bool pre_fused() const { return !stage_ && o_.amg_smoother != NDS_SM_MCGS; }
  void precond_f(const float* v, float* z) {
    if constexpr (!kSame) {
      if (!stage_) {
        amg_apply(v, z);
        return;
      }
      mpnn_forward(*stage_, stage_view(), v, st_z1_.p);
      op_resid(fine_opA(), (const float*)st_z1_.p, v, st_t_.p);
      dot_dev((const float*)st_t_.p, (const float*)st_t_.p, nc_, S_ST_T);
      dot_dev(v, v, nc_, S_ST_V);
      stage_select<<<red_grid(nc_), kBlock, 0, st_>>>(nc_, v, st_t_.p, st_z1_.p, sc_.p, S_ST_T, S_ST_V, st_cnt_.p);
      NDS_LAUNCH();
      amg_apply(st_t_.p, z);
      vaxpy(nc_, 1.0, (const float*)st_z1_.p, z);
    }
  }
  nds_mpnn_graph stage_view() const { return nds_mpnn_graph{nc_, sg_nbr_.p, sg_ew_.p, sg_dscale_.p}; }
  // face graph of the cells and the SELL offsets of its edges
  void build_stage_graph() {
    const Mesh& M = P_.mesh;
    const FineTopo& F = P_.setup.fine;
    std::vector<int32_t> nbr(4 * (size_t)nc_, -1), off(4 * (size_t)nc_, -1);
    std::vector<int> cnt((size_t)nc_, 0);
    auto add = [&](int a, int b) {
      if (cnt[(size_t)a] >= 4) throw std::runtime_error("learned stage: a cell with more than four face neighbours");
      nbr[4 * (size_t)a + cnt[(size_t)a]++] = b;
    };
    for (size_t f = 0; f < M.neighbour.size(); ++f) {
      add(M.owner[f], M.neighbour[f]);
      add(M.neighbour[f], M.owner[f]);
    }
    std::vector<int32_t> base((size_t)(nc_ + 31) / 32 + 1);
    NDS_CUDA(cudaMemcpy(base.data(), sbase_.p, sizeof(int32_t) * base.size(), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nc_; ++i)
      for (int k = 0; k < 4; ++k) {
        const int j = nbr[4 * (size_t)i + k];
        if (j < 0) continue;
        int pos = -1;
        for (int q = F.row[(size_t)i]; q < F.row[(size_t)i + 1]; ++q)
          if (F.col[(size_t)q] == j) pos = q - F.row[(size_t)i];
        if (pos < 0) throw std::runtime_error("learned stage: face neighbour missing from the pressure operator");
        off[4 * (size_t)i + k] = base[(size_t)(i >> 5)] + 128 * (pos >> 2) + 4 * (i & 31) + (pos & 3);
      }
    sg_nbr_.upload(nbr);
    sg_off_.upload(off);
    sg_ew_.alloc(4 * (size_t)nc_);
    sg_dscale_.alloc((size_t)nc_);
    st_z1_.alloc((size_t)nc_);
    st_t_.alloc((size_t)nc_);
    st_cnt_.alloc(2);
    st_cnt_.zero(st_);
  }
  // edge weights and scaling from the operator of the last refresh
  void update_stage_graph() {
    if constexpr (!kSame) {
      stage_dscale<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, fdiag_.p, sg_dscale_.p);
      NDS_LAUNCH();
      stage_edges<<<grid_for(4LL * nc_), kBlock, 0, st_>>>(nc_, sg_nbr_.p, sg_off_.p, fvalA_.p, sg_dscale_.p, sg_ew_.p);
      NDS_LAUNCH();
    }
  }
  void load_stage(const float* host) override {
    if constexpr (kSame) {
      throw SolveFailure(NDS_E_INVALID, "the learned stage needs precision mixed");
    } else {
      if (!mixed_ || fg_m_ == 0) throw SolveFailure(NDS_E_INVALID, "the learned stage needs precision mixed and FGMRES");
      if (!sg_nbr_.p) build_stage_graph();
      if (!stage_) stage_ = make_mpnn(nc_, false, st_);
      mpnn_set_params(*stage_, host);
      // the FGMRES loop body is captured with the stage: rebuild it
      if (g_fgmres_.exec) cudaGraphExecDestroy(g_fgmres_.exec);
      g_fgmres_.exec = nullptr;
      g_fgmres_.failed = false;
    }
  }
  void stage_graph(int32_t* nbr, float* ew, float* dscale) override {
    if constexpr (kSame) {
      throw SolveFailure(NDS_E_INVALID, "the learned stage needs precision mixed");
    } else {
      if (!sg_nbr_.p) build_stage_graph();
      update_stage_graph();
      if (nbr) NDS_CUDA(cudaMemcpyAsync(nbr, sg_nbr_.p, sg_nbr_.bytes(), cudaMemcpyDeviceToDevice, st_));
      if (ew) NDS_CUDA(cudaMemcpyAsync(ew, sg_ew_.p, sg_ew_.bytes(), cudaMemcpyDeviceToDevice, st_));
      if (dscale) NDS_CUDA(cudaMemcpyAsync(dscale, sg_dscale_.p, sg_dscale_.bytes(), cudaMemcpyDeviceToDevice, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
    }
  }
  void pressure_pair(float* rhs, float* x) override {
    if (rhs) {
      to_float<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, rhs_.p, rhs);
      NDS_LAUNCH();
    }
    if (x) {
      to_float<T><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, x_.p, x);
      NDS_LAUNCH();
    }
    NDS_CUDA(cudaStreamSynchronize(st_));
  }
  void apply_operator(const float* x, float* y) override {
    if constexpr (kSame) {
      throw SolveFailure(NDS_E_INVALID, "the FP32 operator product needs precision mixed or amg_fp32");
    } else {
      op_spmv(fine_opA(), x, y);
      NDS_CUDA(cudaStreamSynchronize(st_));
    }
  }
  void stage_counts(long long* applied, long long* fallbacks) override {
    unsigned long long c[2] = {0, 0};
    if (st_cnt_.p) {
      NDS_CUDA(cudaMemcpyAsync(c, st_cnt_.p, sizeof(c), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
    }
    if (applied) *applied = (long long)c[0];
    if (fallbacks) *fallbacks = (long long)c[1];
  }
  // one pass of the FP32 PCG loop: z = M r; rho; p; q = A p; alpha; x, r; check
  void pcgf_body(cudaGraphConditionalHandle h) {
    if constexpr (!kSame) {
      // the fine pre-smoother's first step on r is already in place (taken
      // by scale_to_float before the loop and by xr_update after it)
      if (pre_fused()) amg_apply(rf_.p, zf_.p, true);
      else precond_f(rf_.p, zf_.p);
      const int g = red_grid(nc_);
      k::dot<float><<<g, kBlock, 0, st_>>>(nc_, rf_.p, zf_.p, part_.p);
      NDS_LAUNCH();
      reduce_pcg<k::PCG_RHO>(g, S_RHON);
      k::p_update_dev<float><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, sc_.p + S_BETA, ctl_.p, zf_.p, pf_.p);
      NDS_LAUNCH();
      {
        ProfScope ps(prof, st_, P_FINE_AMG);
        sell_launch<k::SELL_DOT, float>(fine_opA(), g, pf_.p, nullptr, nullptr, 0.0, qf_.p, nullptr);
        NDS_LAUNCH();
      }
      reduce_pcg<k::PCG_ALPHA>(g, S_PQ);
      if (pre_fused()) {
        const PolyPlan pl = fine_plan();
        k::xr_update<float><<<g, kBlock, 0, st_>>>(nc_, 0.0, sc_.p + S_ALPHA, pf_.p, qf_.p, xf_.p, rf_.p, part_.p,
                                                    pl.den0, float(pl.w0), poly_first(pl, zf_.p, fpong_.p));
      } else {
        k::xr_update<float><<<g, kBlock, 0, st_>>>(nc_, 0.0, sc_.p + S_ALPHA, pf_.p, qf_.p, xf_.p, rf_.p, part_.p);
      }
      NDS_LAUNCH();
      reduce_pcg<k::PCG_CHECK>(g, S_RN2, -1, h, in_graph_);
    }
  }
  // one Arnoldi step of FGMRES: z_j = M v_j, w = A z_j, classical Gram-Schmidt
  // with FP64 dot products, Givens update of the least-squares problem
  void fg_body(cudaGraphConditionalHandle h) {
    if constexpr (!kSame) {
      const int g = red_grid(nc_);
      const k::FgLayout L{fg_m_};
      k::fg_fetch<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, fgV_.p, ctl_.p, rf_.p);
      NDS_LAUNCH();
      precond_f(rf_.p, zf_.p);
      k::fg_store<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, zf_.p, ctl_.p, fgZ_.p);
      NDS_LAUNCH();
      op_spmv(fine_opA(), (const float*)zf_.p, qf_.p);
      k::fg_dots<<<dim3(g, fg_m_ + 1), kBlock, 0, st_>>>(nc_, fgV_.p, qf_.p, ctl_.p, fgpart_.p);
      NDS_LAUNCH();
      k::fg_reduce_h<<<fg_m_ + 1, kBlock, 0, st_>>>(fgpart_.p, g, ctl_.p, L, fg_.p);
      NDS_LAUNCH();
      k::fg_orth<<<g, kBlock, 0, st_>>>(nc_, fgV_.p, fg_.p, L, ctl_.p, qf_.p, part_.p);
      NDS_LAUNCH();
      reduce_to<1>(g, S_RN2);
      k::fg_givens<<<1, 1, 0, st_>>>(fg_.p, L, sc_.p, S_RN2, S_WN, S_TARGET, ctl_.p, flags_.p, h, in_graph_);
      NDS_LAUNCH();
      k::fg_normalize<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, qf_.p, sc_.p, S_WN, ctl_.p, fgV_.p);
      NDS_LAUNCH();
    }
  }
  template <class Body>
  bool build_loop(LoopGraph& G, Body&& body) {
    const bool was = prof.on;
    prof.on = false;
    cudaGraph_t graph = nullptr;
    bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess;
    cudaGraphConditionalHandle h{};
    cudaGraphNodeParams cp{};
    cudaGraphNode_t node{};
    if (ok) ok = cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
    }
    const unsigned long long l0 = g_launches;
    if (ok) ok = cudaStreamBeginCaptureToGraph(st_, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      bool body_ok = true;
      in_graph_ = 1;
      try {
        body(h);
      } catch (...) {
        body_ok = false;
      }
      in_graph_ = 0;
      ok = cudaStreamEndCapture(st_, nullptr) == cudaSuccess && body_ok;
    }
    G.body_kernels = g_launches - l0;
    g_launches = l0;
    if (ok) ok = cudaGraphInstantiate(&G.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
      if (G.exec) cudaGraphExecDestroy(G.exec);
      G.exec = nullptr;
      G.failed = true;
      cudaGetLastError();
    }
    prof.on = was;
    return ok;
  }
  // Runs a device loop (or, with graphs off or the profiler on, the same
  // body launch by launch with a host-side test of the loop condition).
  // ctl[0..3] must be set by the caller; returns after the loop ends.
  template <class Body>
  void run_loop(LoopGraph& G, Body&& body) {
    if (use_graphs_ && !prof.on && !G.failed && (G.exec || build_loop(G, body))) {
      NDS_CUDA(cudaGraphLaunch(G.exec, st_));
      NDS_CUDA(cudaMemcpyAsync(hflags_ + 4, ctl_.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaMemcpyAsync(hflags_, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
      g_launches += (unsigned long long)hflags_[4] * G.body_kernels;
      return;
    }
    // host-driven: the body's check kernel (launched with in_graph_ = 0)
    // leaves the decision to this loop, which reads ctl and the flags
    for (;;) {
      body(cudaGraphConditionalHandle{});
      NDS_CUDA(cudaMemcpyAsync(hflags_ + 4, ctl_.p, 4 * sizeof(int), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaMemcpyAsync(hflags_, flags_.p, sizeof(int), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
      prof.collect();
      const int its = hflags_[4], conv = hflags_[5], cap = hflags_[7];
      if (conv || hflags_[0] != 0 || its >= cap) break;
    }
  }
  void set_target(double tol, double r0) {
    hsc_[S_R0] = r0;
    hsc_[S_TARGET] = tol;
    NDS_CUDA(cudaMemcpyAsync(sc_.p + S_R0, hsc_ + S_R0, 2 * sizeof(double), cudaMemcpyHostToDevice, st_));
  }
  void set_ctl(int a, int b, int c, int d) {
    const int init[4] = {a, b, c, d};
    std::memcpy(hflags_ + 4, init, sizeof(init));
    NDS_CUDA(cudaMemcpyAsync(ctl_.p, hflags_ + 4, 4 * sizeof(int), cudaMemcpyHostToDevice, st_));
    NDS_CUDA(cudaMemsetAsync(flags_.p, 0, sizeof(int), st_));
  }
  // inner FP32 PCG on rf_ (unit norm) from xf_ = 0 to ||r|| <= tol within
  // cap iterations; returns the iterations
  int inner_pcg(double tol, int cap) {
    xf_.zero(st_);
    set_target(tol, 1.0);
    set_ctl(0, 0, 1, cap);
    run_loop(g_loopf_, [&](cudaGraphConditionalHandle h) { pcgf_body(h); });
    const int f = hflags_[0];
    if (f & 8) throw SolveFailure(NDS_E_BREAKDOWN, "inner FP32 PCG initial rho nonpositive");
    if (f & 1) throw SolveFailure(NDS_E_BREAKDOWN, "inner FP32 PCG pAp nonpositive");
    if (f & 2) throw SolveFailure(NDS_E_BREAKDOWN, "inner FP32 PCG rho nonpositive");
    if (f & 4) throw SolveFailure(NDS_E_BREAKDOWN, "inner FP32 PCG residual nonfinite");
    return hflags_[4];
  }
  // one FGMRES pass on V_0 = r / rn: x += rn sum y_i z_i; returns the
  // Arnoldi steps taken
  int inner_fgmres(double rn, double tol, int cap) {
    const k::FgLayout L{fg_m_};
    k::scale_to_float<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, r_.p, 1.0 / rn, fgV_.p);
    NDS_LAUNCH();
    set_target(tol, 1.0);
    set_ctl(0, 0, 0, cap);
    k::fg_start<<<1, 1, 0, st_>>>(fg_.p, L, ctl_.p, cap);
    NDS_LAUNCH();
    run_loop(g_fgmres_, [&](cudaGraphConditionalHandle h) { fg_body(h); });
    if (hflags_[0] & 16) throw SolveFailure(NDS_E_BREAKDOWN, "inner FGMRES breakdown or nonfinite value");
    const int k_done = hflags_[4];
    k::fg_backsolve<<<1, 1, 0, st_>>>(fg_.p, L, ctl_.p);
    NDS_LAUNCH();
    k::fg_combine<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, fgZ_.p, fg_.p, L, ctl_.p, rn, x_.p);
    NDS_LAUNCH();
    return k_done;
  }
  // Galerkin guess over the stored corrections and their stored products:
  // sets x_ and the exact FP64 residual r_ = b - A x_; returns ||r|| (or a
  // negative value when the guess is not usable: then nothing is set)
  template <int K>
  double guess_k(const double* rhs) {
    constexpr int NG = K * (K + 1) / 2 + K;
    const int g = red_grid(nc_);
    if constexpr (!kSame) {
      if (o_.p_guess_fresh) {
        // products with this iteration's operator (FP32 copy), widened to FP64
        const size_t n = (size_t)nc_;
        for (int a = 0; a < K; ++a) {
          op_spmv(fine_opA(), (const float*)(gYf_.p + a * n), qf_.p);
          k::cast_copy<float, double><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, qf_.p, gW_.p + a * n);
          NDS_LAUNCH();
        }
      }
    }
    k::guess_dots<K><<<g, kBlock, 0, st_>>>(nc_, gY_.p, gW_.p, rhs, fgpart_.p);
    NDS_LAUNCH();
    k::reduce_partials<NG><<<1, kBlock, 0, st_>>>(fgpart_.p, g, sc_.p + S_GUESS);
    NDS_LAUNCH();
    fetch(S_GUESS, NG);
    // G c = f by Cholesky (no guess when G is not numerically positive
    // definite, e.g. for dependent corrections)
    double G[K][K], f[K], c[K];
    int q = 0;
    for (int a = 0; a < K; ++a)
      for (int b = a; b < K; ++b) G[a][b] = G[b][a] = hsc_[S_GUESS + q++];
    for (int a = 0; a < K; ++a) f[a] = hsc_[S_GUESS + q++];
    double Lc[K][K] = {};
    for (int a = 0; a < K; ++a) {
      for (int b = 0; b <= a; ++b) {
        double sum = G[a][b];
        for (int e = 0; e < b; ++e) sum -= Lc[a][e] * Lc[b][e];
        if (a == b) {
          if (!(sum > 1e-12 * std::max(G[a][a], 1e-300)) || !std::isfinite(sum)) return -1.0;
          Lc[a][a] = std::sqrt(sum);
        } else {
          Lc[a][b] = sum / Lc[b][b];
        }
      }
    }
    for (int a = 0; a < K; ++a) {
      double sum = f[a];
      for (int e = 0; e < a; ++e) sum -= Lc[a][e] * c[e];
      c[a] = sum / Lc[a][a];
    }
    for (int a = K - 1; a >= 0; --a) {
      double sum = c[a];
      for (int e = a + 1; e < K; ++e) sum -= Lc[e][a] * c[e];
      c[a] = sum / Lc[a][a];
    }
    for (int a = 0; a < K; ++a) {
      if (!std::isfinite(c[a])) return -1.0;
      hsc_[S_COEF + a] = c[a];
    }
    NDS_CUDA(cudaMemcpyAsync(sc_.p + S_COEF, hsc_ + S_COEF, K * sizeof(double), cudaMemcpyHostToDevice, st_));
    k::guess_combine<K><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, gY_.p, sc_.p + S_COEF, x_.p);
    NDS_LAUNCH();
    op_resid(fine_op(), (const double*)x_.p, rhs, r_.p);
    return std::sqrt(dot_fetch((const double*)r_.p, (const double*)r_.p, nc_, S_TMP));
  }
  double apply_guess(const double* rhs) {
    switch (std::min(o_.p_guess, nguess_)) {
      case 1: return guess_k<1>(rhs);
      case 2: return guess_k<2>(rhs);
      case 3: return guess_k<3>(rhs);
      case 4: return guess_k<4>(rhs);
      case 5: return guess_k<5>(rhs);
      case 6: return guess_k<6>(rhs);
      case 7: return guess_k<7>(rhs);
      case 8: return guess_k<8>(rhs);
      default: return -1.0;
    }
  }
  // keep the solution and its product with this iteration's operator,
  // w = b - r (r_ holds the final FP64 defect b - A x)
  void store_guess(const double* rhs) {
    if (o_.p_guess <= 0) return;
    const size_t o = (size_t)guess_head_ * nc_;
    k::guess_store<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, x_.p, rhs, r_.p, gY_.p + o, gW_.p + o);
    NDS_LAUNCH();
    if (gYf_.p) {
      k::cast_copy<double, float><<<grid_for(nc_), kBlock, 0, st_>>>(nc_, x_.p, gYf_.p + o);
      NDS_LAUNCH();
    }
    guess_head_ = (guess_head_ + 1) % o_.p_guess;
    nguess_ = std::min(nguess_ + 1, o_.p_guess);
  }
  PRes mixed_solve(const T* rhs_t) {
    PRes R;
    if constexpr (!kSame) {
      const double* rhs = rhs_t;
      // ||b|| = ||B u + fixedDiv||: the continuity norm this iteration already read back
      const double bn = std::sqrt(hsc_[S_CONT2]);
      if (!std::isfinite(bn)) throw SolveFailure(NDS_E_BREAKDOWN, "pressure initial norm nonfinite");
      const double target = std::max(o_.p_atol, o_.p_rtol * bn);
      start_readback();
      if (bn <= o_.p_atol) {
        x_.zero(st_);
        R.ok = true;
        R.rel = 0.0;
        return R;
      }
      if (o_.learned && !stage_) throw SolveFailure(NDS_E_STATE, "learned stage enabled but no parameters loaded");
      if (stage_) update_stage_graph();
      double rn = -1.0;
      if (o_.p_guess > 0 && nguess_ > 0) rn = apply_guess(rhs);
      // a guess that does not reduce the residual is dropped
      if (!(rn >= 0.0) || !std::isfinite(rn) || rn >= bn) {
        x_.zero(st_);
        vcopy(nc_, rhs, r_.p);
        rn = bn;
      }
      int passes = 0;
      for (;;) {
        if (rn <= target) {
          R.ok = true;
          break;
        }
        if (passes >= o_.p_refine_max || R.its >= o_.p_max) break;
        const double tol = std::max(o_.p_inner_rtol, 0.5 * target / rn);
        const int cap = o_.p_max - R.its;
        if (fg_m_ > 0) {
          R.its += inner_fgmres(rn, tol, std::min(cap, fg_m_));
        } else {
          if (pre_fused()) {
            const PolyPlan pl = fine_plan();
            k::scale_to_float<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, r_.p, 1.0 / rn, rf_.p, pl.den0, float(pl.w0),
                                                                 poly_first(pl, zf_.p, fpong_.p));
          } else {
            k::scale_to_float<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, r_.p, 1.0 / rn, rf_.p);
          }
          NDS_LAUNCH();
          R.its += inner_pcg(tol, cap);
          k::axpy_from_float<<<grid_for(nc_), kBlock, 0, st_>>>(nc_, rn, xf_.p, x_.p);
          NDS_LAUNCH();
        }
        ++passes;
        op_resid(fine_op(), (const double*)x_.p, rhs, r_.p);
        rn = std::sqrt(dot_fetch((const double*)r_.p, (const double*)r_.p, nc_, S_TMP));
        if (!std::isfinite(rn)) throw SolveFailure(NDS_E_BREAKDOWN, "pressure defect nonfinite");
      }
      R.rel = rn / std::max(bn, 1e-300);
      last_passes_ = passes;
      if (stage_) mpnn_check(*stage_);
      if (R.ok) store_guess(rhs);
    }
    return R;
  }

  // ------------------------------------------------------ SIMPLE iteration
  void assemble() {
    k::MomArgs<T> a;
    a.nrows = nv_;
    a.span = mspan_.p;
    a.dpos = mdpos_.p;
    a.K = K_.p;
    a.inc_off = inc_off_.p;
    a.inc = inc_.p;
    a.ref = ref_.p;
    a.slot = slot_.p;
    a.C = cconv_.p;
    a.slotz = slotz_.p;
    a.Bz = bz_.p;
    a.pz = pz_.p;
    a.fixz = fixz_.p;
    a.bco = bco_.p;
    a.fixed = fixed_.p;
    a.u0 = uc(0);
    a.u1 = uc(1);
    a.u2 = uc(2);
    a.p = p_.p;
    a.s0 = s_[0].p;
    a.s1 = s_[1].p;
    a.s2 = s_[2].p;
    a.alpha_u = T(o_.alpha_u);
    a.rau_scale = T(o_.rau_scale);
    a.row_cap = row_cap_;
    a.A = A_.p;
    a.delta = delta_.p;
    a.diag = diag_.p;
    a.rau = rau_.p;
    a.b0 = b_[0].p;
    a.b1 = b_[1].p;
    a.b2 = b_[2].p;
    a.invJ = invJ_.p;
    a.det = det_.p;
    a.centT = centT_.p;
    ProfScope ps(prof, st_, P_ASSEMBLE);
    if (fused_assembly_) {
      // one pass: each incidence's convection row is evaluated in place
      k::mom_assemble<T, 1><<<grid_for(nv_, kBlock / 8), kBlock, mom_smem_ + 1536 * sizeof(T), st_>>>(a);
      NDS_LAUNCH();
      return;
    }
    // cell blocks: a grid of 8 blocks per SM amortises the shared tensor load
    k::SupgArgs sa{P_.setup.pipe.nu, o_.supg_tau_scale, o_.supg_magic};
    const int gc = std::min(grid_for(nc_, kBlock / 8), 8 * 148);
    if (o_.supg)
      k::mom_cell_conv<T, true><<<gc, kBlock, 0, st_>>>(nc_, ref_.p, fixed_.p, uc(0), uc(1), uc(2), invJ_.p,
                                                       det_.p, centT_.p, zpos_.p, cconv_.p, p_.p, pz_.p, supg_rule_.p,
                                                       h2_.p, sa);
    else
      k::mom_cell_conv<T, false><<<gc, kBlock, 0, st_>>>(nc_, ref_.p, fixed_.p, uc(0), uc(1), uc(2), invJ_.p,
                                                        det_.p, centT_.p, zpos_.p, cconv_.p, p_.p, pz_.p, nullptr,
                                                        nullptr, sa);
    NDS_LAUNCH();
    k::mom_assemble<T><<<grid_for(nv_, kBlock / 8), kBlock, mom_smem_, st_>>>(a);
    NDS_LAUNCH();
  }
  void gs_pass(bool reverse) {
    const int ncol = (int)color_off_.size() - 1;
    for (int qq = 0; qq < ncol; ++qq) {
      const int c = reverse ? ncol - 1 - qq : qq;
      const int s = color_off_[(size_t)c], n = color_off_[(size_t)c + 1] - s;
      if (!n) continue;
      ProfScope ps(prof, st_, P_GS);
      k::mom_gs_color<T><<<grid_for((long long)n * 8), kBlock, 0, st_>>>(
          n, color_rows_.p + s, gspan_.p + s, mcol_.p, A_.p, diag_.p, b_[0].p, b_[1].p, b_[2].p, uc(0), uc(1), uc(2),
          T(o_.mom_omega));
      NDS_LAUNCH();
    }
  }
  std::array<double, 3> audit() {
    const int g = red_grid((long long)nv_ * 8);
    k::mom_audit<T><<<g, kBlock, 0, st_>>>(nv_, mspan_.p, mcol_.p, A_.p, b_[0].p, b_[1].p, b_[2].p, uc(0), uc(1),
                                           uc(2), part_.p);
    NDS_LAUNCH();
    reduce_to<6>(g, S_AUDIT);
    fetch(S_AUDIT, 6);
    std::array<double, 3> q{};
    for (int d = 0; d < 3; ++d) {
      double bn = std::sqrt(std::max(0.0, hsc_[S_AUDIT + d]));
      if (bn == 0.0) bn = 1.0;
      q[(size_t)d] = std::sqrt(std::max(0.0, hsc_[S_AUDIT + 3 + d])) / bn;
    }
    return q;
  }
  double rau_snapshot_rel() {
    // ||rau - rau_setup|| / ||rau_setup||, in double on the host copies
    std::vector<T> a((size_t)nv_), b((size_t)nv_);
    NDS_CUDA(cudaMemcpyAsync(a.data(), rau_.p, sizeof(T) * nv_, cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaMemcpyAsync(b.data(), rau_pc_.p, sizeof(T) * nv_, cudaMemcpyDeviceToHost, st_));
    NDS_CUDA(cudaStreamSynchronize(st_));
    long double d = 0, r = 0;
    for (int i = 0; i < nv_; ++i) {
      const long double q = (long double)a[(size_t)i] - (long double)b[(size_t)i];
      d += q * q;
      r += (long double)b[(size_t)i] * b[(size_t)i];
    }
    return std::sqrt((double)d) / std::max(std::sqrt((double)r), 1e-300);
  }

  void reset() override {
    u3_.zero(st_);
    p_.zero(st_);
    it_ = 0;
    nguess_ = 0;
    guess_head_ = 0;
    cont0_ = -1.0;
    cont_rel_ = 1.0;
    NDS_CUDA(cudaStreamSynchronize(st_));
  }

  void step(nds_iter_report* rep) override {
    const int it = ++it_;
    nds_iter_report R{};
    R.it = it;
    NDS_CUDA(cudaEventRecord(ev_[0], st_));
    assemble();
    NDS_CUDA(cudaEventRecord(ev_[1], st_));
    // The fine Schur refresh needs only rAU from the assembly: it runs on the
    // side stream while the momentum sweep and the continuity residual run
    // on the main stream (it writes only the pressure operator, which
    // nothing reads until the pressure solve waits for it).
    NDS_CUDA(cudaEventRecord(ev_side_[0], st_));
    NDS_CUDA(cudaStreamWaitEvent(st2_, ev_side_[0], 0));
    refresh_fine(rau_.p, st2_);
    NDS_CUDA(cudaEventRecord(ev_side_[1], st2_));
    if (it == 1) {
      const double rr = rau_snapshot_rel();
      if (!(rr < o_.snapshot_tol))
        throw SolveFailure(NDS_E_SETUP, "setup rAU snapshot mismatch (rel " + std::to_string(rr) + ")");
    }
    const bool converge = o_.run_mode == NDS_RUN_CONVERGE;
    if (converge && it > 1 && cont_rel_ <= o_.simple_tol) {
      auto q = audit();
      R.audited = 1;
      for (int d = 0; d < 3; ++d) R.audit_rel[d] = q[(size_t)d];
    }
    if (o_.momentum_work == NDS_MOM_FGS1) gs_pass(false);
    else if (o_.momentum_work == NDS_MOM_ALTGS1) gs_pass((it & 1) == 0);
    else { gs_pass(false); gs_pass(true); }
    NDS_CUDA(cudaEventRecord(ev_[2], st_));
    {
      const int g = red_grid(nc_);
      ProfScope ps(prof, st_, P_CONTINUITY);
      k::continuity<T><<<g, kBlock, 0, st_>>>(nc_, ref_.p, bco_.p, fixed_div_.p, uc(0), uc(1), uc(2), rhs_.p,
                                             part_.p);
      NDS_LAUNCH();
      reduce_to<1>(g, S_CONT2);
      fetch(S_CONT2, 1);
    }
    const double cn = std::sqrt(hsc_[S_CONT2]);
    if (it == 1) cont0_ = cn;
    cont_rel_ = cn / std::max(cont0_, 1e-300);
    R.cont_norm = cn;
    R.rel_cont = cont_rel_;
    NDS_CUDA(cudaEventRecord(ev_[3], st_));
    NDS_CUDA(cudaStreamWaitEvent(st_, ev_side_[1], 0));
    NDS_CUDA(cudaEventRecord(ev_[6], st_));
    PRes pr;
    if (mixed_) pr = mixed_solve(rhs_.p);
    else if (o_.pressure_solver == NDS_P_PCG) pr = pcg(rhs_.p);
    else pr = stationary(rhs_.p, o_.pressure_solver == NDS_P_CHEB);
    R.p_its = pr.its;
    R.p_rel = pr.rel;
    NDS_CUDA(cudaEventRecord(ev_[4], st_));
    if (!pr.ok) {
      last_ = R;
      throw SolveFailure(NDS_E_NOT_CONVERGED, "pressure solve failed its requested target");
    }
    vaxpy(nc_, o_.alpha_p, x_.p, p_.p);
    NDS_CUDA(cudaEventRecord(ev_[5], st_));
    if constexpr (std::is_same<T, double>::value) {
      if (io_out_ && io_out_[3]) NDS_CUDA(cudaMemcpyAsync(io_out_[3], p_.p, p_.bytes(), cudaMemcpyDeviceToHost, st_));
    }
    NDS_CUDA(cudaStreamSynchronize(st_));
    if (io_pending_) {
      NDS_CUDA(cudaEventSynchronize(ev_io_));
      io_pending_ = false;
    }
    prof.collect();
    float ms[5];
    for (int q = 0; q < 5; ++q) NDS_CUDA(cudaEventElapsedTime(&ms[q], ev_[q], ev_[q + 1]));
    R.ms_assembly = ms[0];
    R.ms_momentum = ms[1];
    R.ms_continuity = ms[2];
    R.ms_pressure = ms[3];
    R.ms_update = ms[4];
    float msr = 0.f;
    NDS_CUDA(cudaEventElapsedTime(&msr, ev_[3], ev_[6]));
    R.ms_refresh = msr;
    const bool finite = std::isfinite(R.rel_cont) && std::isfinite(R.p_rel) &&
                        (!R.audited || (std::isfinite(R.audit_rel[0]) && std::isfinite(R.audit_rel[1]) &&
                                        std::isfinite(R.audit_rel[2])));
    finite_all_ = finite_all_ && finite;
    if (R.audited)
      R.all_momentum_met = R.audit_rel[0] <= o_.simple_tol && R.audit_rel[1] <= o_.simple_tol &&
                           R.audit_rel[2] <= o_.simple_tol;
    R.converged = converge && finite_all_ && R.rel_cont <= o_.simple_tol && R.audited && R.all_momentum_met;
    last_ = R;
    if (rep) *rep = R;
  }

  void solve(nds_solve_report* rep) override {
    nds_solve_report S{};
    S.pressure_all = 1;
    finite_all_ = true;
    long long sumP = 0;
    for (int it = 1; it <= o_.max_outer; ++it) {
      nds_iter_report R{};
      step(&R);
      sumP += R.p_its;
      S.outer_its = R.it;
      S.final_rel_cont = R.rel_cont;
      if (R.audited)
        for (int d = 0; d < 3; ++d) S.final_audit_rel[d] = R.audit_rel[d];
      S.assembly_ms += R.ms_assembly;
      S.momentum_ms += R.ms_momentum;
      S.continuity_ms += R.ms_continuity;
      S.pressure_ms += R.ms_pressure;
      S.update_ms += R.ms_update;
      if (o_.verbose)
        std::printf(
            "NODALS_GPU_H8_SIMPLE it=%d relCont=%.12e pCG=%d pTrueRel=%.3e residualAudit=%s auditInitRel=[%.3e,%.3e,%.3e] "
            "allMomentumMet=%d converged=%d\n",
            R.it, R.rel_cont, R.p_its, R.p_rel, R.audited ? "DONE" : "SKIPPED", R.audit_rel[0], R.audit_rel[1],
            R.audit_rel[2], R.all_momentum_met, R.converged);
      if (R.converged) {
        S.converged = 1;
        break;
      }
    }
    S.finite_all = finite_all_;
    S.avg_pressure_its = S.outer_its ? (double)sumP / S.outer_its : 0.0;
    S.loop_ms = S.assembly_ms + S.momentum_ms + S.continuity_ms + S.pressure_ms + S.update_ms;
    if (rep) *rep = S;
  }

  bool cell_arrays(const int32_t** ref, const double** bco, const double** fixed_div, int* nc,
                   int* device) const override {
    if constexpr (std::is_same<T, double>::value) {
      *ref = ref_.p;
      *bco = bco_.p;
      *fixed_div = fixed_div_.p;
      *nc = nc_;
      *device = o_.device;
      return true;
    } else {
      return false;
    }
  }
  void get_fields(double* u0, double* u1, double* u2, double* p) override {
    std::vector<T> h;
    auto get = [&](const DBuf<T>& b, double* out) {
      if (!out) return;
      if (std::is_same<T, double>::value) {  // straight DMA into the caller's buffer
        NDS_CUDA(cudaMemcpyAsync(out, b.p, b.bytes(), cudaMemcpyDeviceToHost, st_));
        NDS_CUDA(cudaStreamSynchronize(st_));
        return;
      }
      h.resize(b.n);
      NDS_CUDA(cudaMemcpyAsync(h.data(), b.p, b.bytes(), cudaMemcpyDeviceToHost, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
      for (size_t i = 0; i < b.n; ++i) out[i] = (double)h[i];
    };
    if (u0 || u1 || u2) {
      k::deinterleave3<T><<<grid_for(nv_), kBlock, 0, st_>>>(nv_, u3_.p, v_[0].p, v_[1].p, v_[2].p);
      NDS_LAUNCH();
    }
    get(v_[0], u0);
    get(v_[1], u1);
    get(v_[2], u2);
    get(p_, p);
  }
  void set_fields(const double* u0, const double* u1, const double* u2, const double* p) override {
    auto put = [&](DBuf<T>& b, const double* in) {
      if (!in) return;
      if (std::is_same<T, double>::value) {
        NDS_CUDA(cudaMemcpyAsync(b.p, in, b.bytes(), cudaMemcpyHostToDevice, st_));
        NDS_CUDA(cudaStreamSynchronize(st_));
        return;
      }
      std::vector<T> h(in, in + b.n);
      NDS_CUDA(cudaMemcpyAsync(b.p, h.data(), b.bytes(), cudaMemcpyHostToDevice, st_));
      NDS_CUDA(cudaStreamSynchronize(st_));
    };
    put(v_[0], u0);
    put(v_[1], u1);
    put(v_[2], u2);
    if (u0 || u1 || u2) {
      k::interleave3<T><<<grid_for(nv_), kBlock, 0, st_>>>(nv_, u0 ? v_[0].p : nullptr, u1 ? v_[1].p : nullptr,
                                                           u2 ? v_[2].p : nullptr, u3_.p);
      NDS_LAUNCH();
      NDS_CUDA(cudaStreamSynchronize(st_));
    }
    put(p_, p);
  }

  // step_io: the velocity is final after the momentum sweep (event ev_[2]);
  // it is read back on the I/O stream once the pressure solve has read its
  // initial norm, so that the copy runs under the device-side Krylov loop.
  // (Issued earlier, it would hold up the small reads the host waits for
  // between the sweep and the loop: they share the copy engine.)
  void start_readback() {
    if constexpr (std::is_same<T, double>::value) {
      if (!io_out_ || io_issued_ || !(io_out_[0] || io_out_[1] || io_out_[2])) return;
      io_issued_ = true;
      NDS_CUDA(cudaStreamWaitEvent(st_io_, ev_[2], 0));
      k::deinterleave3<T><<<grid_for(nv_), kBlock, 0, st_io_>>>(nv_, u3_.p, v_[0].p, v_[1].p, v_[2].p);
      NDS_LAUNCH();
      for (int d = 0; d < 3; ++d)
        if (io_out_[d]) NDS_CUDA(cudaMemcpyAsync(io_out_[d], v_[d].p, v_[d].bytes(), cudaMemcpyDeviceToHost, st_io_));
      NDS_CUDA(cudaEventRecord(ev_io_, st_io_));
      io_pending_ = true;
    }
  }
  void step_io(const double* const in[4], double* const out[4], nds_iter_report* rep) override {
    set_fields(in[0], in[1], in[2], in[3]);
    // Overlapped read-back needs an FP64 state (no host-side conversion) and
    // page-locked outputs (a copy into pageable memory would block the host
    // before the rest of the step is queued).
    bool overlap = std::is_same<T, double>::value;
    for (int q = 0; q < 4 && overlap; ++q) {
      if (!out[q]) continue;
      cudaPointerAttributes a{};
      if (cudaPointerGetAttributes(&a, out[q]) != cudaSuccess || a.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        overlap = false;
      }
    }
    if (!overlap) {
      step(rep);
      get_fields(out[0], out[1], out[2], out[3]);
      return;
    }
    io_out_ = out;
    io_issued_ = false;
    try {
      step(rep);
      start_readback();  // no-op unless the pressure stage did not issue it
      if (io_pending_) {
        NDS_CUDA(cudaEventSynchronize(ev_io_));
        io_pending_ = false;
      }
    } catch (...) {
      // no copy may write the caller's arrays after the call returns
      io_out_ = nullptr;
      cudaStreamSynchronize(st_io_);
      cudaStreamSynchronize(st_);
      io_pending_ = false;
      throw;
    }
    io_out_ = nullptr;
  }

  nds_iter_report last_{};

 private:
  const Problem& P_;
  nds_options o_;
  cudaStream_t st_ = nullptr;
  cudaStream_t st2_ = nullptr;      // side stream of the fine Schur refresh
  cudaEvent_t ev_side_[2] = {};     // assembly done -> refresh; refresh done -> pressure
  cudaStream_t st_io_ = nullptr;    // read-back of step_io
  cudaEvent_t ev_io_ = nullptr;
  double* const* io_out_ = nullptr;  // outputs of the step_io call in progress
  bool io_pending_ = false, io_issued_ = false;
  cudaEvent_t ev_[7] = {};
  int nc_ = 0, nv_ = 0, row_cap_ = 0, it_ = 0;
  size_t mom_smem_ = 0, refresh_smem_ = 0;
  double cont0_ = -1, cont_rel_ = 1, fine_lambda_ = 1, p_cheb_lambda_ = 1;
  bool finite_all_ = true;
  bool fused_assembly_ = false;
  // lanes per row of the FP16 level SpMVs and of the restriction in the
  // mixed FP16 V-cycle (16 measured best at pipe1m: 0.25 ms per SIMPLE
  // iteration less than 32 or 8); NDS_LEVEL_LANES=8|16|32 overrides
  int level_lanes_ = std::getenv("NDS_LEVEL_LANES") ? std::atoi(std::getenv("NDS_LEVEL_LANES")) : 16;
  std::vector<double> level_lambda_;
  // momentum
  DBuf<int32_t> mcol_, mdpos_, inc_off_, ref_, color_rows_;
  DBuf<uint32_t> inc_;
  DBuf<int32_t> zpos_;  // incidence of (cell, basis), -1 for a fixed dof
  DBuf<uint8_t> slot_, slotz_, fixz_;  // slots per (cell, basis) and per incidence; fixed-dof masks
  DBuf<T> K_, A_, diag_, delta_, rau_, rau_pc_, det_, invJ_, bco_, fixed_, fixed_div_, centT_, cconv_, fgeo_, p_, bz_, pz_;
  DBuf<T> h2_, supg_rule_;
  DBuf<T> u3_, b_[3], s_[3], v_[3];  // u3_: interleaved velocity; v_: staging of get/set fields
  static constexpr int kVelComponents = k::kVel;
  T* uc(int d) const { return u3_.p + d; }
  std::vector<int> color_off_;
  DBuf<int2> mspan_, gspan_;  // momentum rows' storage spans, by row / by colour position
  // pressure
  DBuf<int32_t> fcoff_, fine_crows_, sbase_, swidth_, scol_, fdslot_;
  DBuf<int16_t> sdcol_;
  k::Sell sell_{};
  long long sell_nnz_ = 0;
  std::vector<int> fine_coff_;
  DBuf<uint16_t> fcs_;
  DBuf<int> ctl_;

  DBuf<T> fval_, x_, r_, z_, pp_, q_, rhs_;
  DBuf<TA> fvalA_, fdiag_, fl1_, fr_, ftmp_, fcorr_, frhs_, fpong_, tinv_, rA_, zA_;
  std::vector<Level> L_;
  std::vector<Xfer> X_;
  // mixed precision (NDS_MIXED): inner FP32 Krylov vectors, FGMRES basis
  // V (m+1 vectors) and preconditioned vectors Z (m), its FP64 work array,
  // and the stored corrections Y (and A Y) of the Galerkin guess
  bool mixed_ = false;
  int in_graph_ = 0;  // 1 while a loop body is being captured (its check kernel sets the graph condition)
  int fg_m_ = 0, nguess_ = 0, guess_head_ = 0, last_passes_ = 0;
  DBuf<float> xf_, rf_, zf_, pf_, qf_, fgV_, fgZ_, gYf_;
  DBuf<__half> fvalH_;  // FP16 copy of the fine operator for the V-cycle (amg_half)
  double hscale_ = 1.0;
  DBuf<double> fg_, fgpart_, gY_, gW_;
  LoopGraph g_loopf_, g_fgmres_;
  // learned stage: network state, face graph (neighbours, SELL offsets of
  // the edges, edge weights, Jacobi scaling), work vectors, counters
  MpnnPtr stage_;
  DBuf<int32_t> sg_nbr_, sg_off_;
  DBuf<float> sg_ew_, sg_dscale_, st_z1_, st_t_;
  DBuf<unsigned long long> st_cnt_;
  DBuf<double> part_, sc_;
  DBuf<int> flags_;
  double* hsc_ = nullptr;
  int* hflags_ = nullptr;  // [0] flags, [4..7] device-loop control words
};

}  // namespace nds

// ============================================================== C ABI
struct nds_solver {
  std::unique_ptr<nds::ISolver> impl;
};

namespace {
int fail(int code, const std::string& m) {
  nds::set_error(m);
  return code;
}
template <class F>
int guarded(F&& f) {
  try {
    f();
    return NDS_OK;
  } catch (const nds::SolveFailure& e) {
    return fail(e.code, e.what());
  } catch (const nds::CudaError& e) {
    return fail(NDS_E_CUDA, e.what());
  } catch (const std::exception& e) {
    return fail(NDS_E_SETUP, e.what());
  }
}
}  // namespace

extern "C" {

int nds_solver_create(const nds_problem* pp, nds_solver** out) {
  if (!pp || !out) return fail(NDS_E_INVALID, "null argument");
  const auto* P = reinterpret_cast<const nds::Problem*>(pp);
  return guarded([&] {
    int ndev = 0;
    const cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= P->opt.device)
      throw nds::CudaError(std::string("no CUDA device available: ") + cudaGetErrorString(e));
    auto s = std::make_unique<nds_solver>();
    if (P->opt.precision == NDS_FP64) s->impl = std::make_unique<nds::Solver<double, double>>(*P);
    else if (P->opt.precision == NDS_FP32) s->impl = std::make_unique<nds::Solver<float, float>>(*P);
    else s->impl = std::make_unique<nds::Solver<double, float>>(*P);
    *out = s.release();
  });
}
int nds_solver_reset(nds_solver* s) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->reset(); });
}
int nds_simple_step(nds_solver* s, nds_iter_report* r) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->step(r); });
}
int nds_solve(nds_solver* s, nds_solve_report* r) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->solve(r); });
}
int nds_get_fields(nds_solver* s, double* u0, double* u1, double* u2, double* p) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->get_fields(u0, u1, u2, p); });
}
int nds_set_fields(nds_solver* s, const double* u0, const double* u1, const double* u2, const double* p) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->set_fields(u0, u1, u2, p); });
}
int nds_simple_step_io(nds_solver* s, const double* u0_in, const double* u1_in, const double* u2_in,
                       const double* p_in, double* u0_out, double* u1_out, double* u2_out, double* p_out,
                       nds_iter_report* r) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] {
    const double* in[4] = {u0_in, u1_in, u2_in, p_in};
    double* const out[4] = {u0_out, u1_out, u2_out, p_out};
    s->impl->step_io(in, out, r);
  });
}
void nds_solver_destroy(nds_solver* s) { delete s; }
int nds_solver_load_stage(nds_solver* s, const float* host_params, int count) {
  if (!s || !host_params || count != NDS_MPNN_NPARAM) return fail(NDS_E_INVALID, "nds_solver_load_stage: bad argument");
  return guarded([&] { s->impl->load_stage(host_params); });
}
int nds_solver_stage_graph(nds_solver* s, int32_t* nbr, float* ew, float* dscale) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->stage_graph(nbr, ew, dscale); });
}
int nds_solver_pressure_pair(nds_solver* s, float* rhs, float* x) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->pressure_pair(rhs, x); });
}
int nds_solver_apply_operator(nds_solver* s, const float* x, float* y) {
  if (!s || !x || !y) return fail(NDS_E_INVALID, "null argument");
  return guarded([&] { s->impl->apply_operator(x, y); });
}
int nds_solver_stage_counts(nds_solver* s, long long* applied, long long* fallbacks) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] { s->impl->stage_counts(applied, fallbacks); });
}

unsigned long long nds_launch_count(void) { return nds::g_launches; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free continuity residual.
//
// Callers that may not allocate device memory -- code running between the
// steps of its own captured or real-time loop, or under an allocator that
// forbids cudaMalloc after start-up -- get the continuity residual of the
// solver's mesh for velocity vectors they own.  The partial sums of the
// continuity kernel go to a file-scope device array instead of a cudaMalloc'd
// buffer: at most kNoAllocBlocks blocks (the same 8 x 148 cap as the solver's
// own reductions), 16 KiB per device.  Every block overwrites its own slot
// and the reduction reads only the slots written by the same call, so
// nothing has to start at zero.  The array is shared by all calls on a
// device: calls that overlap in time (two host threads, or two streams
// without ordering between them) race on it.
//
// The array's device address is looked up (cudaGetSymbolAddress) on every
// call with the solver's device current: the lookup allocates nothing, and
// an address kept from an earlier call could be stale once the caller has
// torn the context down (cudaDeviceReset) and the module was loaded again.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocBlocks = 1184;
constexpr int kNoAllocScratch = 2048;  // doubles; >= kNoAllocBlocks
static_assert(kNoAllocScratch >= kNoAllocBlocks, "scratch too small for the block cap");

__global__ void sqrt_in_place(double* x) { *x = sqrt(*x); }
}  // namespace

static __device__ __align__(256) double g_noalloc_part[kNoAllocScratch];

extern "C" {

int nds_continuity_noalloc(nds_solver* s, const double* u0, const double* u1, const double* u2, double* r,
                           double* norm, void* stream) {
  if (!s || !u0 || !u1 || !u2 || !r || !norm) return NDS_E_INVALID;
  const int32_t* ref = nullptr;
  const double *bco = nullptr, *fdiv = nullptr;
  int nc = 0, dev = 0;
  if (!s->impl->cell_arrays(&ref, &bco, &fdiv, &nc, &dev)) return NDS_E_INVALID;
  if (nc < 1 || dev < 0) return NDS_E_INVALID;
  const int grid = std::min(nds::grid_for(nc), kNoAllocBlocks);
  if (grid > kNoAllocScratch) return NDS_E_INVALID;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return NDS_E_CUDA;
  if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return NDS_E_CUDA;
  int st = NDS_OK;
  double* part = nullptr;
  {
    void* a = nullptr;
    if (cudaGetSymbolAddress(&a, g_noalloc_part) == cudaSuccess) part = static_cast<double*>(a);
    else st = NDS_E_CUDA;
  }
  // every launch is checked with cudaPeekAtLastError, which leaves an error
  // pending from the caller's own earlier work in place for the caller
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  if (st == NDS_OK) {
    nds::k::continuity<double, 1><<<grid, nds::kBlock, 0, cs>>>(nc, ref, bco, fdiv, u0, u1, u2, r, part);
    ++nds::g_launches;
    if (cudaPeekAtLastError() != cudaSuccess) st = NDS_E_CUDA;
  }
  if (st == NDS_OK) {
    nds::k::reduce_partials<1><<<1, nds::kBlock, 0, cs>>>(part, grid, norm);
    ++nds::g_launches;
    if (cudaPeekAtLastError() != cudaSuccess) st = NDS_E_CUDA;
  }
  if (st == NDS_OK) {
    sqrt_in_place<<<1, 1, 0, cs>>>(norm);
    ++nds::g_launches;
    if (cudaPeekAtLastError() != cudaSuccess) st = NDS_E_CUDA;
  }
  if (prev != dev) cudaSetDevice(prev);
  return st;
}

int nds_profile_enable(nds_solver* s, int on) {
  if (!s) return fail(NDS_E_INVALID, "null solver");
  return guarded([&] {
    s->impl->prof.collect();
    s->impl->prof.reset();
    s->impl->prof.on = on != 0;
  });
}
int nds_profile_read(nds_solver* s, nds_profile_entry* out, int max_entries, int* n_out) {
  if (!s || !out || !n_out) return fail(NDS_E_INVALID, "null argument");
  return guarded([&] {
    auto& P = s->impl->prof;
    P.collect();
    int n = 0;
    for (int c = 0; c < nds::P_NCAT && n < max_entries; ++c, ++n) {
      std::snprintf(out[n].name, sizeof(out[n].name), "%s", nds::kProfNames[c]);
      out[n].calls = P.calls[c];
      out[n].total_ms = P.total[c];
    }
    *n_out = n;
  });
}

}  // extern "C"
