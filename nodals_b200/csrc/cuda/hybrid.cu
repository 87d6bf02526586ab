// Mixed hex/tet Stokes gate on the GPU (the reference's HXT4A,
// gpu/serial_cuda/hybrid_hxt4a/hxt4a_main.cu:405-518): manufactured axial
// pressure p*, forcing f = B^T p*, and a SIMPLE loop of three Jacobi-PCG
// momentum solves with the Nitsche-coupled velocity operator A and one
// Jacobi-PCG solve of the Schur operator S = B diag(rAU) B^T per iteration.
//
// The operators come assembled from the host (csrc/host/hybrid.cpp); the
// device runs warp-per-row products of A, B and B^T (B^T as its own CSR, so
// no atomics), the vector updates and the block reductions.  Dots follow the
// reference's Reducer: at most 256 blocks of 256 threads, per-block partial
// sums, summed on the host in long double.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/nodals_b200.h"
#include "../host/fem.hpp"
#include "../host/hybrid.hpp"
#include "common.cuh"

namespace nds {
void set_error(const std::string& m);
namespace hy {

constexpr int kTPB = 256;

// 3-point Gauss rule on [-1,1]: nodes then weights
struct Rules3 {
  double v[6];
};
inline Rules3 rules3() {
  const double a = std::sqrt(0.6);
  return Rules3{{-a, 0.0, a, 5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0}};
}

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  Buf() = default;
  explicit Buf(const std::vector<T>& v) { upload(v); }
  explicit Buf(size_t m) {
    n = m;
    if (m) {
      NDS_CUDA(cudaMalloc((void**)&p, m * sizeof(T)));
      NDS_CUDA(cudaMemset(p, 0, m * sizeof(T)));
    }
  }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  ~Buf() {
    if (p) cudaFree(p);
  }
  void upload(const std::vector<T>& v) {
    n = v.size();
    if (n) {
      NDS_CUDA(cudaMalloc((void**)&p, n * sizeof(T)));
      NDS_CUDA(cudaMemcpy(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice));
    }
  }
};

// y = A x, one warp per row
__global__ void csr_mv(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  double s = 0;
  for (int k = row[i] + lane; k < row[i + 1]; k += 32) s += val[k] * x[col[k]];
  s = warp_sum(s);
  if (lane == 0) y[i] = s;
}
// y = B (u0, u1, u2) or, on the transposed rows, (v0, v1, v2) = B^T p
__global__ void b_mv(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                     const double* __restrict__ bx, const double* __restrict__ by, const double* __restrict__ bz,
                     const double* __restrict__ u0, const double* __restrict__ u1, const double* __restrict__ u2,
                     double* __restrict__ y) {
  const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  double s = 0;
  for (int k = row[i] + lane; k < row[i + 1]; k += 32) {
    const int g = col[k];
    s += bx[k] * u0[g] + by[k] * u1[g] + bz[k] * u2[g];
  }
  s = warp_sum(s);
  if (lane == 0) y[i] = s;
}
// sum over the L lanes of an aligned lane group; every lane of the warp calls it
template <int L>
__device__ __forceinline__ double group_sum(double v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// (v0, v1, v2) = B^T p: the transposed rows are short (a velocity unknown
// touches a few cells), so eight lanes take a row
constexpr int kBtLanes = 8;
__global__ void bt_mv(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                      const double* __restrict__ bx, const double* __restrict__ by, const double* __restrict__ bz,
                      const double* __restrict__ p, double* __restrict__ v0, double* __restrict__ v1,
                      double* __restrict__ v2) {
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int i = (int)(gt / kBtLanes), lane = (int)(gt % kBtLanes);
  const bool live = i < n;
  double s0 = 0, s1 = 0, s2 = 0;
  if (live)
    for (int k = row[i] + lane; k < row[i + 1]; k += kBtLanes) {
      const double q = p[col[k]];
      s0 += bx[k] * q;
      s1 += by[k] * q;
      s2 += bz[k] * q;
    }
  s0 = group_sum<kBtLanes>(s0);
  s1 = group_sum<kBtLanes>(s1);
  s2 = group_sum<kBtLanes>(s2);
  if (live && lane == 0) {
    v0[i] = s0;
    v1[i] = s1;
    v2[i] = s2;
  }
}
__global__ void scale3(int n, const double* __restrict__ r, double* v0, double* v1, double* v2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    v0[i] *= r[i];
    v1[i] *= r[i];
    v2[i] *= r[i];
  }
}
__global__ void set_at(int i, double v, double* x) {
  if (blockIdx.x == 0 && threadIdx.x == 0) x[i] = v;
}
__global__ void residual(int n, const double* b, const double* Ax, double* r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = b[i] - Ax[i];
}
__global__ void mul(int n, const double* a, const double* b, double* c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = a[i] * b[i];
}
__global__ void axpy2(int n, double a, const double* p, const double* q, double* x, double* r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    x[i] += a * p[i];
    r[i] -= a * q[i];
  }
}
__global__ void xpby(int n, double b, const double* z, double* p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = z[i] + b * p[i];
}
// rhs = fixed ? 0 : f - bt
__global__ void force_rhs(int n, const uint8_t* fixed, const double* f, const double* bt, double* rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rhs[i] = fixed[i] ? 0.0 : f[i] - bt[i];
}
__global__ void zero_fixed(int n, const uint8_t* fixed, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && fixed[i]) x[i] = 0.0;
}
__global__ void p_update(int n, int pin, double a, const double* dp, double* p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = (i == pin) ? 0.0 : p[i] + a * dp[i];
}
// d_i = sum_k rAU_col (bx^2 + by^2 + bz^2); 1 at the pin
__global__ void schur_diag_inv(int n, const int32_t* row, const int32_t* col, const double* bx, const double* by,
                               const double* bz, const double* rau, int pin, double* id) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i == pin) {
    id[i] = 1.0;
    return;
  }
  double s = 0;
  for (int k = row[i]; k < row[i + 1]; ++k) s += rau[col[k]] * (bx[k] * bx[k] + by[k] * by[k] + bz[k] * bz[k]);
  id[i] = 1.0 / s;
}
__global__ void dot_blocks(const double* x, const double* y, int n, double* out) {
  __shared__ double s[kTPB];
  const int t = threadIdx.x;
  double q = 0;
  for (int k = blockIdx.x * blockDim.x + t; k < n; k += gridDim.x * blockDim.x) q += x[k] * y[k];
  s[t] = q;
  __syncthreads();
  for (int d = kTPB / 2; d > 0; d >>= 1) {
    if (t < d) s[t] += s[t + d];
    __syncthreads();
  }
  if (t == 0) out[blockIdx.x] = s[0];
}

int grid(long long n, int per = kTPB) { return (int)std::max(1LL, (n + per - 1) / per); }

struct Reducer {
  int n, blocks;
  Buf<double> part;
  std::vector<double> host;
  explicit Reducer(int n_) : n(n_), blocks(std::max(1, std::min(256, (n_ + kTPB - 1) / kTPB))), part((size_t)blocks),
                             host((size_t)blocks) {}
  double dot(const double* x, const double* y) {
    dot_blocks<<<blocks, kTPB>>>(x, y, n, part.p);
    NDS_LAUNCH();
    NDS_CUDA(cudaMemcpy(host.data(), part.p, host.size() * sizeof(double), cudaMemcpyDeviceToHost));
    long double q = 0;
    for (double v : host) q += v;
    return (double)q;
  }
  double norm(const double* x) {
    const double q = dot(x, x);
    return std::isfinite(q) ? std::sqrt(std::max(0.0, q)) : NAN;
  }
};

struct Csr {
  int n;
  Buf<int32_t> row, col;
  Buf<double> val;
  Csr(int n_, const std::vector<int32_t>& r, const std::vector<int32_t>& c, const std::vector<double>& v)
      : n(n_), row(r), col(c), val(v) {}
  void apply(const double* x, double* y) {
    csr_mv<<<grid((long long)n * 32), kTPB>>>(n, row.p, col.p, val.p, x, y);
    NDS_LAUNCH();
  }
};
struct Div {
  int np, nv;
  Buf<int32_t> row, col, trow, tcol;
  Buf<double> bx, by, bz, tx, ty, tz;
  explicit Div(const HybridStokes& H)
      : np(H.np), nv(H.nvel), row(H.b_row), col(H.b_col), trow(H.bt_row), tcol(H.bt_col), bx(H.bx), by(H.by),
        bz(H.bz), tx(H.btx), ty(H.bty), tz(H.btz) {}
  void B(const double* u0, const double* u1, const double* u2, double* y) {
    b_mv<<<grid((long long)np * 32), kTPB>>>(np, row.p, col.p, bx.p, by.p, bz.p, u0, u1, u2, y);
    NDS_LAUNCH();
  }
  void BT(const double* p, double* v0, double* v1, double* v2) {
    bt_mv<<<grid((long long)nv * kBtLanes), kTPB>>>(nv, trow.p, tcol.p, tx.p, ty.p, tz.p, p, v0, v1, v2);
    NDS_LAUNCH();
  }
};
// S x = B diag(rAU) B^T x with the pin row zeroed
struct Schur {
  Div& D;
  const double* rau;
  int pin;
  Buf<double> v0, v1, v2;
  Schur(Div& d, const double* r, int p) : D(d), rau(r), pin(p), v0((size_t)d.nv), v1((size_t)d.nv), v2((size_t)d.nv) {}
  void apply(const double* x, double* y) {
    D.BT(x, v0.p, v1.p, v2.p);
    scale3<<<grid(D.nv), kTPB>>>(D.nv, rau, v0.p, v1.p, v2.p);
    NDS_LAUNCH();
    D.B(v0.p, v1.p, v2.p, y);
    set_at<<<1, 1>>>(pin, 0.0, y);
    NDS_LAUNCH();
  }
};
// ---- CG with its iteration loop on the device.  This file is compiled with
// the per-thread default stream, so every launch below can be captured: the
// loop is one graph whose conditional while node runs one iteration per
// pass, with the scalars (rho, alpha, beta, ||r||) kept on the device and
// each partial-sum vector reduced by one block in a fixed order.  Per solve
// the host waits twice (initial norm, final state) instead of three times
// per iteration.
enum { CG_RHO = 0, CG_BETA = 1, CG_ALPHA = 2, CG_RN = 3, CG_TARGET = 4 };
enum { CG_ITS = 0, CG_CONV = 1, CG_FIRST = 2, CG_MAXIT = 3, CG_FLAGS = 4 };
// flags: 1 pAp nonpositive, 2 rho nonpositive, 4 residual not finite, 8 initial rho nonpositive

__device__ double sum_partials(const double* __restrict__ part, int nb) {
  double s = 0;
  for (int k = 0; k < nb; ++k) s += part[k];
  return s;
}
// rho = r.z: the first pass takes it as the initial rho, later passes form beta
__global__ void cg_rho(const double* __restrict__ part, int nb, double* __restrict__ sc, int* __restrict__ ctl) {
  const double nr = sum_partials(part, nb);
  const bool bad = !(nr > 0) || !isfinite(nr);
  if (ctl[CG_FIRST]) {
    if (bad) ctl[CG_FLAGS] |= 8;
    sc[CG_BETA] = 0;
  } else {
    if (bad) ctl[CG_FLAGS] |= 2;
    sc[CG_BETA] = bad ? 0.0 : nr / sc[CG_RHO];
  }
  sc[CG_RHO] = nr;
}
// p = z on the first pass, else z + beta p; zero at the pin
__global__ void cg_p(int n, const double* __restrict__ sc, const int* __restrict__ ctl, const double* __restrict__ z,
                     double* __restrict__ p, int pin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  p[i] = i == pin ? 0.0 : (ctl[CG_FIRST] ? z[i] : z[i] + sc[CG_BETA] * p[i]);
}
__global__ void cg_alpha(const double* __restrict__ part, int nb, double* __restrict__ sc, int* __restrict__ ctl) {
  const double pq = sum_partials(part, nb);
  ctl[CG_FIRST] = 0;
  if (!(pq > 0) || !isfinite(pq)) {
    ctl[CG_FLAGS] |= 1;
    sc[CG_ALPHA] = 0;
  } else {
    sc[CG_ALPHA] = sc[CG_RHO] / pq;
  }
}
__global__ void cg_xr(int n, const double* __restrict__ sc, const double* __restrict__ p, const double* __restrict__ q,
                      double* __restrict__ x, double* __restrict__ r, int pin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double a = sc[CG_ALPHA];
  x[i] = i == pin ? 0.0 : x[i] + a * p[i];
  r[i] = i == pin ? 0.0 : r[i] - a * q[i];
}
// end of a pass: ||r||, the iteration count and the stopping test; the loop
// always ends, at the latest when the count reaches max_it
__global__ void cg_check(const double* __restrict__ part, int nb, double* __restrict__ sc, int* __restrict__ ctl,
                         cudaGraphConditionalHandle loop) {
  const double q = sum_partials(part, nb);
  const double rn = isfinite(q) ? sqrt(fmax(0.0, q)) : NAN;
  const int it = ++ctl[CG_ITS];
  sc[CG_RN] = rn;
  if (!isfinite(rn)) ctl[CG_FLAGS] |= 4;
  const int conv = rn <= sc[CG_TARGET];
  ctl[CG_CONV] = conv;
  cudaGraphSetConditional(loop, (conv || ctl[CG_FLAGS] != 0 || it >= ctl[CG_MAXIT]) ? 0u : 1u);
}
// z = r / d with zero at the pin
__global__ void cg_jacobi(int n, const double* __restrict__ inv, const double* __restrict__ r, double* __restrict__ z,
                          int pin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = i == pin ? 0.0 : inv[i] * r[i];
}

// The captured loop body bakes in x, the pin, the operator's buffers and the
// preconditioner's buffers (its closure).  It is rebuilt when x, the pin or
// the operator object changes; the preconditioner is not compared, so every
// CgWork serves one (operator, preconditioner) pair for its whole life (each
// solve site of this file owns its own CgWork).
struct CgLoop {
  cudaGraphExec_t exec = nullptr;
  const void* bound = nullptr;     // x of the captured body
  const void* bound_op = nullptr;  // operator object of the captured body
  int bound_pin = -2;
  unsigned long long body_kernels = 0;
  bool failed = false;
  CgLoop() = default;
  CgLoop(const CgLoop&) = delete;
  ~CgLoop() {
    if (exec) cudaGraphExecDestroy(exec);
  }
};
struct CgWork {
  int n;
  Buf<double> r, z, p, q, sc;
  Buf<int> ctl;
  Reducer red;
  CgLoop loop;
  double* hsc = nullptr;
  int* hctl = nullptr;
  explicit CgWork(int n_)
      : n(n_), r((size_t)n_), z((size_t)n_), p((size_t)n_), q((size_t)n_), sc((size_t)8), ctl((size_t)8), red(n_) {
    NDS_CUDA(cudaMallocHost((void**)&hsc, 8 * sizeof(double)));
    NDS_CUDA(cudaMallocHost((void**)&hctl, 8 * sizeof(int)));
  }
  CgWork(const CgWork&) = delete;
  ~CgWork() {
    if (hsc) cudaFreeHost(hsc);
    if (hctl) cudaFreeHost(hctl);
  }
};
struct CgResult {
  int its = 0;
  double rel = 1;
  bool ok = false;
};
bool hybrid_graphs_enabled() {
  static const bool on = std::getenv("NDS_NO_GRAPHS") == nullptr;
  return on;
}

// Preconditioned CG on the device from the guess in x: r = rhs - A x (zero at
// pin, pin < 0 for none), r0 = ||r||; returns at once when r0 <= floor, else
// iterates to ||r|| <= max(atol, rtol r0) within maxit.  pre(r, z) applies
// the preconditioner (zero at the pin included).  Arithmetic and stopping
// rule as the host loops below; false when the graph could not be built.
template <class Op, class Pre>
bool cg_device(Op& A, Pre&& pre, const double* rhs, double* x, double rtol, double atol, double floor, int maxit,
               CgWork& W, int pin, CgResult& R) {
  CgLoop& L = W.loop;
  if (!hybrid_graphs_enabled() || L.failed) return false;
  const int n = W.n, nb = W.red.blocks;
  A.apply(x, W.q.p);
  residual<<<grid(n), kTPB>>>(n, rhs, W.q.p, W.r.p);
  NDS_LAUNCH();
  if (pin >= 0) set_at<<<1, 1>>>(pin, 0.0, W.r.p);
  const double r0 = W.red.norm(W.r.p);
  if (!std::isfinite(r0)) throw std::runtime_error("mixed-mesh CG: initial residual not finite");
  R = CgResult{};
  if (r0 <= floor) {
    R.rel = 0;
    R.ok = true;
    return true;
  }
  if (L.exec && (L.bound != x || L.bound_op != (const void*)&A || L.bound_pin != pin)) {
    cudaGraphExecDestroy(L.exec);
    L.exec = nullptr;
  }
  if (!L.exec) {
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
    if (ok)
      ok = cudaStreamBeginCaptureToGraph(cudaStreamPerThread, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      bool body_ok = true;
      try {
        pre(W.r.p, W.z.p);
        dot_blocks<<<nb, kTPB>>>(W.r.p, W.z.p, n, W.red.part.p);
        cg_rho<<<1, 1>>>(W.red.part.p, nb, W.sc.p, W.ctl.p);
        cg_p<<<grid(n), kTPB>>>(n, W.sc.p, W.ctl.p, W.z.p, W.p.p, pin);
        A.apply(W.p.p, W.q.p);
        dot_blocks<<<nb, kTPB>>>(W.p.p, W.q.p, n, W.red.part.p);
        cg_alpha<<<1, 1>>>(W.red.part.p, nb, W.sc.p, W.ctl.p);
        cg_xr<<<grid(n), kTPB>>>(n, W.sc.p, W.p.p, W.q.p, x, W.r.p, pin);
        dot_blocks<<<nb, kTPB>>>(W.r.p, W.r.p, n, W.red.part.p);
        cg_check<<<1, 1>>>(W.red.part.p, nb, W.sc.p, W.ctl.p, h);
        g_launches += 8;
        body_ok = cudaGetLastError() == cudaSuccess;
      } catch (...) {
        body_ok = false;
      }
      cudaGraph_t captured = nullptr;
      ok = cudaStreamEndCapture(cudaStreamPerThread, &captured) == cudaSuccess && body_ok;
    }
    L.body_kernels = g_launches - l0;
    g_launches = l0;
    if (ok) ok = cudaGraphInstantiate(&L.exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    if (!ok) {
      if (L.exec) cudaGraphExecDestroy(L.exec);
      L.exec = nullptr;
      L.failed = true;
      cudaGetLastError();
      return false;
    }
    L.bound = x;
    L.bound_op = (const void*)&A;
    L.bound_pin = pin;
  }
  W.hsc[CG_TARGET] = std::max(atol, rtol * r0);
  const int init[5] = {0, 0, 1, maxit, 0};
  std::memcpy(W.hctl, init, sizeof(init));
  NDS_CUDA(cudaMemcpyAsync(W.sc.p + CG_TARGET, W.hsc + CG_TARGET, sizeof(double), cudaMemcpyHostToDevice,
                           cudaStreamPerThread));
  NDS_CUDA(cudaMemcpyAsync(W.ctl.p, W.hctl, 5 * sizeof(int), cudaMemcpyHostToDevice, cudaStreamPerThread));
  NDS_CUDA(cudaGraphLaunch(L.exec, cudaStreamPerThread));
  NDS_CUDA(cudaMemcpyAsync(W.hctl, W.ctl.p, 5 * sizeof(int), cudaMemcpyDeviceToHost, cudaStreamPerThread));
  NDS_CUDA(cudaMemcpyAsync(W.hsc + CG_RN, W.sc.p + CG_RN, sizeof(double), cudaMemcpyDeviceToHost, cudaStreamPerThread));
  NDS_CUDA(cudaStreamSynchronize(cudaStreamPerThread));
  const int f = W.hctl[CG_FLAGS];
  g_launches += (unsigned long long)W.hctl[CG_ITS] * L.body_kernels;
  if (f & 8) throw std::runtime_error("mixed-mesh CG: initial rho nonpositive");
  if (f & 1) throw std::runtime_error("mixed-mesh CG: pAp nonpositive");
  if (f & 2) throw std::runtime_error("mixed-mesh CG: rho nonpositive");
  if (f & 4) throw std::runtime_error("mixed-mesh CG: residual not finite");
  R.its = W.hctl[CG_ITS];
  R.rel = W.hsc[CG_RN] / r0;
  R.ok = W.hctl[CG_CONV] != 0;
  return true;
}
// Jacobi-preconditioned CG to ||r|| <= rtol ||r0|| from the guess in x
// (hybrid_hxt4a/hxt4a_main.cu:309-326; pin >= 0 keeps x, r, p zero there)
template <class Op>
CgResult cg(Op& A, const double* rhs, double* x, const double* invdiag, double rtol, int maxit, CgWork& W,
            int pin = -1) {
  const int n = W.n;
  {
    CgResult D;
    auto jac = [&](const double* r, double* z) {
      cg_jacobi<<<grid(n), kTPB>>>(n, invdiag, r, z, pin);
      NDS_LAUNCH();
    };
    if (cg_device(A, jac, rhs, x, rtol, 0.0, 0.0, maxit, W, pin, D)) return D;
  }
  A.apply(x, W.q.p);
  residual<<<grid(n), kTPB>>>(n, rhs, W.q.p, W.r.p);
  NDS_LAUNCH();
  if (pin >= 0) set_at<<<1, 1>>>(pin, 0.0, W.r.p);
  const double r0 = W.red.norm(W.r.p);
  if (!std::isfinite(r0)) throw std::runtime_error("hybrid CG initial residual nonfinite");
  if (r0 == 0) return {0, 0, true};
  mul<<<grid(n), kTPB>>>(n, invdiag, W.r.p, W.z.p);
  NDS_LAUNCH();
  NDS_CUDA(cudaMemcpy(W.p.p, W.z.p, n * sizeof(double), cudaMemcpyDeviceToDevice));
  double rho = W.red.dot(W.r.p, W.z.p);
  if (!(rho > 0)) throw std::runtime_error("hybrid CG initial rho nonpositive");
  CgResult R;
  const double target = rtol * r0;
  for (int k = 0; k < maxit; ++k) {
    A.apply(W.p.p, W.q.p);
    const double pq = W.red.dot(W.p.p, W.q.p);
    if (!(pq > 0) || !std::isfinite(pq)) throw std::runtime_error("hybrid CG pAp nonpositive");
    axpy2<<<grid(n), kTPB>>>(n, rho / pq, W.p.p, W.q.p, x, W.r.p);
    NDS_LAUNCH();
    if (pin >= 0) {
      set_at<<<1, 1>>>(pin, 0.0, x);
      set_at<<<1, 1>>>(pin, 0.0, W.r.p);
    }
    const double rn = W.red.norm(W.r.p);
    R.its = k + 1;
    R.rel = rn / r0;
    if (rn <= target) {
      R.ok = true;
      break;
    }
    mul<<<grid(n), kTPB>>>(n, invdiag, W.r.p, W.z.p);
    NDS_LAUNCH();
    const double nr = W.red.dot(W.r.p, W.z.p);
    if (!(nr > 0)) throw std::runtime_error("hybrid CG rho nonpositive");
    xpby<<<grid(n), kTPB>>>(n, nr / rho, W.z.p, W.p.p);
    NDS_LAUNCH();
    if (pin >= 0) set_at<<<1, 1>>>(pin, 0.0, W.p.p);
    rho = nr;
  }
  return R;
}

double rel_l2(const std::vector<double>& a, const std::vector<double>& b) {
  long double n = 0, d = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    const long double q = a[i] - b[i];
    n += q * q;
    d += (long double)b[i] * b[i];
  }
  return std::sqrt((double)n / std::max((double)d, 1e-300));
}

void run_gate(const char* path, double nu, double gamma, double rau_scale, double alpha_p, double simple_tol,
              int max_outer, int verbose, nds_hybrid_report* out) {
  const HybridMesh M = read_hxt1_hybrid(path);
  const auto P = interface_plans(M);
  const HybridStokes H = build_hybrid_stokes(M, P, nu, gamma);
  const int nv = H.nvel, np = H.np, pin = 0;
  // diagonals: full for the momentum preconditioner, penalty-free for rAU
  std::vector<double> idf((size_t)nv), rau((size_t)nv);
  for (int i = 0; i < nv; ++i) {
    if (H.fixed[(size_t)i]) {
      idf[(size_t)i] = 1.0;
      rau[(size_t)i] = 0.0;
      continue;
    }
    const double a = H.diag_full[(size_t)i], b = H.diag_rau[(size_t)i];
    if (!(a > 0) || !(b > 0) || !std::isfinite(a) || !std::isfinite(b))
      throw std::runtime_error("hybrid gate: nonpositive diagonal at unknown " + std::to_string(i));
    idf[(size_t)i] = 1.0 / a;
    rau[(size_t)i] = rau_scale / b;
  }
  Csr A(nv, H.a_row, H.a_col, H.a_val);
  Div B(H);
  Buf<double> d_idf(idf), d_rau(rau), d_isd((size_t)np);
  Buf<uint8_t> d_fixed(H.fixed);
  schur_diag_inv<<<grid(np), kTPB>>>(np, B.row.p, B.col.p, B.bx.p, B.by.p, B.bz.p, d_rau.p, pin, d_isd.p);
  NDS_LAUNCH();
  Schur S(B, d_rau.p, pin);
  Reducer ured(nv), pred(np);
  // operator audit on fixed deterministic vectors (hxt4a_main.cu:430-437)
  std::vector<double> ha((size_t)nv), hb0((size_t)nv), hb1((size_t)nv), hb2((size_t)nv), hp((size_t)np);
  for (int g = 0; g < nv; ++g) {
    const double q = g + 1;
    ha[(size_t)g] = std::sin(0.00113 * q);
    hb0[(size_t)g] = std::cos(.00131 * q);
    hb1[(size_t)g] = std::sin(.00091 * q + .2);
    hb2[(size_t)g] = std::cos(.00157 * q - .1);
  }
  for (int i = 0; i < np; ++i) hp[(size_t)i] = std::sin(.00107 * (i + 1));
  Buf<double> da(ha), dAr((size_t)nv), db0(hb0), db1(hb1), db2(hb2), dBr((size_t)np), dpa(hp), dSr((size_t)np);
  A.apply(da.p, dAr.p);
  B.B(db0.p, db1.p, db2.p, dBr.p);
  S.apply(dpa.p, dSr.p);
  const double a_norm = ured.norm(dAr.p), b_norm = pred.norm(dBr.p), s_norm = pred.norm(dSr.p);
  // forcing f = B^T p*, zero on fixed rows
  Buf<double> d_pex(H.p_exact), f0((size_t)nv), f1((size_t)nv), f2((size_t)nv);
  B.BT(d_pex.p, f0.p, f1.p, f2.p);
  for (double* f : {f0.p, f1.p, f2.p}) {
    zero_fixed<<<grid(nv), kTPB>>>(nv, d_fixed.p, f);
    NDS_LAUNCH();
  }
  Buf<double> u0((size_t)nv), u1((size_t)nv), u2((size_t)nv), p((size_t)np), dp((size_t)np), cont((size_t)np);
  Buf<double> bt0((size_t)nv), bt1((size_t)nv), bt2((size_t)nv), r0((size_t)nv), r1((size_t)nv), r2((size_t)nv);
  CgWork W0(nv), W1(nv), W2(nv), WP(np);
  const double m_rtol = 1e-10, p_rtol = 1e-10;
  if (verbose) {
    std::printf("NODALS_HXT4A_CONFIG precision=fp64 scalarBytes=8 geometry=fp64 reductions=fp64 stateOperator=fp64 "
                "gamma=%.6f rauScale=%.6f alphaP=%.6f simpleTol=%.3e pressureSolver=PCG_JACOBI status=PASS\n",
                gamma, rau_scale, alpha_p, simple_tol);
    std::printf("NODALS_HXT4A_OPERATOR_AUDIT precision=fp64 Anorm=%.12e Bnorm=%.12e Snorm=%.12e status=PASS\n", a_norm,
                b_norm, s_norm);
  }
  const auto t0 = std::chrono::steady_clock::now();
  double cont0 = -1, first_u = -1, final_rel = 1;
  int outer = 0;
  long long mcg = 0, pcg = 0;
  bool conv = false;
  auto momentum = [&](CgResult* m) {
    B.BT(p.p, bt0.p, bt1.p, bt2.p);
    force_rhs<<<grid(nv), kTPB>>>(nv, d_fixed.p, f0.p, bt0.p, r0.p);
    force_rhs<<<grid(nv), kTPB>>>(nv, d_fixed.p, f1.p, bt1.p, r1.p);
    force_rhs<<<grid(nv), kTPB>>>(nv, d_fixed.p, f2.p, bt2.p, r2.p);
    NDS_LAUNCH();
    m[0] = cg(A, r0.p, u0.p, d_idf.p, m_rtol, 2500, W0);
    m[1] = cg(A, r1.p, u1.p, d_idf.p, m_rtol, 2500, W1);
    m[2] = cg(A, r2.p, u2.p, d_idf.p, m_rtol, 2500, W2);
    if (!(m[0].ok && m[1].ok && m[2].ok)) throw std::runtime_error("hybrid gate: momentum CG failed");
  };
  for (int it = 1; it <= max_outer; ++it) {
    CgResult m[3];
    momentum(m);
    mcg += m[0].its + m[1].its + m[2].its;
    B.B(u0.p, u1.p, u2.p, cont.p);
    set_at<<<1, 1>>>(pin, 0.0, cont.p);
    NDS_LAUNCH();
    const double cn = pred.norm(cont.p);
    if (it == 1) cont0 = cn;
    final_rel = cn / std::max(cont0, 1e-300);
    const double un = std::sqrt(ured.dot(u0.p, u0.p) + ured.dot(u1.p, u1.p) + ured.dot(u2.p, u2.p));
    if (it == 1) first_u = un;
    NDS_CUDA(cudaMemset(dp.p, 0, np * sizeof(double)));
    const CgResult pr = cg(S, cont.p, dp.p, d_isd.p, p_rtol, 2500, WP, pin);
    if (!pr.ok) throw std::runtime_error("hybrid gate: pressure CG failed");
    pcg += pr.its;
    p_update<<<grid(np), kTPB>>>(np, pin, alpha_p, dp.p, p.p);
    NDS_LAUNCH();
    outer = it;
    conv = it > 1 && final_rel <= simple_tol;
    if (verbose && (it <= 5 || it % 20 == 0 || conv))
      std::printf("NODALS_HXT4A_SIMPLE precision=fp64 it=%d relCont=%.12e velocityNorm=%.12e mCG=[%d,%d,%d] pCG=%d "
                  "converged=%d status=PASS\n",
                  it, final_rel, un, m[0].its, m[1].its, m[2].its, pr.its, (int)conv);
    if (conv) break;
  }
  if (!conv) throw std::runtime_error("hybrid gate: no convergence within max_outer");
  // final predictor at the final pressure
  CgResult fm[3];
  momentum(fm);
  B.B(u0.p, u1.p, u2.p, cont.p);
  set_at<<<1, 1>>>(pin, 0.0, cont.p);
  NDS_LAUNCH();
  const double final_c = pred.norm(cont.p), final_cr = final_c / std::max(cont0, 1e-300);
  const double final_u = std::sqrt(ured.dot(u0.p, u0.p) + ured.dot(u1.p, u1.p) + ured.dot(u2.p, u2.p));
  const double loop_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::vector<double> pf((size_t)np);
  NDS_CUDA(cudaMemcpy(pf.data(), p.p, np * sizeof(double), cudaMemcpyDeviceToHost));
  nds_hybrid_report R{};
  R.outer_its = outer;
  R.converged = 1;
  R.final_rel_cont = final_cr;
  R.pressure_rel_l2 = rel_l2(pf, H.p_exact);
  R.slope = hybrid_pressure_slope(M, pf);
  R.slope_exact = hybrid_pressure_slope(M, H.p_exact);
  R.delta = hybrid_boundary_pressure(M, pf, false) - hybrid_boundary_pressure(M, pf, true);
  R.delta_exact = hybrid_boundary_pressure(M, H.p_exact, false) - hybrid_boundary_pressure(M, H.p_exact, true);
  R.velocity_rel = final_u / std::max(first_u, 1e-300);
  R.avg_momentum_cg = outer ? (double)mcg / (3.0 * outer) : 0.0;
  R.avg_pressure_cg = outer ? (double)pcg / outer : 0.0;
  R.a_norm = a_norm;
  R.b_norm = b_norm;
  R.s_norm = s_norm;
  R.loop_ms = loop_ms;
  R.pass = final_cr <= 1.2e-3 && R.velocity_rel < 5e-4 && std::abs(R.slope - R.slope_exact) / std::abs(R.slope_exact) < 5e-3 &&
           std::abs(R.delta - R.delta_exact) / std::abs(R.delta_exact) < 5e-3;
  R.n_hex = M.nhex();
  R.n_tet = M.ntet();
  R.n_interface = (int)P.size();
  R.n_velocity = nv;
  if (verbose)
    std::printf("NODALS_HXT4A_RESULT precision=fp64 outer=%d finalRelCont=%.12e pressureRelL2=%.12e slope=%.12e "
                "slopeExact=%.12e delta=%.12e deltaExact=%.12e velocityRel=%.12e avgMomentumCG=%.6f avgPressureCG=%.6f "
                "Anorm=%.12e Bnorm=%.12e Snorm=%.12e status=%s\n",
                R.outer_its, R.final_rel_cont, R.pressure_rel_l2, R.slope, R.slope_exact, R.delta, R.delta_exact,
                R.velocity_rel, R.avg_momentum_cg, R.avg_pressure_cg, R.a_norm, R.b_norm, R.s_norm,
                R.pass ? "PASS" : "FAIL");
  if (out) *out = R;
}

// ===================================================================
// Mixed-mesh pipe SIMPLE (the reference's HXT4B,
// gpu/serial_cuda/hybrid_hxt4b/hxt4b_main.cu:211-268)
// ===================================================================
__constant__ double c_g3[6];                   // 3-point Gauss nodes, then weights
__constant__ double c_tet_conv[8 * 8 * 8 * 3];  // T[a][m][b][j] = int phi_a phi_m dphi_b/dxi_j
__constant__ int c_hex_sign[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                     {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

// Q1 + BF2 basis (values, reference gradients) at (x, y, z) in [-1,1]^3
__device__ void hex_basis_dev(double x, double y, double z, double phi[14], double g[14][3]) {
  for (int a = 0; a < 8; ++a) {
    const double sx = c_hex_sign[a][0], sy = c_hex_sign[a][1], sz = c_hex_sign[a][2];
    const double ax = 1.0 + sx * x, ay = 1.0 + sy * y, az = 1.0 + sz * z;
    phi[a] = 0.125 * ax * ay * az;
    g[a][0] = 0.125 * sx * ay * az;
    g[a][1] = 0.125 * sy * ax * az;
    g[a][2] = 0.125 * sz * ax * ay;
  }
  const double c[3] = {x, y, z}, b[3] = {1 - x * x, 1 - y * y, 1 - z * z}, d[3] = {-2 * x, -2 * y, -2 * z};
  const int nrm[6] = {2, 2, 1, 0, 1, 0};
  const double sgn[6] = {-1, 1, -1, 1, 1, -1};
  for (int f = 0; f < 6; ++f) {
    const int n = nrm[f], t1 = n == 0 ? 1 : 0, t2 = n == 2 ? 1 : 2;
    const double s = 0.5 * (1.0 + sgn[f] * c[n]);
    phi[8 + f] = s * b[t1] * b[t2];
    g[8 + f][n] = 0.5 * sgn[f] * b[t1] * b[t2];
    g[8 + f][t1] = s * d[t1] * b[t2];
    g[8 + f][t2] = s * b[t1] * d[t2];
  }
}

// Convection block of each hex at the lagged velocity:
// C_ab = sum_q det w phi_a (u_q . grad phi_b), u_q = sum_m u_m phi_m(q), 27 points.
// Persistent blocks walk the hexes.  Each block first copies the basis
// values and reference gradients at the 27 points into shared memory (the
// same for every hex); per hex, 27 threads build the metric of their point
// and the velocity there, all threads then form, per (point, function),
// det w phi and u . grad phi, and finally the 196 entries, summed over the
// points in order.
struct HexConvShared {
  double phi[27][14], gref[27][14][3], inv[27][9], dw[27], u[27][3], ul[3][14], v[8][3];
  double dwphi[27][14], ugrad[27][14];  // det w phi_a and u_q . grad phi_b at each point
};
// basis values and reference gradients at the 27 points: tab[q][a][0] = phi,
// tab[q][a][1..3] = gradient (filled once per run)
__global__ void hex_point_table(double* __restrict__ tab) {
  const int t = threadIdx.x;
  if (t >= 27) return;
  const int ix = t / 9, iy = (t / 3) % 3, iz = t % 3;
  double ph[14], g[14][3];
  hex_basis_dev(c_g3[ix], c_g3[iy], c_g3[iz], ph, g);
  for (int a = 0; a < 14; ++a) {
    double* o = tab + (t * 14 + a) * 4;
    o[0] = ph[a];
    for (int d = 0; d < 3; ++d) o[1 + d] = g[a][d];
  }
}
__global__ void __launch_bounds__(kTPB) hex_conv_local(int nh, const double* __restrict__ xyz,
                                                        const int32_t* __restrict__ hexes,
                                                        const int32_t* __restrict__ dofs, const double* __restrict__ u0,
                                                        const double* __restrict__ u1, const double* __restrict__ u2,
                                                        const double* __restrict__ tab, double* __restrict__ local,
                                                        int* __restrict__ bad) {
  __shared__ HexConvShared S;
  const int t = threadIdx.x;
  for (int k = t; k < 27 * 14; k += blockDim.x) {
    const int q = k / 14, a = k % 14;
    S.phi[q][a] = tab[4 * k];
    for (int d = 0; d < 3; ++d) S.gref[q][a][d] = tab[4 * k + 1 + d];
  }
  for (int c = blockIdx.x; c < nh; c += gridDim.x) {
    __syncthreads();  // the previous hex's entries are written; tables are ready
    if (t < 14) {
      const int g = dofs[14 * (size_t)c + t];
      S.ul[0][t] = u0[g];
      S.ul[1][t] = u1[g];
      S.ul[2][t] = u2[g];
    } else if (t >= 32 && t < 56) {
      const int a = (t - 32) / 3, i = (t - 32) % 3;
      S.v[a][i] = xyz[3 * (size_t)hexes[8 * (size_t)c + a] + i];
    }
    __syncthreads();
    if (t < 27) {
      const int ix = t / 9, iy = (t / 3) % 3, iz = t % 3;
      const double w = c_g3[3 + ix] * c_g3[3 + iy] * c_g3[3 + iz];
      double J[9] = {};
      for (int a = 0; a < 8; ++a)
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[3 * i + j] += S.v[a][i] * S.gref[t][a][j];
      const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
      if (!(det > 0)) atomicAdd(bad, 1);
      const double q = 1.0 / det;
      S.inv[t][0] = (J[4] * J[8] - J[5] * J[7]) * q;
      S.inv[t][1] = (J[2] * J[7] - J[1] * J[8]) * q;
      S.inv[t][2] = (J[1] * J[5] - J[2] * J[4]) * q;
      S.inv[t][3] = (J[5] * J[6] - J[3] * J[8]) * q;
      S.inv[t][4] = (J[0] * J[8] - J[2] * J[6]) * q;
      S.inv[t][5] = (J[2] * J[3] - J[0] * J[5]) * q;
      S.inv[t][6] = (J[3] * J[7] - J[4] * J[6]) * q;
      S.inv[t][7] = (J[1] * J[6] - J[0] * J[7]) * q;
      S.inv[t][8] = (J[0] * J[4] - J[1] * J[3]) * q;
      S.dw[t] = det * w;
      double uq[3] = {0, 0, 0};
      for (int a = 0; a < 14; ++a)
        for (int d = 0; d < 3; ++d) uq[d] += S.ul[d][a] * S.phi[t][a];
      for (int d = 0; d < 3; ++d) S.u[t][d] = uq[d];
    }
    __syncthreads();
    for (int e = t; e < 27 * 14; e += blockDim.x) {
      const int q = e / 14, a = e % 14;
      const double* g = S.gref[q][a];
      const double* I = S.inv[q];
      double gp[3];
      for (int d = 0; d < 3; ++d) gp[d] = g[0] * I[d] + g[1] * I[3 + d] + g[2] * I[6 + d];
      S.ugrad[q][a] = S.u[q][0] * gp[0] + S.u[q][1] * gp[1] + S.u[q][2] * gp[2];
      S.dwphi[q][a] = S.dw[q] * S.phi[q][a];
    }
    __syncthreads();
    for (int e = t; e < 196; e += blockDim.x) {
      const int a = e / 14, b = e % 14;
      double s = 0;
      for (int q = 0; q < 27; ++q) s += S.dwphi[q][a] * S.ugrad[q][b];
      local[196 * (size_t)c + e] = s;
    }
  }
}
// Convection block of each tet: C_ab = det sum_m sum_j (J^-1 u_m)_j T[a][m][b][j].
// Persistent blocks of 256 threads take four tets at a time (64 threads
// each, one per entry); the tensor is staged once per block in shared memory
// as [m][j][a][b], so a warp's 32 entries read 32 consecutive values.
__global__ void __launch_bounds__(kTPB) tet_conv_local(int nt, const double* __restrict__ geom,
                                                        const int32_t* __restrict__ dofs,
                                                        const double* __restrict__ u0, const double* __restrict__ u1,
                                                        const double* __restrict__ u2, double* __restrict__ local) {
  __shared__ double T[8 * 3 * 64];
  __shared__ double ur[4][8][3];
  const int t = threadIdx.x, slot = t / 64, e = t % 64, a = e / 8, b = e % 8;
  for (int k = t; k < 8 * 3 * 64; k += blockDim.x) {
    const int mj = k / 64, ab = k % 64, m = mj / 3, j = mj % 3, aa = ab / 8, bb = ab % 8;
    T[k] = c_tet_conv[((aa * 8 + m) * 8 + bb) * 3 + j];
  }
  for (int c0 = 4 * blockIdx.x; c0 < nt; c0 += 4 * gridDim.x) {
    const int c = c0 + slot;
    __syncthreads();  // T staged; the previous tets' velocities are no longer read
    if (c < nt && e < 8) {
      const double* G = geom + 12 * (size_t)c;
      const int g = dofs[8 * (size_t)c + e];
      const double u[3] = {u0[g], u1[g], u2[g]};
      for (int j = 0; j < 3; ++j) ur[slot][e][j] = u[0] * G[3 + 3 * j] + u[1] * G[4 + 3 * j] + u[2] * G[5 + 3 * j];
    }
    __syncthreads();
    if (c < nt) {
      double q = 0;
      for (int m = 0; m < 8; ++m)
        for (int j = 0; j < 3; ++j) q += ur[slot][m][j] * T[(m * 3 + j) * 64 + a * 8 + b];
      local[64 * (size_t)c + e] = q * geom[12 * (size_t)c + 2];
    }
  }
}
// conv[k] = sum of its cells' local values, in cell order
__global__ void conv_gather(int nnz, const int32_t* __restrict__ off, const int32_t* __restrict__ src,
                            const double* __restrict__ local, double* __restrict__ conv) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  double s = 0;
  for (int q = off[k]; q < off[k + 1]; ++q) s += local[src[q]];
  conv[k] = s;
}
// val = base + conv; relaxed diagonal val_ii / alpha_u; rAU = scale alpha_u / (penalty-free diag + conv_ii)
__global__ void flow_rows(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ dpos,
                          const uint8_t* __restrict__ fixed, const double* __restrict__ base,
                          const double* __restrict__ conv, const double* __restrict__ dr, double alpha_u,
                          double rau_scale, double* __restrict__ val, double* __restrict__ dorig,
                          double* __restrict__ rau, int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = row[i]; k < row[i + 1]; ++k) val[k] = base[k] + conv[k];
  const int d = dpos[i];
  const double orig = val[d];
  dorig[i] = orig;
  if (fixed[i]) {
    rau[i] = 0.0;
    return;
  }
  const double den = dr[i] + conv[d];
  if (!(orig > 0) || !(den > 0) || !isfinite(orig) || !isfinite(den)) {
    atomicAdd(bad, 1);
    rau[i] = 0.0;
    return;
  }
  val[d] = orig / alpha_u;
  rau[i] = rau_scale * alpha_u / den;
}
// rhs = fixed ? 0 : B^T p + (1 - alpha_u) / alpha_u diag_i u_i
__global__ void flow_rhs(int n, const uint8_t* fixed, const double* bt, const double* u, const double* dorig,
                         double alpha_u, double* rhs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rhs[i] = fixed[i] ? 0.0 : bt[i] + ((1.0 - alpha_u) / alpha_u) * dorig[i] * u[i];
}
// Gauss-Seidel on the rows of one colour, a warp per row:
// x_i += omega ((rhs_i - sum_{j != i} a_ij x_j) / a_ii - x_i)
// the same colour step for the three velocity components at once: they share
// the matrix, so each row is read once; per component the arithmetic is
// gs_colour's
__global__ void gs_colour3(int count, const int32_t* __restrict__ rows, const int32_t* __restrict__ row,
                           const int32_t* __restrict__ col, const double* __restrict__ val,
                           const int32_t* __restrict__ dpos, const double* __restrict__ r0,
                           const double* __restrict__ r1, const double* __restrict__ r2, double* x0, double* x1,
                           double* x2, double omega) {
  const int q = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (q >= count) return;
  const int i = rows[q];
  double o0 = 0, o1 = 0, o2 = 0;
  for (int k = row[i] + lane; k < row[i + 1]; k += 32) {
    const int j = col[k];
    if (j != i) {
      const double v = val[k];
      o0 += v * x0[j];
      o1 += v * x1[j];
      o2 += v * x2[j];
    }
  }
  o0 = warp_sum(o0);
  o1 = warp_sum(o1);
  o2 = warp_sum(o2);
  if (lane == 0) {
    const double d = val[dpos[i]];
    const double g0 = (r0[i] - o0) / d, g1 = (r1[i] - o1) / d, g2 = (r2[i] - o2) / d;
    x0[i] = x0[i] + omega * (g0 - x0[i]);
    x1[i] = x1[i] + omega * (g1 - x1[i]);
    x2[i] = x2[i] + omega * (g2 - x2[i]);
  }
}
__global__ void residual_free(int n, const uint8_t* fixed, const double* b, const double* Ax, double* r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = fixed[i] ? 0.0 : b[i] - Ax[i];
}
__global__ void p_update_minus(int n, int pin, double a, const double* dp, double* p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = (i == pin) ? 0.0 : p[i] - a * dp[i];
}
__global__ void twice(size_t n, const double* a, double* b) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i] + a[i];
}

// Jacobi PCG to max(atol, rtol ||r0||) from the guess in x, pin kept zero
// (hxt4b_main.cu:197-201)
template <class Op>
CgResult pcg_prod(Op& A, const double* rhs, double* x, const double* invdiag, double rtol, double atol, int maxit,
                  CgWork& W, int pin) {
  const int n = W.n;
  {
    CgResult D;
    auto jac = [&](const double* r, double* z) {
      cg_jacobi<<<grid(n), kTPB>>>(n, invdiag, r, z, pin);
      NDS_LAUNCH();
    };
    if (cg_device(A, jac, rhs, x, rtol, atol, 0.0, maxit, W, pin, D)) return D;
  }
  A.apply(x, W.q.p);
  residual<<<grid(n), kTPB>>>(n, rhs, W.q.p, W.r.p);
  NDS_LAUNCH();
  set_at<<<1, 1>>>(pin, 0.0, W.r.p);
  const double r0 = W.red.norm(W.r.p);
  if (r0 == 0) return {0, 0, true};
  const double target = std::max(atol, rtol * r0);
  mul<<<grid(n), kTPB>>>(n, invdiag, W.r.p, W.z.p);
  NDS_LAUNCH();
  NDS_CUDA(cudaMemcpy(W.p.p, W.z.p, n * sizeof(double), cudaMemcpyDeviceToDevice));
  double rho = W.red.dot(W.r.p, W.z.p);
  CgResult R;
  for (int k = 0; k < maxit; ++k) {
    A.apply(W.p.p, W.q.p);
    const double pq = W.red.dot(W.p.p, W.q.p);
    if (!(pq > 0)) throw std::runtime_error("mixed-mesh pressure PCG pAp nonpositive");
    axpy2<<<grid(n), kTPB>>>(n, rho / pq, W.p.p, W.q.p, x, W.r.p);
    NDS_LAUNCH();
    set_at<<<1, 1>>>(pin, 0.0, x);
    set_at<<<1, 1>>>(pin, 0.0, W.r.p);
    const double rn = W.red.norm(W.r.p);
    R.its = k + 1;
    R.rel = rn / r0;
    if (rn <= target) {
      R.ok = true;
      break;
    }
    mul<<<grid(n), kTPB>>>(n, invdiag, W.r.p, W.z.p);
    NDS_LAUNCH();
    const double nr = W.red.dot(W.r.p, W.z.p);
    xpby<<<grid(n), kTPB>>>(n, nr / rho, W.z.p, W.p.p);
    NDS_LAUNCH();
    set_at<<<1, 1>>>(pin, 0.0, W.p.p);
    rho = nr;
  }
  return R;
}

// ---- classical AMG preconditioner of the pressure correction (the
// reference's hxt4c::HybridAMG, hybrid_hxt5b/hybrid_amg.cuh:127-533).  The
// hierarchy is built once on the host from the initial rAU; the fine matrix
// B diag(rAU) B^T is refreshed on the device every SIMPLE iteration.
// Restriction gathers through the explicit transpose of each transfer, so
// the V-cycle sums in a fixed order (the reference scatters with atomics).

// entry k of the fine matrix: merge of the sorted B rows i and j
__global__ void amg_fine_refresh(int nnz, const int32_t* __restrict__ erow, const int32_t* __restrict__ acol,
                                 const int32_t* __restrict__ brow, const int32_t* __restrict__ bcol,
                                 const double* __restrict__ bx, const double* __restrict__ by,
                                 const double* __restrict__ bz, const double* __restrict__ rau, int pin,
                                 double* __restrict__ aval) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int i = erow[k], j = acol[k];
  if (i == pin || j == pin) {
    aval[k] = (i == pin && j == pin) ? 1.0 : 0.0;
    return;
  }
  int a = brow[i], b = brow[j];
  const int ae = brow[i + 1], be = brow[j + 1];
  double s = 0;
  while (a < ae && b < be) {
    const int ga = bcol[a], gb = bcol[b];
    if (ga < gb) {
      ++a;
    } else if (gb < ga) {
      ++b;
    } else {
      s += rau[ga] * (bx[a] * bx[b] + by[a] * by[b] + bz[a] * bz[b]);
      ++a;
      ++b;
    }
  }
  aval[k] = s;
}
// diagonal and absolute row sum; flags a nonpositive or non-finite one
__global__ void amg_diag_l1(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ dpos,
                            const double* __restrict__ val, double* __restrict__ diag, double* __restrict__ l1,
                            int* __restrict__ bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d = val[dpos[i]];
  double s = 0;
  for (int k = row[i]; k < row[i + 1]; ++k) s += fabs(val[k]);
  diag[i] = d;
  l1[i] = s;
  if (!(d > 0) || !isfinite(d) || !(s > 0) || !isfinite(s)) atomicAdd(bad, 1);
}
__global__ void amg_jacobi_set(int n, double w, const double* b, const double* den, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = w * b[i] / den[i];
}
__global__ void amg_jacobi_add(int n, double w, const double* r, const double* den, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += w * r[i] / den[i];
}
// symmetric Chebyshev on D^-1/2 A D^-1/2: bs = b / sqrt(d) (b may be bs)
__global__ void amg_scale_rhs(int n, const double* b, const double* d, double* bs) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) bs[i] = b[i] / sqrt(d[i]);
}
__global__ void amg_scaled_copy(int n, double w, const double* bs, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = w * bs[i];
}
__global__ void amg_unscale(int n, const double* y, const double* d, double* x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = y[i] / sqrt(d[i]);
}
__global__ void amg_unscale_inplace(int n, double* x, const double* d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] /= sqrt(d[i]);
}
// y += w (bs - Hy); Hy may be y itself
__global__ void amg_cheb_add(int n, double w, const double* bs, const double* Hy, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += w * (bs[i] - Hy[i]);
}
// one colour of a Gauss-Seidel sweep, one warp per row
__global__ void amg_gs_colour(int count, const int32_t* __restrict__ rows, const int32_t* __restrict__ row,
                              const int32_t* __restrict__ col, const double* __restrict__ val,
                              const double* __restrict__ diag, const double* __restrict__ b, double* x, double w) {
  const int q = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (q >= count) return;
  const int i = rows[q];
  double off = 0;
  for (int k = row[i] + lane; k < row[i + 1]; k += 32) {
    const int j = col[k];
    if (j != i) off += val[k] * x[j];
  }
  off = warp_sum(off);
  if (lane == 0) {
    const double old = x[i];
    x[i] = old + w * ((b[i] - off) / diag[i] - old);
  }
}
// y += A x (prolongation) or y = A x (levels, restriction through P^T), L
// lanes per row (8 for the short rows of P, 32 otherwise)
template <int L>
__global__ void amg_csr_add(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                            const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                            int accumulate) {
  const long long gt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int i = (int)(gt / L), lane = (int)(gt % L);
  const bool live = i < n;
  double s = 0;
  if (live)
    for (int k = row[i] + lane; k < row[i + 1]; k += L) s += val[k] * x[col[k]];
  s = group_sum<L>(s);
  if (live && lane == 0) y[i] = accumulate ? y[i] + s : s;
}
// x = inv b with a dense row-major inverse, warp per row
__global__ void amg_dense(int n, const double* __restrict__ inv, const double* __restrict__ b, double* __restrict__ x) {
  const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  double s = 0;
  for (int j = lane; j < n; j += 32) s += inv[(size_t)i * n + j] * b[j];
  s = warp_sum(s);
  if (lane == 0) x[i] = s;
}
__global__ void amg_axpy(int n, const double* x, double* y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

// greedy colouring of a symmetric pattern: each row takes the smallest colour
// not held by a lower-numbered neighbour (hybrid_amg.cuh:195-215)
void amg_colours(const CsrHost& A, std::vector<int32_t>& off, std::vector<int32_t>& rows) {
  std::vector<int> colour((size_t)A.n, -1), mark;
  int nc = 0;
  for (int i = 0; i < A.n; ++i) {
    for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
      const int j = A.col[(size_t)k];
      if (j >= i) continue;
      const int c = colour[(size_t)j];
      if (c >= (int)mark.size()) mark.resize((size_t)c + 32, -1);
      mark[(size_t)c] = i;
    }
    int c = 0;
    while (c < (int)mark.size() && mark[(size_t)c] == i) ++c;
    colour[(size_t)i] = c;
    nc = std::max(nc, c + 1);
  }
  off.assign((size_t)nc + 1, 0);
  for (int c : colour) ++off[(size_t)c + 1];
  for (int c = 0; c < nc; ++c) off[(size_t)c + 1] += off[(size_t)c];
  rows.resize((size_t)A.n);
  std::vector<int32_t> next(off.begin(), off.end() - 1);
  for (int i = 0; i < A.n; ++i) rows[(size_t)next[(size_t)colour[(size_t)i]]++] = i;
}

std::vector<int32_t> rows32(const std::vector<int64_t>& r) {
  std::vector<int32_t> o(r.size());
  for (size_t i = 0; i < r.size(); ++i) {
    if (r[i] > INT32_MAX) throw std::runtime_error("AMG level too large for 32-bit row offsets");
    o[i] = (int32_t)r[i];
  }
  return o;
}

struct AmgLevel {
  int n = 0;
  Buf<int32_t> row, col, dpos, crows;
  Buf<double> val, diag, l1, b, x, r, tmp, corr;
  Buf<double> r2, corr2;  // post-smoothing work vectors of the separate-buffer V-cycle
  std::vector<int32_t> coff;
  AmgLevel(const CsrHost& A, bool colour)
      : n(A.n), row(rows32(A.row)), col(A.col), val(A.val), diag(A.diag), b((size_t)A.n), x((size_t)A.n),
        r((size_t)A.n), tmp((size_t)A.n), corr((size_t)A.n), r2((size_t)A.n), corr2((size_t)A.n) {
    std::vector<int32_t> dp((size_t)n, -1);
    std::vector<double> l((size_t)n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int64_t k = A.row[(size_t)i]; k < A.row[(size_t)i + 1]; ++k) {
        if (A.col[(size_t)k] == i) dp[(size_t)i] = (int32_t)k;
        l[(size_t)i] += std::abs(A.val[(size_t)k]);
      }
    for (int v : dp)
      if (v < 0) throw std::runtime_error("AMG level without a diagonal entry");
    dpos.upload(dp);
    l1.upload(l);
    if (colour) {
      std::vector<int32_t> rows;
      amg_colours(A, coff, rows);
      crows.upload(rows);
    }
  }
  void apply(const double* in, double* out) const {
    amg_csr_add<32><<<grid((long long)n * 32), kTPB>>>(n, row.p, col.p, val.p, in, out, 0);
    NDS_LAUNCH();
  }
};
struct AmgTransfer {
  int nf, nc;
  Buf<int32_t> prow, pcol, rrow, rcol;
  Buf<double> pval, rval;
  explicit AmgTransfer(const Transfer& P) : nf(P.nf), nc(P.nc), prow(rows32(P.row)), pcol(P.col), pval(P.val) {
    // R = P^T, rows ascending in the fine index
    std::vector<int32_t> rr((size_t)nc + 1, 0), rc(P.col.size());
    std::vector<double> rv(P.col.size());
    for (int32_t c : P.col) ++rr[(size_t)c + 1];
    for (int c = 0; c < nc; ++c) rr[(size_t)c + 1] += rr[(size_t)c];
    std::vector<int32_t> next(rr.begin(), rr.end() - 1);
    for (int i = 0; i < nf; ++i)
      for (int64_t k = P.row[(size_t)i]; k < P.row[(size_t)i + 1]; ++k) {
        const int32_t q = next[(size_t)P.col[(size_t)k]]++;
        rc[(size_t)q] = i;
        rv[(size_t)q] = P.val[(size_t)k];
      }
    rrow.upload(rr);
    rcol.upload(rc);
    rval.upload(rv);
  }
  void restrict_to(const double* f, double* c) const {
    amg_csr_add<32><<<grid((long long)nc * 32), kTPB>>>(nc, rrow.p, rcol.p, rval.p, f, c, 0);
    NDS_LAUNCH();
  }
  void prolong_add(const double* c, double* f) const {
    amg_csr_add<8><<<grid((long long)nf * 8), kTPB>>>(nf, prow.p, pcol.p, pval.p, c, f, 1);
    NDS_LAUNCH();
  }
};

struct HybridAmgDevice {
  const nds_hybrid_flow_options& o;
  int pin;
  std::unique_ptr<AmgLevel> fine;
  Buf<int32_t> erow;
  std::vector<std::unique_ptr<AmgLevel>> L;
  std::vector<std::unique_ptr<AmgTransfer>> P;
  Buf<double> tinv;
  int tn = 0;
  double fine_lambda = 0;
  std::vector<double> level_lambda;
  HybridAmgDevice(const HybridSchurCsr& F, const Hierarchy& H, int pin_, const nds_hybrid_flow_options& opt)
      : o(opt), pin(pin_), erow(F.entry_row), tinv(H.terminal_inv), tn(H.terminal_n), fine_lambda(H.fine_lambda),
        level_lambda(H.level_lambda) {
    const bool mc = o.amg_smoother == NDS_SM_MCGS;
    fine = std::make_unique<AmgLevel>(F.A, mc);
    for (size_t l = 0; l < H.A.size(); ++l) L.push_back(std::make_unique<AmgLevel>(H.A[l], mc && l + 1 < H.A.size()));
    for (const auto& t : H.P) P.push_back(std::make_unique<AmgTransfer>(t));
    if (L.empty() || P.size() != L.size() || tn != L.back()->n) throw std::runtime_error("AMG hierarchy shape");
  }
  void refresh(const Div& B, const double* rau, int* bad) {
    const int nnz = (int)fine->val.n;
    amg_fine_refresh<<<grid(nnz), kTPB>>>(nnz, erow.p, fine->col.p, B.row.p, B.col.p, B.bx.p, B.by.p, B.bz.p, rau,
                                          pin, fine->val.p);
    amg_diag_l1<<<grid(fine->n), kTPB>>>(fine->n, fine->row.p, fine->dpos.p, fine->val.p, fine->diag.p, fine->l1.p,
                                         bad);
    NDS_LAUNCH();
  }
  static double cheb_root(double hi, double lo, int k, int degree) {
    const double centre = 0.5 * (hi + lo), radius = 0.5 * (hi - lo), pi = 3.141592653589793238462643383279502884;
    return centre - radius * std::cos(pi * (2.0 * k + 1.0) / (2.0 * degree));
  }
  // zero initial guess: x = S b.  The work vectors are passed as the
  // reference passes them (hybrid_amg.cuh:445-506): its post-smoothing calls
  // hand the same vector as x and corr (and, on the fine level, as b and r),
  // and the in-place updates below reproduce what that aliasing computes.
  void smooth(AmgLevel& A, const double* b, double* x, double* tmp, double* r, double* corr, int sweeps,
              double lambda) {
    const int n = A.n;
    if (o.amg_smoother == NDS_SM_MCGS) {
      NDS_CUDA(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double)));
      auto one = [&](bool forward) {
        const int nc = (int)A.coff.size() - 1;
        for (int q = 0; q < nc; ++q) {
          const int c = forward ? q : nc - 1 - q;
          const int beg = A.coff[(size_t)c], cnt = A.coff[(size_t)c + 1] - beg;
          amg_gs_colour<<<grid((long long)cnt * 32), kTPB>>>(cnt, A.crows.p + beg, A.row.p, A.col.p, A.val.p,
                                                             A.diag.p, b, x, o.amg_mcgs_omega);
        }
      };
      for (int s = 0; s < sweeps; ++s) {
        if (o.amg_mcgs_order == NDS_MCGS_SYMMETRIC) {
          one(true);
          one(false);
        } else {
          one(o.amg_mcgs_order == NDS_MCGS_FORWARD);
        }
      }
      NDS_LAUNCH();
      return;
    }
    if (o.amg_smoother == NDS_SM_JACOBI || o.amg_smoother == NDS_SM_L1JACOBI) {
      const double* den = o.amg_smoother == NDS_SM_L1JACOBI ? A.l1.p : A.diag.p;
      amg_jacobi_set<<<grid(n), kTPB>>>(n, o.amg_jacobi_omega, b, den, x);
      for (int s = 1; s < sweeps; ++s) {
        A.apply(x, tmp);
        residual<<<grid(n), kTPB>>>(n, b, tmp, r);
        amg_jacobi_add<<<grid(n), kTPB>>>(n, o.amg_jacobi_omega, r, den, x);
      }
      NDS_LAUNCH();
      return;
    }
    const double lo = o.amg_lambda_low_fraction * lambda;
    if (!(lambda > lo && lo > 0)) throw std::runtime_error("AMG Chebyshev interval invalid");
    const int deg = o.amg_cheb_degree;
    amg_scale_rhs<<<grid(n), kTPB>>>(n, b, A.diag.p, r);
    amg_scaled_copy<<<grid(n), kTPB>>>(n, 1.0 / cheb_root(lambda, lo, 0, deg), r, x);
    for (int k = 1; k < deg; ++k) {
      amg_unscale<<<grid(n), kTPB>>>(n, x, A.diag.p, tmp);
      A.apply(tmp, corr);
      amg_unscale_inplace<<<grid(n), kTPB>>>(n, corr, A.diag.p);
      amg_cheb_add<<<grid(n), kTPB>>>(n, 1.0 / cheb_root(lambda, lo, k, deg), r, corr, x);
    }
    amg_unscale<<<grid(n), kTPB>>>(n, x, A.diag.p, x);
    NDS_LAUNCH();
  }
  // post = true: the post-smoothing call; with amg_separate_post it gets work
  // vectors of its own, which makes the V-cycle symmetric
  void smooth_fine(const double* b, double* x, bool post = false) {
    AmgLevel& F = *fine;
    const bool sep = post && o.amg_separate_post;
    smooth(F, b, x, F.tmp.p, sep ? F.r2.p : F.r.p, sep ? F.corr2.p : F.corr.p,
           o.amg_smoother == NDS_SM_MCGS ? o.amg_mcgs_fine_sweeps : o.amg_jacobi_fine_sweeps, fine_lambda);
  }
  void smooth_coarse(size_t l, const double* b, double* x, bool post = false) {
    AmgLevel& A = *L[l];
    const bool sep = post && o.amg_separate_post;
    smooth(A, b, x, A.tmp.p, sep ? A.r2.p : A.r.p, sep ? A.corr2.p : A.corr.p,
           o.amg_smoother == NDS_SM_MCGS ? o.amg_mcgs_coarse_sweeps : o.amg_jacobi_coarse_sweeps,
           l < level_lambda.size() ? level_lambda[l] : 0.0);
  }
  void vcycle(size_t l, const double* b, double* x) {
    AmgLevel& A = *L[l];
    if (l + 1 == L.size()) {
      amg_dense<<<grid((long long)A.n * 32), kTPB>>>(A.n, tinv.p, b, x);
      NDS_LAUNCH();
      return;
    }
    smooth_coarse(l, b, x);
    A.apply(x, A.tmp.p);
    residual<<<grid(A.n), kTPB>>>(A.n, b, A.tmp.p, A.r.p);
    AmgLevel& Cn = *L[l + 1];
    P[l + 1]->restrict_to(A.r.p, Cn.b.p);
    vcycle(l + 1, Cn.b.p, Cn.x.p);
    P[l + 1]->prolong_add(Cn.x.p, x);
    A.apply(x, A.tmp.p);
    residual<<<grid(A.n), kTPB>>>(A.n, b, A.tmp.p, A.r.p);
    NDS_CUDA(cudaMemcpyAsync(A.b.p, A.r.p, (size_t)A.n * sizeof(double), cudaMemcpyDeviceToDevice));
    smooth_coarse(l, A.b.p, A.corr.p, true);
    amg_axpy<<<grid(A.n), kTPB>>>(A.n, A.corr.p, x);
    NDS_LAUNCH();
  }
  // z = V-cycle(b) with the fine smoother on both sides
  void apply(const double* b, double* z) {
    AmgLevel& F = *fine;
    smooth_fine(b, z);
    F.apply(z, F.tmp.p);
    residual<<<grid(F.n), kTPB>>>(F.n, b, F.tmp.p, F.r.p);
    AmgLevel& C0 = *L[0];
    P[0]->restrict_to(F.r.p, C0.b.p);
    vcycle(0, C0.b.p, C0.x.p);
    P[0]->prolong_add(C0.x.p, z);
    F.apply(z, F.tmp.p);
    residual<<<grid(F.n), kTPB>>>(F.n, b, F.tmp.p, F.r.p);
    smooth_fine(F.r.p, F.corr.p, true);
    amg_axpy<<<grid(F.n), kTPB>>>(F.n, F.corr.p, z);
    NDS_LAUNCH();
  }
};

// AMG-preconditioned CG on the pinned pressure system
// (hybrid_amg.cuh:535-580): stops at max(atol, rtol ||r0||)
template <class Op>
CgResult pcg_amg(Op& A, HybridAmgDevice& M, const double* rhs, double* x, double rtol, double atol, int maxit,
                 CgWork& W, int pin) {
  const int n = W.n;
  {
    CgResult D;
    auto vc = [&](const double* r, double* z) {
      M.apply(r, z);
      set_at<<<1, 1>>>(pin, 0.0, z);
      NDS_LAUNCH();
    };
    if (cg_device(A, vc, rhs, x, rtol, atol, atol, maxit, W, pin, D)) return D;
  }
  A.apply(x, W.q.p);
  residual<<<grid(n), kTPB>>>(n, rhs, W.q.p, W.r.p);
  NDS_LAUNCH();
  set_at<<<1, 1>>>(pin, 0.0, W.r.p);
  const double r0 = W.red.norm(W.r.p);
  if (!std::isfinite(r0)) throw std::runtime_error("mixed-mesh pressure PCG: initial residual not finite");
  if (r0 <= atol) return {0, 0, true};
  const double target = std::max(atol, rtol * r0);
  M.apply(W.r.p, W.z.p);
  set_at<<<1, 1>>>(pin, 0.0, W.z.p);
  NDS_CUDA(cudaMemcpy(W.p.p, W.z.p, n * sizeof(double), cudaMemcpyDeviceToDevice));
  double rho = W.red.dot(W.r.p, W.z.p);
  if (!(rho > 0) || !std::isfinite(rho)) throw std::runtime_error("mixed-mesh pressure PCG: initial rho nonpositive");
  CgResult R;
  for (int k = 0; k < maxit; ++k) {
    A.apply(W.p.p, W.q.p);
    const double pq = W.red.dot(W.p.p, W.q.p);
    if (!(pq > 0) || !std::isfinite(pq)) throw std::runtime_error("mixed-mesh pressure PCG pAp nonpositive");
    axpy2<<<grid(n), kTPB>>>(n, rho / pq, W.p.p, W.q.p, x, W.r.p);
    NDS_LAUNCH();
    set_at<<<1, 1>>>(pin, 0.0, x);
    set_at<<<1, 1>>>(pin, 0.0, W.r.p);
    const double rn = W.red.norm(W.r.p);
    R.its = k + 1;
    R.rel = rn / r0;
    if (rn <= target) {
      R.ok = true;
      break;
    }
    M.apply(W.r.p, W.z.p);
    set_at<<<1, 1>>>(pin, 0.0, W.z.p);
    const double nr = W.red.dot(W.r.p, W.z.p);
    if (!(nr > 0) || !std::isfinite(nr)) throw std::runtime_error("mixed-mesh pressure PCG rho nonpositive");
    xpby<<<grid(n), kTPB>>>(n, nr / rho, W.z.p, W.p.p);
    NDS_LAUNCH();
    set_at<<<1, 1>>>(pin, 0.0, W.p.p);
    rho = nr;
  }
  return R;
}

void run_flow(const char* path, const nds_hybrid_flow_options& o, int verbose, nds_hybrid_flow_report* out,
              double* const fields[4]) {
  const HybridMesh M = read_hxt1_hybrid(path);
  const auto P = interface_plans(M);
  HybridFlow F = build_hybrid_flow(M, P, o.re, o.bulk, o.gamma);
  HybridStokes Hb;
  build_hybrid_divergence(M, P, Hb);
  const int nv = F.nvel, np = F.np, nh = F.nhex, nt = F.ntet, nnz = (int)F.col.size(), pin = F.pin;
  {
    const Rules3 r = rules3();
    NDS_CUDA(cudaMemcpyToSymbol(c_g3, r.v, sizeof(r.v)));
    const auto& T = ref_tensors().T;
    NDS_CUDA(cudaMemcpyToSymbol(c_tet_conv, &T[0][0][0][0], sizeof(double) * 8 * 8 * 8 * 3));
  }
  std::vector<int32_t> hexes(8 * (size_t)nh), hdofs(14 * (size_t)nh), tdofs(8 * (size_t)nt);
  std::vector<double> tgeom(12 * (size_t)nt);
  for (int c = 0; c < nh; ++c) {
    for (int a = 0; a < 8; ++a) hexes[8 * (size_t)c + a] = M.hexes[(size_t)c][(size_t)a];
    for (int a = 0; a < 14; ++a) hdofs[14 * (size_t)c + a] = M.hex_dofs[(size_t)c][(size_t)a];
  }
  for (int c = 0; c < nt; ++c) {
    for (int a = 0; a < 8; ++a) tdofs[8 * (size_t)c + a] = M.tet_dofs[(size_t)c][(size_t)a];
    for (int a = 0; a < 12; ++a) tgeom[12 * (size_t)c + a] = M.tet_geom[(size_t)c][(size_t)a];
  }
  Buf<double> d_xyz(M.xyz), d_tgeom(tgeom), d_base(F.base), d_dr(F.diag_r_base), d_local((size_t)nh * 196 + (size_t)nt * 64);
  Buf<int32_t> d_hexes(hexes), d_hdofs(hdofs), d_tdofs(tdofs), d_row(F.row), d_col(F.col), d_dpos(F.diag_pos),
      d_soff(F.src_off), d_src(F.src), d_crows(F.colour_rows);
  Buf<uint8_t> d_fixed(F.fixed);
  Buf<double> u0(F.u0), u1(F.u1), u2(F.u2), conv((size_t)nnz), val((size_t)nnz), dorig((size_t)nv), rau((size_t)nv),
      isd((size_t)np), p((size_t)np), dp((size_t)np), cont((size_t)np), bt0((size_t)nv), bt1((size_t)nv),
      bt2((size_t)nv), r0((size_t)nv), r1((size_t)nv), r2((size_t)nv), tmp((size_t)nv), res((size_t)nv);
  Buf<int> d_bad((size_t)2);  // [0] momentum rows / hex Jacobians, [1] refreshed pressure matrix
  Div B(Hb);
  Schur S(B, rau.p, pin);
  Reducer pred(np), ured(nv);
  CgWork WP(np);
  auto apply_val = [&](const double* x, double* y) {
    csr_mv<<<grid((long long)nv * 32), kTPB>>>(nv, d_row.p, d_col.p, val.p, x, y);
    NDS_LAUNCH();
  };
  const double dpdz_exact = -32 * F.nu * o.bulk / (F.diameter * F.diameter), drop_exact = -dpdz_exact * F.length;
  const int ncol = (int)F.colour_off.size() - 1;
  const char* work = o.momentum_work == 0 ? "fgs1" : o.momentum_work == 1 ? "altgs1" : "sgs1";
  if (verbose) {
    std::printf("NODALS_HXT4B_CONFIG precision=fp64 geometry=fp64 reductions=fp64 cellsHex=%d cellsTet=%d velocityDofs=%d "
                "pressureDofs=%d csrNnz=%d colors=%d maxColor=%d Re=%.12g bulk=%.12g nu=%.12e D=%.12e L=%.12e gamma=%.6g "
                "convection=CENTRAL_ADVECTIVE_LAGGED interfaceConvection=VOLUME_ONLY_TANGENTIAL_RE20_GATE momentumWork=%s "
                "momOmega=%.6g momRtol=%.3e momAtol=%.3e fixedWorkIgnoresMomTolerances=1 pressureSolver=%s "
                "momentumSign=A_u_MINUS_BT_p pRtol=%.3e pAtol=%.3e pMax=%d alphaU=%.6g alphaP=%.6g rauScale=%.6g "
                "rauPenaltyIncluded=0 simpleTol=%.3e status=PASS\n",
                nh, nt, nv, np, nnz, ncol, F.max_colour, o.re, o.bulk, F.nu, F.diameter, F.length, o.gamma, work,
                o.mom_omega, o.mom_rtol, o.mom_atol, o.pressure_solver == 1 ? "PCG_AMG" : "PCG_JACOBI", o.p_rtol,
                o.p_atol, o.p_max, o.alpha_u, o.alpha_p, o.rau_scale, o.simple_tol);
    std::printf("NODALS_HXT4B_HAGEN_POISEUILLE expectedDpDz=%.12e expectedDropPinMinusPout=%.12e inlet=STRONG_PARABOLIC "
                "wall=STRONG_NOSLIP outlet=NATURAL_TRACTION pressureGaugePin=%d status=PASS\n",
                dpdz_exact, drop_exact, pin);
  }
  auto sweep3 = [&](bool forward) {
    for (int q = 0; q < ncol; ++q) {
      const int c = forward ? q : ncol - 1 - q;
      const int b = F.colour_off[(size_t)c], n = F.colour_off[(size_t)c + 1] - b;
      gs_colour3<<<grid((long long)n * 32), kTPB>>>(n, d_crows.p + b, d_row.p, d_col.p, val.p, d_dpos.p, r0.p, r1.p,
                                                    r2.p, u0.p, u1.p, u2.p, o.mom_omega);
      NDS_LAUNCH();
    }
  };
  // the momentum work of the three components (independent systems with one
  // matrix), swept together
  auto momentum_work3 = [&](int it) {
    if (o.momentum_work == 0) sweep3(true);
    else if (o.momentum_work == 1) sweep3((it & 1) != 0);
    else {
      sweep3(true);
      sweep3(false);
    }
  };
  // persistent grids of the convection kernels: 8 blocks of 256 threads per SM
  int conv_blocks = 0;
  {
    int dev = 0, sms = 0;
    NDS_CUDA(cudaGetDevice(&dev));
    NDS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    conv_blocks = 8 * std::max(sms, 1);
  }
  Buf<double> d_ptab((size_t)27 * 14 * 4);
  hex_point_table<<<1, 32>>>(d_ptab.p);
  NDS_LAUNCH();
  // lagged convection of the current velocity, relaxed rows and rAU
  auto assemble = [&]() {
    if (nh) {
      hex_conv_local<<<std::min(nh, conv_blocks), kTPB>>>(nh, d_xyz.p, d_hexes.p, d_hdofs.p, u0.p, u1.p, u2.p,
                                                          d_ptab.p, d_local.p, d_bad.p);
      NDS_LAUNCH();
    }
    if (nt) {
      tet_conv_local<<<std::min((nt + 3) / 4, conv_blocks), kTPB>>>(nt, d_tgeom.p, d_tdofs.p, u0.p, u1.p, u2.p,
                                                                    d_local.p + 196 * (size_t)nh);
      NDS_LAUNCH();
    }
    conv_gather<<<grid(nnz), kTPB>>>(nnz, d_soff.p, d_src.p, d_local.p, conv.p);
    NDS_LAUNCH();
    flow_rows<<<grid(nv), kTPB>>>(nv, d_row.p, d_dpos.p, d_fixed.p, d_base.p, conv.p, d_dr.p, o.alpha_u, o.rau_scale,
                                  val.p, dorig.p, rau.p, d_bad.p);
    NDS_LAUNCH();
  };
  auto check_bad = [&]() {
    int bad[2] = {0, 0};
    NDS_CUDA(cudaMemcpy(bad, d_bad.p, sizeof(bad), cudaMemcpyDeviceToHost));
    if (bad[0]) throw std::runtime_error("mixed-mesh SIMPLE: nonpositive momentum diagonal or hex Jacobian");
    if (bad[1]) throw std::runtime_error("mixed-mesh SIMPLE: refreshed pressure matrix has an invalid diagonal");
  };
  // AMG preconditioner: hierarchy from the initial rAU, as the reference's
  // turbulent entry builds it before its loop (hxt5b_main.cu:185-212)
  std::unique_ptr<HybridAmgDevice> amg;
  if (o.pressure_solver == 1) {
    const AmgOptions ao = hybrid_amg_options(o);
    assemble();
    check_bad();
    std::vector<double> rau_h((size_t)nv);
    NDS_CUDA(cudaMemcpy(rau_h.data(), rau.p, nv * sizeof(double), cudaMemcpyDeviceToHost));
    const HybridSchurCsr FS = hybrid_schur_csr(Hb, pin, rau_h);
    const Hierarchy HH = build_cf_hierarchy(FS.A, ao);
    amg = std::make_unique<HybridAmgDevice>(FS, HH, pin, o);
    if (verbose) {
      static const char* sm[] = {"cheb2", "jacobi", "l1jacobi", "mcgs"};
      std::printf("NODALS_HXT4C_FINE_HOST rows=%d nnz=%zu avgNnz=%.6f pin=%d source=B_DIAG_RAU_BT_REDUCED_PIN "
                  "status=PASS\n",
                  FS.A.n, FS.A.val.size(), FS.A.n ? (double)FS.A.val.size() / FS.A.n : 0.0, pin);
      std::printf("NODALS_HXT4C_AMG_UPLOAD levels=%zu transfers=%zu terminal=%d smoother=%s chebScaling=%s "
                  "status=PASS\n",
                  HH.A.size(), HH.P.size(), HH.terminal_n, sm[o.amg_smoother],
                  o.amg_smoother == NDS_SM_CHEB2 ? "SYMMETRIC_D_HALF" : "NA");
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  double c0 = -1, rel = 1;
  bool conv_ok = false;
  int outer = 0;
  long long pits = 0;
  for (int it = 1; it <= o.max_outer; ++it) {
    assemble();
    if (amg) {
      amg->refresh(B, rau.p, d_bad.p + 1);
    } else {
      schur_diag_inv<<<grid(np), kTPB>>>(np, B.row.p, B.col.p, B.bx.p, B.by.p, B.bz.p, rau.p, pin, isd.p);
      NDS_LAUNCH();
    }
    check_bad();
    B.BT(p.p, bt0.p, bt1.p, bt2.p);
    flow_rhs<<<grid(nv), kTPB>>>(nv, d_fixed.p, bt0.p, u0.p, dorig.p, o.alpha_u, r0.p);
    flow_rhs<<<grid(nv), kTPB>>>(nv, d_fixed.p, bt1.p, u1.p, dorig.p, o.alpha_u, r1.p);
    flow_rhs<<<grid(nv), kTPB>>>(nv, d_fixed.p, bt2.p, u2.p, dorig.p, o.alpha_u, r2.p);
    NDS_LAUNCH();
    momentum_work3(it);
    B.B(u0.p, u1.p, u2.p, cont.p);
    set_at<<<1, 1>>>(pin, 0.0, cont.p);
    NDS_LAUNCH();
    const double cn = pred.norm(cont.p);
    if (it == 1) c0 = cn;
    rel = cn / std::max(c0, 1e-300);
    NDS_CUDA(cudaMemset(dp.p, 0, np * sizeof(double)));
    const CgResult pr = amg ? pcg_amg(S, *amg, cont.p, dp.p, o.p_rtol, o.p_atol, o.p_max, WP, pin)
                            : pcg_prod(S, cont.p, dp.p, isd.p, o.p_rtol, o.p_atol, o.p_max, WP, pin);
    if (!pr.ok) throw std::runtime_error("mixed-mesh SIMPLE: pressure PCG missed its target within p_max");
    pits += pr.its;
    p_update_minus<<<grid(np), kTPB>>>(np, pin, o.alpha_p, dp.p, p.p);
    NDS_LAUNCH();
    outer = it;
    conv_ok = it > 1 && rel <= o.simple_tol;
    if (verbose && (it <= 5 || it % 20 == 0 || conv_ok)) {
      apply_val(u2.p, tmp.p);
      residual_free<<<grid(nv), kTPB>>>(nv, d_fixed.p, r2.p, tmp.p, res.p);
      NDS_LAUNCH();
      const double mr = ured.norm(res.p) / std::max(ured.norm(r2.p), 1e-300);
      std::printf("NODALS_HXT4B_SIMPLE it=%d relCont=%.12e absCont=%.12e zMomentumResidualRel=%.12e pCG=%d pRel=%.3e "
                  "converged=%d status=PASS\n",
                  it, rel, cn, mr, pr.its, pr.rel, (int)conv_ok);
    }
    if (it >= 5 && (!std::isfinite(rel) || rel > 1e8)) throw std::runtime_error("mixed-mesh SIMPLE diverged");
    if (conv_ok) break;
  }
  if (!conv_ok) throw std::runtime_error("mixed-mesh SIMPLE: no convergence within max_outer");
  const double loop_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::vector<double> hp((size_t)np), hu0((size_t)nv), hu1((size_t)nv), hu2((size_t)nv);
  NDS_CUDA(cudaMemcpy(hp.data(), p.p, np * sizeof(double), cudaMemcpyDeviceToHost));
  NDS_CUDA(cudaMemcpy(hu0.data(), u0.p, nv * sizeof(double), cudaMemcpyDeviceToHost));
  NDS_CUDA(cudaMemcpy(hu1.data(), u1.p, nv * sizeof(double), cudaMemcpyDeviceToHost));
  NDS_CUDA(cudaMemcpy(hu2.data(), u2.p, nv * sizeof(double), cudaMemcpyDeviceToHost));
  nds_hybrid_flow_report R{};
  R.outer_its = outer;
  R.converged = 1;
  R.n_hex = nh;
  R.n_tet = nt;
  R.n_velocity = nv;
  R.final_rel_cont = rel;
  R.slope = hybrid_pressure_slope(M, hp);
  R.slope_exact = dpdz_exact;
  const double pin_p = hybrid_boundary_pressure(M, hp, true), pout_p = hybrid_boundary_pressure(M, hp, false);
  R.p_in = pin_p;
  R.p_out = pout_p;
  R.drop = pin_p - pout_p;
  R.drop_exact = drop_exact;
  long double en = 0, ed = 0, et = 0;
  for (int v = 0; v < M.nv(); ++v) {
    const double ex = pipe_profile(M.xyz[3 * (size_t)v], M.xyz[3 * (size_t)v + 1], F.radius, o.bulk);
    const double e = hu2[(size_t)v] - ex;
    en += e * e;
    ed += ex * ex;
    et += hu0[(size_t)v] * hu0[(size_t)v] + hu1[(size_t)v] * hu1[(size_t)v];
  }
  R.profile_rel_l2 = std::sqrt((double)(en / std::max((long double)1e-300, ed)));
  R.transverse_rel_l2 = std::sqrt((double)(et / std::max((long double)1e-300, ed)));
  // the last convection matrix applied to the axial velocity
  twice<<<grid(nnz), kTPB>>>((size_t)nnz, conv.p, val.p);
  NDS_LAUNCH();
  apply_val(u2.p, tmp.p);
  R.conv_norm = 0.5 * ured.norm(tmp.p);
  R.velocity_norm = ured.norm(u2.p);
  R.avg_pressure_cg = outer ? (double)pits / outer : 0.0;
  R.loop_ms = loop_ms;
  const double slope_err = std::abs(R.slope - dpdz_exact) / std::abs(dpdz_exact);
  const double drop_err = std::abs(R.drop - drop_exact) / std::abs(drop_exact);
  R.pass = drop_err < 0.05 && slope_err < 0.05 && R.profile_rel_l2 < 0.15 && std::isfinite(R.conv_norm);
  if (verbose)
    std::printf("NODALS_HXT4B_PHYSICS pressureSlope=%.12e exactSlope=%.12e slopeRelError=%.12e pIn=%.12e pOut=%.12e "
                "pressureDrop=%.12e exactDrop=%.12e dropRelError=%.12e vertexVelocityProfileRelL2=%.12e "
                "transverseVertexRelL2=%.12e convectionActionNorm=%.12e velocityNorm=%.12e avgPressureCG=%.6f status=%s\n",
                R.slope, dpdz_exact, slope_err, pin_p, pout_p, R.drop, drop_exact, drop_err, R.profile_rel_l2,
                R.transverse_rel_l2, R.conv_norm, R.velocity_norm, R.avg_pressure_cg, R.pass ? "PASS" : "FAIL");
  if (out) *out = R;
  const std::vector<double>* host[4] = {&hu0, &hu1, &hu2, &hp};
  for (int k = 0; k < 4; ++k)
    if (fields[k]) std::copy(host[k]->begin(), host[k]->end(), fields[k]);
}

}  // namespace hy
}  // namespace nds

namespace nds {
namespace hy {
void run_amg_vcycle(const char* path, const double* rau_in, const nds_hybrid_flow_options& o, const double* b,
                    double* z) {
  const AmgOptions ao = hybrid_amg_options(o);
  const HybridMesh M = read_hxt1_hybrid(path);
  HybridStokes Hb;
  build_hybrid_divergence(M, interface_plans(M), Hb);
  const int pin = hybrid_pin(M), np = Hb.np;
  const std::vector<double> rau_h(rau_in, rau_in + Hb.nvel);
  const HybridSchurCsr FS = hybrid_schur_csr(Hb, pin, rau_h);
  const Hierarchy HH = build_cf_hierarchy(FS.A, ao);
  HybridAmgDevice amg(FS, HH, pin, o);
  Div B(Hb);
  Buf<double> rau(rau_h), db(std::vector<double>(b, b + np)), dz((size_t)np);
  Buf<int> bad((size_t)1);
  amg.refresh(B, rau.p, bad.p);
  int nb = 0;
  NDS_CUDA(cudaMemcpy(&nb, bad.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (nb) throw std::runtime_error("pressure matrix has an invalid diagonal");
  amg.apply(db.p, dz.p);
  NDS_CUDA(cudaMemcpy(z, dz.p, np * sizeof(double), cudaMemcpyDeviceToHost));
}
}  // namespace hy
}  // namespace nds

extern "C" int nds_hybrid_amg_vcycle(const char* hxt1_path, const double* rau, const nds_hybrid_flow_options* o,
                                     int device, const double* b, double* z) {
  if (!hxt1_path || !rau || !o || !b || !z) {
    nds::set_error("nds_hybrid_amg_vcycle: null argument");
    return NDS_E_INVALID;
  }
  try {
    nds::hybrid_amg_options(*o);  // option errors before any device work
    int ndev = 0;
    const cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= device) throw nds::CudaError(std::string("no CUDA device available: ") + cudaGetErrorString(e));
    NDS_CUDA(cudaSetDevice(device));
    nds::hy::run_amg_vcycle(hxt1_path, rau, *o, b, z);
    return NDS_OK;
  } catch (const std::invalid_argument& e) {
    nds::set_error(e.what());
    return NDS_E_INVALID;
  } catch (const nds::CudaError& e) {
    nds::set_error(e.what());
    return NDS_E_CUDA;
  } catch (const std::exception& e) {
    nds::set_error(e.what());
    return NDS_E_SETUP;
  }
}

extern "C" int nds_hybrid_stokes_gate(const char* hxt1_path, double nu, double gamma, double rau_scale, double alpha_p,
                                      double simple_tol, int max_outer, int device, int verbose,
                                      nds_hybrid_report* out) {
  if (!hxt1_path || !(nu > 0) || !(gamma > 0) || !(rau_scale > 0) || !(alpha_p > 0) || max_outer < 1) {
    nds::set_error("nds_hybrid_stokes_gate: bad argument");
    return NDS_E_INVALID;
  }
  try {
    int ndev = 0;
    const cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= device) throw nds::CudaError(std::string("no CUDA device available: ") + cudaGetErrorString(e));
    NDS_CUDA(cudaSetDevice(device));
    nds::hy::run_gate(hxt1_path, nu, gamma, rau_scale, alpha_p, simple_tol, max_outer, verbose, out);
    return NDS_OK;
  } catch (const nds::CudaError& e) {
    nds::set_error(e.what());
    return NDS_E_CUDA;
  } catch (const std::exception& e) {
    nds::set_error(e.what());
    return NDS_E_SETUP;
  }
}

extern "C" void nds_hybrid_flow_defaults(nds_hybrid_flow_options* o) {
  if (!o) return;
  *o = nds_hybrid_flow_options{};
  o->re = 20;
  o->bulk = 1;
  o->gamma = 50;
  o->alpha_u = 0.7;
  o->alpha_p = 1.0;
  o->rau_scale = 2.0;
  o->simple_tol = 1e-3;
  o->max_outer = 3000;
  o->momentum_work = 2;
  o->mom_omega = 1.0;
  o->mom_rtol = 0.5;
  o->mom_atol = 1e-8;
  o->p_rtol = 0.9;
  o->p_atol = 1e-12;
  o->p_max = 50;
  o->pressure_solver = 0;
  o->amg_smoother = NDS_SM_CHEB2;
  o->amg_spectrum_policy = NDS_SPEC_AUTO;
  o->amg_terminal = 1000;
  o->amg_power_its = 16;
  o->amg_cheb_degree = 4;
  o->amg_jacobi_fine_sweeps = 1;
  o->amg_jacobi_coarse_sweeps = 1;
  o->amg_mcgs_fine_sweeps = 1;
  o->amg_mcgs_coarse_sweeps = 1;
  o->amg_mcgs_order = NDS_MCGS_SYMMETRIC;
  o->cf_pmax = 8;
  o->cf_interp = NDS_CF_EXTI;
  o->cf_aggressive_first = 0;
  o->cf_theta = 0.25;
  o->amg_lambda_safety = 1.5;
  o->amg_lambda_low_fraction = 0.05;
  o->amg_jacobi_omega = 0.7;
  o->amg_mcgs_omega = 1.0;
  o->amg_separate_post = 0;
}

extern "C" int nds_hybrid_flow(const char* hxt1_path, const nds_hybrid_flow_options* o, int device, int verbose,
                               nds_hybrid_flow_report* out) {
  return nds_hybrid_flow_fields(hxt1_path, o, device, verbose, out, nullptr, nullptr, nullptr, nullptr);
}

extern "C" int nds_hybrid_flow_fields(const char* hxt1_path, const nds_hybrid_flow_options* o, int device, int verbose,
                                      nds_hybrid_flow_report* out, double* u0, double* u1, double* u2,
                                      double* pressure) {
  if (!hxt1_path || !o || !(o->re > 0) || !(o->bulk > 0) || !(o->gamma > 0) || !(o->alpha_u > 0 && o->alpha_u <= 1) ||
      !(o->alpha_p > 0) || !(o->rau_scale > 0) || o->max_outer < 1 || o->p_max < 1 || o->momentum_work < 0 ||
      o->momentum_work > 2 || o->pressure_solver < 0 || o->pressure_solver > 1) {
    nds::set_error("nds_hybrid_flow: bad argument");
    return NDS_E_INVALID;
  }
  try {
    if (o->pressure_solver == 1) nds::hybrid_amg_options(*o);  // option errors before any device work
    int ndev = 0;
    const cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= device) throw nds::CudaError(std::string("no CUDA device available: ") + cudaGetErrorString(e));
    NDS_CUDA(cudaSetDevice(device));
    double* const fields[4] = {u0, u1, u2, pressure};
    nds::hy::run_flow(hxt1_path, *o, verbose, out, fields);
    return NDS_OK;
  } catch (const std::invalid_argument& e) {
    nds::set_error(e.what());
    return NDS_E_INVALID;
  } catch (const nds::CudaError& e) {
    nds::set_error(e.what());
    return NDS_E_CUDA;
  } catch (const std::exception& e) {
    nds::set_error(e.what());
    return NDS_E_SETUP;
  }
}
