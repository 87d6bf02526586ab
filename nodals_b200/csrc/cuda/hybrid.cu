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
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/nodals_b200.h"
#include "../host/hybrid.hpp"
#include "common.cuh"

namespace nds {
void set_error(const std::string& m);
namespace hy {

constexpr int kTPB = 256;

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
__global__ void bt_mv(int n, const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                      const double* __restrict__ bx, const double* __restrict__ by, const double* __restrict__ bz,
                      const double* __restrict__ p, double* __restrict__ v0, double* __restrict__ v1,
                      double* __restrict__ v2) {
  const int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (i >= n) return;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int k = row[i] + lane; k < row[i + 1]; k += 32) {
    const double q = p[col[k]];
    s0 += bx[k] * q;
    s1 += by[k] * q;
    s2 += bz[k] * q;
  }
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  s2 = warp_sum(s2);
  if (lane == 0) {
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
    bt_mv<<<grid((long long)nv * 32), kTPB>>>(nv, trow.p, tcol.p, tx.p, ty.p, tz.p, p, v0, v1, v2);
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
struct CgWork {
  int n;
  Buf<double> r, z, p, q;
  Reducer red;
  explicit CgWork(int n_) : n(n_), r((size_t)n_), z((size_t)n_), p((size_t)n_), q((size_t)n_), red(n_) {}
};
struct CgResult {
  int its = 0;
  double rel = 1;
  bool ok = false;
};
// Jacobi-preconditioned CG to ||r|| <= rtol ||r0|| from the guess in x
// (hybrid_hxt4a/hxt4a_main.cu:309-326; pin >= 0 keeps x, r, p zero there)
template <class Op>
CgResult cg(Op& A, const double* rhs, double* x, const double* invdiag, double rtol, int maxit, CgWork& W,
            int pin = -1) {
  const int n = W.n;
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

}  // namespace hy
}  // namespace nds

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
