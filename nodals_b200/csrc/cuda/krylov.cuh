// Kernels of the mixed-precision pressure solve (precision NDS_MIXED, no
// reference counterpart; the reference solves the pressure correction with
// FP64 or FP32 PCG / Richardson / outer Chebyshev, h8_main_base.cu:569-726):
//
//  * FP64 defect correction: r = b - A x in FP64 on the FP64 fine operator,
//    the inner solve of A d = r / ||r|| in FP32 (PCG, or FGMRES whose
//    Gram-Schmidt dot products and Hessenberg least squares are FP64), then
//    x += ||r|| d in FP64;
//  * FGMRES(m) with right preconditioning run on the device: the iteration
//    index j, the Hessenberg matrix, the Givens rotations and the residual
//    estimate live in device memory, so one loop body (a conditional while
//    node of a CUDA graph) serves every j;
//  * the Galerkin initial guess over earlier pressure corrections.
//
// Every reduction goes through fixed-order block partials (deterministic).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"

namespace nds {
namespace k {

// y = float(s x)
// y = s x in FP32; with x1 also the first (diagonal) step of the fine
// pre-smoother on y, x1 = w0 y / den0 (the expression of jacobi_zero)
__global__ void scale_to_float(int n, const double* __restrict__ x, double s, float* __restrict__ y,
                               const float* __restrict__ den0 = nullptr, float w0 = 0.f, float* __restrict__ x1 = nullptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float v = (float)(s * x[i]);
  y[i] = v;
  if (x1) x1[i] = w0 * v / den0[i];
}
// x += s y (y in FP32, x in FP64)
__global__ void axpy_from_float(int n, double s, const float* __restrict__ y, double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] += s * (double)y[i];
}

// ---------------------------------------------------------------------------
// FGMRES(m) device loop.  Layout of the FP64 work array fg (m = restart):
//   H  [(m+1) x m], column j at fg + j (m+1)   (rotated in place: becomes R)
//   cs [m], sn [m], g [m+1], y [m]
// ctl: [0] j = basis vectors built in this pass, [1] converged, [2] -,
//      [3] iteration cap of this pass.   flags bit 16: breakdown / non-finite.
// sc[slot_wn]: ||w||^2 of the current Arnoldi vector (block partial sum).
// ---------------------------------------------------------------------------
struct FgLayout {
  int m;
  __host__ __device__ int H(int i, int j) const { return j * (m + 1) + i; }
  __host__ __device__ int cs(int j) const { return (m + 1) * m + j; }
  __host__ __device__ int sn(int j) const { return (m + 1) * m + m + j; }
  __host__ __device__ int g(int j) const { return (m + 1) * m + 2 * m + j; }
  __host__ __device__ int y(int j) const { return (m + 1) * m + 3 * m + 1 + j; }
  __host__ __device__ int size() const { return (m + 1) * m + 4 * m + 1; }
};

// out = V[ctl[0]]   (the preconditioner's input, a fixed buffer)
__global__ void fg_fetch(int n, const float* __restrict__ V, const int* __restrict__ ctl, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = V[(size_t)ctl[0] * n + i];
}
// Z[ctl[0]] = z
__global__ void fg_store(int n, const float* __restrict__ z, const int* __restrict__ ctl, float* __restrict__ Z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) Z[(size_t)ctl[0] * n + i] = z[i];
}
// block partials of V_i . w for i = blockIdx.y <= ctl[0]: part[i gridDim.x + block]
__global__ void __launch_bounds__(kBlock) fg_dots(int n, const float* __restrict__ V, const float* __restrict__ w,
                                                  const int* __restrict__ ctl, double* __restrict__ part) {
  const int vi = blockIdx.y;
  if (vi > ctl[0]) return;
  const float* v = V + (size_t)vi * n;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] += (double)v[i] * (double)w[i];
  block_sum<1>(acc);
  if (threadIdx.x == 0) part[(size_t)vi * gridDim.x + blockIdx.x] = acc[0];
}
// H[i][j] = sum of the partials of V_i . w (one block per i <= j)
__global__ void __launch_bounds__(kBlock) fg_reduce_h(const double* __restrict__ part, int nblocks,
                                                      const int* __restrict__ ctl, FgLayout L,
                                                      double* __restrict__ fg) {
  const int vi = blockIdx.x, j = ctl[0];
  if (vi > j) return;
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v[0] += part[(size_t)vi * nblocks + b];
  block_sum<1>(v);
  if (threadIdx.x == 0) fg[L.H(vi, j)] = v[0];
}
// w -= sum_{i <= j} H[i][j] V_i (FP64 sums, FP32 storage); partials of ||w||^2
__global__ void __launch_bounds__(kBlock) fg_orth(int n, const float* __restrict__ V, const double* __restrict__ fg,
                                                  FgLayout L, const int* __restrict__ ctl, float* __restrict__ w,
                                                  double* __restrict__ part) {
  const int j = ctl[0];
  const double* h = fg + L.H(0, j);
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = (double)w[i];
    for (int q = 0; q <= j; ++q) s -= h[q] * (double)V[(size_t)q * n + i];
    const float f = (float)s;
    w[i] = f;
    acc[0] += (double)f * (double)f;
  }
  write_partials<1>(acc, part);
}
// Hessenberg column j: H[j+1][j] = ||w||, the earlier rotations, a new one;
// g and the residual estimate |g[j+1]| (relative: the pass starts from a
// unit vector, g[0] = 1).  Counts the vector, stores ||w|| for fg_normalize,
// and stops the loop on convergence (|g[j+1]| <= tol), at the cap, on a
// happy breakdown (||w|| = 0) or on a non-finite value.
__global__ void fg_givens(double* __restrict__ fg, FgLayout L, double* __restrict__ sc, int wn2_slot, int wn_slot,
                          int tol_slot, int* __restrict__ ctl, int* __restrict__ flags,
                          cudaGraphConditionalHandle loop, int in_graph) {
  const double tol = sc[tol_slot];
  const int j = ctl[0];
  const double wn = sqrt(sc[wn2_slot]);
  sc[wn_slot] = wn;
  double* col = fg + L.H(0, j);
  col[j + 1] = wn;
  for (int i = 0; i < j; ++i) {
    const double c = fg[L.cs(i)], s = fg[L.sn(i)];
    const double a = col[i], b = col[i + 1];
    col[i] = c * a + s * b;
    col[i + 1] = -s * a + c * b;
  }
  const double a = col[j], b = col[j + 1];
  const double r = hypot(a, b);
  bool bad = !isfinite(r) || !isfinite(wn);
  double c = 1.0, s = 0.0;
  if (r > 0.0) {
    c = a / r;
    s = b / r;
  } else {
    bad = true;  // a zero column: the preconditioned operator is singular on this vector
  }
  fg[L.cs(j)] = c;
  fg[L.sn(j)] = s;
  col[j] = r;
  col[j + 1] = 0.0;
  const double gj = fg[L.g(j)];
  fg[L.g(j)] = c * gj;
  fg[L.g(j + 1)] = -s * gj;
  const double res = fabs(fg[L.g(j + 1)]);
  if (bad) *flags |= 16;
  ctl[0] = j + 1;
  const int conv = !bad && (res <= tol || wn == 0.0);
  ctl[1] = conv;
  const bool stop = conv || bad || j + 1 >= ctl[3];
  if (in_graph) cudaGraphSetConditional(loop, stop ? 0u : 1u);
}
// V[ctl[0]] = w / ||w|| (zero when ||w|| = 0)
__global__ void fg_normalize(int n, const float* __restrict__ w, const double* __restrict__ sc, int wn_slot,
                             const int* __restrict__ ctl, float* __restrict__ V) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double wn = sc[wn_slot];
  V[(size_t)ctl[0] * n + i] = wn > 0.0 ? (float)((double)w[i] / wn) : 0.0f;
}
// start of a pass: g = (1, 0, ...), j = 0
__global__ void fg_start(double* __restrict__ fg, FgLayout L, int* __restrict__ ctl, int cap) {
  for (int q = 0; q <= L.m; ++q) fg[L.g(q)] = 0.0;
  fg[L.g(0)] = 1.0;
  ctl[0] = 0;
  ctl[1] = 0;
  ctl[3] = cap;
}
// y = R^-1 g over the k = ctl[0] columns built (back substitution, FP64)
__global__ void fg_backsolve(double* __restrict__ fg, FgLayout L, const int* __restrict__ ctl) {
  const int k = ctl[0];
  for (int i = k - 1; i >= 0; --i) {
    double s = fg[L.g(i)];
    for (int q = i + 1; q < k; ++q) s -= fg[L.H(i, q)] * fg[L.y(q)];
    const double d = fg[L.H(i, i)];
    fg[L.y(i)] = d != 0.0 ? s / d : 0.0;
  }
}
// x += scale sum_{i < k} y_i Z_i  (FP64 sums into the FP64 iterate)
__global__ void fg_combine(int n, const float* __restrict__ Z, const double* __restrict__ fg, FgLayout L,
                           const int* __restrict__ ctl, double scale, double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = ctl[0];
  double s = 0.0;
  for (int q = 0; q < k; ++q) s += fg[L.y(q)] * (double)Z[(size_t)q * n + i];
  x[i] += scale * s;
}

// ---------------------------------------------------------------------------
// Galerkin initial guess over K earlier corrections y_0..y_{K-1} (FP64),
// with w_a = A_a y_a kept from the solve that made y_a (A_a: the pressure
// operator of that SIMPLE iteration; w = b - r of its last FP64 defect, so
// it costs nothing): solve G c = f with G_ab = y_a . w_b (a <= b, mirrored)
// and f_a = y_a . b, then x = sum c_a y_a.  The operator changes slowly from
// one SIMPLE iteration to the next, so G is close to the Galerkin matrix of
// the current operator; the residual of x is then evaluated exactly, so the
// guess only changes the starting point, never the FP64 stopping test.
// ---------------------------------------------------------------------------
constexpr int kMaxGuess = 8;
// partials, per block: G (upper triangle, row-major a <= b) then f
template <int K>
__global__ void __launch_bounds__(kBlock) guess_dots(int n, const double* __restrict__ Y, const double* __restrict__ W,
                                                     const double* __restrict__ b, double* __restrict__ part) {
  constexpr int NG = K * (K + 1) / 2 + K;
  double acc[NG];
#pragma unroll
  for (int q = 0; q < NG; ++q) acc[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double y[K], w[K];
#pragma unroll
    for (int a = 0; a < K; ++a) {
      y[a] = Y[(size_t)a * n + i];
      w[a] = W[(size_t)a * n + i];
    }
    const double bi = b[i];
    int q = 0;
#pragma unroll
    for (int a = 0; a < K; ++a)
#pragma unroll
      for (int c = a; c < K; ++c) acc[q++] += y[a] * w[c];
#pragma unroll
    for (int a = 0; a < K; ++a) acc[q++] += y[a] * bi;
  }
  write_partials<NG>(acc, part);
}
// x = sum c_a y_a (c in coef[0..K))
template <int K>
__global__ void guess_combine(int n, const double* __restrict__ Y, const double* __restrict__ coef,
                              double* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double xs = 0.0;
#pragma unroll
  for (int a = 0; a < K; ++a) xs += coef[a] * Y[(size_t)a * n + i];
  x[i] = xs;
}
// the stored product of a new correction: w = b - r (= A x for r = b - A x)
__global__ void guess_store(int n, const double* __restrict__ x, const double* __restrict__ b,
                            const double* __restrict__ r, double* __restrict__ y, double* __restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = x[i];
  w[i] = b[i] - r[i];
}

}  // namespace k
}  // namespace nds
