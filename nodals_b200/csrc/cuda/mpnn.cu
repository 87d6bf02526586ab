// Learned pressure-correction stage: a message-passing network on the face
// graph of the P0 pressure cells (no reference counterpart).  It is an extra
// flexible-preconditioner stage ahead of the AMG V-cycle inside FGMRES (the
// V-cycle it precedes: gpu/serial_cuda/h8_main_base.cu:557-564).
//
// Network (width H = 64, 3 message-passing layers), for a residual v on a
// graph with face neighbours N(i) and edge weights e_ij = a_ij / sqrt(a_ii
// a_jj) (the Jacobi-scaled pressure operator), per graph segment s:
//   q_i = v_i / sqrt(a_ii),  sigma_s = rms of q over the segment,
//   s_i = q_i / sigma_s,     f_i = (s_i, sum_j e_ij s_j)
//   h0_i = relu(We f_i + be)                          (CUDA cores)
//   h^l_i = relu(W_l [h^{l-1}_i ; sum_j e_ij h^{l-1}_j] + b_l),  l = 1..3
//                                                     (tcgen05 BF16 GEMM, F32 in TMEM)
//   out_i = wd . h3_i + bd + cs s_i
//   z_i = sigma_s out_i / sqrt(a_ii)
// Activations are stored in BF16; every GEMM accumulates in FP32.
// Training minimises, per segment, sum_i (out_i - t_i)^2 / sum_i t_i^2 with
// t_i = x_i sqrt(a_ii) / sigma_s for pairs (v, x) of pressure-correction
// right-hand sides and solutions: the diagonal-weighted error of z against x.
//
// Layer kernel (forward): persistent CTAs of 128 threads, one 128-row tile at
// a time: each thread gathers its row's own features and its neighbours'
// (L2-resident under the mesh numbering), writes the row [h_i ; m_i] as BF16
// into the A tile (canonical no-swizzle layout), one thread issues 8 MMAs
// (M = 128, N = 64, K = 16) against the weight tile kept in shared memory,
// the accumulator (128 lanes x 64 columns of TMEM) is read back with
// tcgen05.ld for the bias + ReLU epilogue.  Backward uses the same tiles:
// dX = delta W (M 128, N 128, K 64) and dW^T += X^T delta (M 128, N 64,
// K = the 128 nodes of the tile, both operands read MN-major from the same
// shared-memory tiles), accumulated in TMEM over all tiles of a CTA.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../capi_internal.hpp"
#include "common.cuh"
#include "mpnn.hpp"
#include "tc.cuh"

namespace nds {
namespace mp {

constexpr int kH = 64;         // hidden width
constexpr int kX = 2 * kH;     // dense-layer input width [h ; m]
constexpr int kTile = 128;     // rows per tile (= threads per CTA)
constexpr uint64_t kWaitNs = 2000000000ull;  // bound of every mbarrier wait: 2 s of wall time

// parameter layout (FP32 master copy; gradients use the same layout)
constexpr int OFF_WE = 0, OFF_BE = 128;
__host__ __device__ constexpr int off_w(int l) { return 192 + (l - 1) * (kH * kX + kH); }
__host__ __device__ constexpr int off_b(int l) { return off_w(l) + kH * kX; }
constexpr int OFF_WD = 192 + 3 * (kH * kX + kH), OFF_BD = OFF_WD + kH, OFF_CS = OFF_BD + 1;
constexpr int kNParam = OFF_CS + 1;
static_assert(kNParam == NDS_MPNN_NPARAM, "parameter count");

// fixed-order block partials (one row of NV doubles per block) and their sum
template <int NV>
__device__ __forceinline__ void write_partials(double (&v)[NV], double* part) {
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) part[(size_t)blockIdx.x * NV + k] = v[k];
}
template <int NV>
__global__ void reduce_partials(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += part[(size_t)b * NV + k];
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = v[k];
}

// canonical no-swizzle K-major tile: rows r (8-row groups at sbo bytes),
// 16-byte K chunks c at 128 bytes
__device__ __forceinline__ uint32_t tile_off(int r, int c, int sbo) { return (r >> 3) * sbo + c * 128 + (r & 7) * 16; }

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ void unpack8(const uint4& u, float (&f)[8]) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float2 t = __bfloat1622float2(h[q]);
    f[2 * q] = t.x;
    f[2 * q + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
  uint4 u;
  u.x = pack2(f[0], f[1]);
  u.y = pack2(f[2], f[3]);
  u.z = pack2(f[4], f[5]);
  u.w = pack2(f[6], f[7]);
  return u;
}
__device__ __forceinline__ int seg_of(int i, const int32_t* __restrict__ seg_off, int nseg) {
  int s = 0;
  while (s + 1 < nseg && i >= seg_off[s + 1]) ++s;
  return s;
}

// ---------------------------------------------------------------------------
// input: q = v dscale, sigma per segment, f = (s, sum e s)
// ---------------------------------------------------------------------------
// partials of (v dscale)^2 over [lo, hi)
__global__ void __launch_bounds__(kBlock) seg_sq(int lo, int hi, const float* __restrict__ v,
                                                 const float* __restrict__ dscale, double* __restrict__ part) {
  double acc[1] = {0.0};
  for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x) {
    const double q = (double)v[i] * (double)dscale[i];
    acc[0] += q * q;
  }
  write_partials<1>(acc, part);
}
// sigma[s] = sqrt(sum / count) (1 when the segment is zero)
__global__ void seg_sigma(const double* __restrict__ part, int nblocks, int count, float* __restrict__ sigma) {
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v[0] += part[b];
  block_sum<1>(v);
  if (threadIdx.x == 0) {
    const double s = sqrt(v[0] / (double)max(count, 1));
    *sigma = (s > 0.0 && isfinite(s)) ? (float)s : 1.0f;
  }
}
// s_i = v_i dscale_i / sigma
__global__ void scaled_input(int n, const float* __restrict__ v, const float* __restrict__ dscale,
                             const float* __restrict__ sigma, const int32_t* __restrict__ seg_off, int nseg,
                             float* __restrict__ s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  s[i] = v[i] * dscale[i] / sigma[seg_of(i, seg_off, nseg)];
}
// f_i = (s_i, sum_j e_ij s_j).  A neighbour index outside [-1, n) is an
// error of the caller's graph: it sets err bit 2 and is skipped (the layer
// kernels skip such entries too).
__global__ void features(int n, const float* __restrict__ s, const int32_t* __restrict__ nbr,
                         const float* __restrict__ ew, float2* __restrict__ f, int* __restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float m = 0.f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int j = nbr[4 * (size_t)i + k];
    if (j >= n || j < -1) {
      atomicOr(err, 2);
      continue;
    }
    if (j >= 0) m += ew[4 * (size_t)i + k] * s[j];
  }
  f[i] = make_float2(s[i], m);
}

// ---------------------------------------------------------------------------
// tile assembly shared by the forward and backward layer kernels: row r of
// the A tile = [h_i ; sum_j e_ij h_j] in BF16.  Layer 1 recomputes h0 from f
// (encoder in FP32, rounded to BF16 like a stored activation).
// ---------------------------------------------------------------------------
struct LayerIn {
  int n;
  const int32_t* nbr;
  const float* ew;
  const float2* f;                 // layer 1
  const __nv_bfloat16* hin;        // layers 2, 3
};
template <bool ENC>
__device__ __forceinline__ void encoder_row(float2 fi, const float* __restrict__ s_we, const float* __restrict__ s_be,
                                            float (&h)[kH]) {
#pragma unroll
  for (int k = 0; k < kH; ++k) {
    const float v = fmaf(s_we[2 * k], fi.x, fmaf(s_we[2 * k + 1], fi.y, s_be[k]));
    h[k] = __bfloat162float(__float2bfloat16_rn(fmaxf(v, 0.f)));
  }
}
template <bool ENC>
__device__ void build_row(const LayerIn& in, int row, uint8_t* __restrict__ X, int r, const float* __restrict__ s_we,
                          const float* __restrict__ s_be) {
  float m[kH];
#pragma unroll
  for (int k = 0; k < kH; ++k) m[k] = 0.f;
  if (row >= in.n) {
    const uint4 z = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int c = 0; c < 16; ++c) *reinterpret_cast<uint4*>(X + tile_off(r, c, 2048)) = z;
    return;
  }
  if (ENC) {
    float h[kH];
    encoder_row<true>(in.f[row], s_we, s_be, h);
#pragma unroll
    for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(X + tile_off(r, c, 2048)) = pack8(h + 8 * c);
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
      const int j = in.nbr[4 * (size_t)row + k];
      if (j < 0 || j >= in.n) continue;
      const float w = in.ew[4 * (size_t)row + k];
      encoder_row<true>(in.f[j], s_we, s_be, h);
#pragma unroll
      for (int q = 0; q < kH; ++q) m[q] = fmaf(w, h[q], m[q]);
    }
  } else {
    const uint4* self = reinterpret_cast<const uint4*>(in.hin + (size_t)row * kH);
#pragma unroll
    for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(X + tile_off(r, c, 2048)) = self[c];
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
      const int j = in.nbr[4 * (size_t)row + k];
      if (j < 0 || j >= in.n) continue;
      const float w = in.ew[4 * (size_t)row + k];
      const uint4* hj = reinterpret_cast<const uint4*>(in.hin + (size_t)j * kH);
      uint4 u[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) u[c] = hj[c];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        float t[8];
        unpack8(u[c], t);
#pragma unroll
        for (int q = 0; q < 8; ++q) m[8 * c + q] = fmaf(w, t[q], m[8 * c + q]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(X + tile_off(r, 8 + c, 2048)) = pack8(m + 8 * c);
}

// ---------------------------------------------------------------------------
// forward layer
// ---------------------------------------------------------------------------
struct FwdArgs {
  LayerIn in;
  const __nv_bfloat16* W;   // [64][128] row-major (out x in)
  const float* params;      // FP32 parameters (encoder, bias, decoder)
  int layer;                // 1..3
  __nv_bfloat16* hout;      // h^layer (null: not stored)
  // decoder (layer 3 with dec = 1)
  float* out;               // normalized output (may be null)
  float* z;                 // z = out sigma dscale (may be null)
  const float* dscale;
  const float* sigma;
  const int32_t* seg_off;
  int nseg;
  int* err;
};
constexpr int kFwdSmem = 16384 + 32768 + 1024;  // W tile, X tile, alignment slack

template <bool ENC, bool DEC>
__global__ void __launch_bounds__(kTile) layer_fwd(FwdArgs a) {
  extern __shared__ uint8_t dsm[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));
  uint8_t* Wsm = base;
  uint8_t* Xsm = base + 16384;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tbase_s;
  __shared__ float s_we[2 * kH], s_be[kH], s_b[kH], s_wd[kH];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // weight tile: W[o][i] as B (N = 64 rows o, K = 128), K-major
  for (int e = tid; e < kH * 16; e += kTile) {
    const int o = e >> 4, c = e & 15;
    *reinterpret_cast<uint4*>(Wsm + tile_off(o, c, 2048)) = reinterpret_cast<const uint4*>(a.W)[e];
  }
  for (int q = tid; q < kH; q += kTile) {
    s_b[q] = a.params[off_b(a.layer) + q];
    s_be[q] = a.params[OFF_BE + q];
    s_wd[q] = a.params[OFF_WD + q];
  }
  for (int q = tid; q < 2 * kH; q += kTile) s_we[q] = a.params[OFF_WE + q];
  if (warp == 0) {
    tc::tmem_alloc(&tbase_s, 64);
    tc::tmem_relinquish();
  }
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tbase_s;
  constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 64, 0, 0);
  const uint32_t xs = tc::smem_addr(Xsm), ws = tc::smem_addr(Wsm);
  const float bd = a.params[OFF_BD], cs = a.params[OFF_CS];
  uint32_t phase = 0;
  const int ntiles = (a.in.n + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row = tile * kTile + tid;
    build_row<ENC>(a.in, row, Xsm, tid, s_we, s_be);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 8; ++s)
        tc::mma_bf16(tbase, tc::sdesc(xs + 256 * s, 128, 2048), tc::sdesc(ws + 256 * s, 128, 2048), idesc, s > 0);
      tc::mma_commit(&mbar);
    }
    const bool ok = tc::mbar_wait_bounded(&mbar, phase, kWaitNs);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(a.err, 1);
      tc::mbar_wait_bounded(&mbar, phase ^ 1u, kWaitNs);  // the MMAs of this tile, if still running
      break;
    }
    tc::fence_after_sync();
    float acc[kH];
    {
      float t[32];
      tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16), t);
#pragma unroll
      for (int q = 0; q < 32; ++q) acc[q] = t[q];
      tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + 32, t);
#pragma unroll
      for (int q = 0; q < 32; ++q) acc[32 + q] = t[q];
    }
    if (row < a.in.n) {
      float h[kH];
#pragma unroll
      for (int q = 0; q < kH; ++q) h[q] = __bfloat162float(__float2bfloat16_rn(fmaxf(acc[q] + s_b[q], 0.f)));
      if (a.hout) {
        uint4* dst = reinterpret_cast<uint4*>(a.hout + (size_t)row * kH);
#pragma unroll
        for (int c = 0; c < 8; ++c) dst[c] = pack8(h + 8 * c);
      }
      if (DEC) {
        float o = bd;
#pragma unroll
        for (int q = 0; q < kH; ++q) o = fmaf(s_wd[q], h[q], o);
        const float si = a.in.f[row].x;
        o = fmaf(cs, si, o);
        if (a.out) a.out[row] = o;
        if (a.z) a.z[row] = o * a.sigma[seg_of(row, a.seg_off, a.nseg)] * a.dscale[row];
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 64);
  (void)lane;
}

// ---------------------------------------------------------------------------
// backward layer: delta = dh (.) [h > 0]; dX = delta W -> (dh_self, dm);
// dW^T += X^T delta and db += sum delta per CTA (partials)
// ---------------------------------------------------------------------------
struct BwdArgs {
  LayerIn in;
  const __nv_bfloat16* W;      // [64][128] row-major
  const float* params;
  int layer;
  const float* dh;             // [n][64] gradient w.r.t. h^layer
  const __nv_bfloat16* h;      // [n][64] h^layer (ReLU mask)
  float* dself;                // [n][64] gradient w.r.t. h^{layer-1} (own part)
  float* dm;                   // [n][64] gradient w.r.t. m^{layer-1}
  float* wpart;                // [gridDim.x][128][64]: dW^T partials
  float* bpart;                // [gridDim.x][64]: db partials
  int* err;
};
constexpr int kBwdSmem = 16384 + 32768 + 16384 + 1024 + 40000;  // W^T, X, delta tiles; slack limits 2 CTAs / SM

template <bool ENC>
__global__ void __launch_bounds__(kTile) layer_bwd(BwdArgs a) {
  extern __shared__ uint8_t dsm[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dsm) + 1023) & ~uintptr_t(1023));
  uint8_t* WTsm = base;            // B of dX: N = 128 (i), K = 64 (o), K-major, 8-row groups at 1024 B
  uint8_t* Xsm = base + 16384;     // [128 nodes][128] K-major (groups at 2048 B)
  uint8_t* Dsm = base + 49152;     // [128 nodes][64] K-major (groups at 1024 B)
  __shared__ uint64_t mbar;
  __shared__ uint32_t tbase_s;
  __shared__ float s_we[2 * kH], s_be[kH];
  const int tid = threadIdx.x, warp = tid >> 5;

  for (int e = tid; e < kX * 8; e += kTile) {
    // W^T[i][o]: row i, 16-byte chunk c covers o = 8c..8c+7
    const int i = e >> 3, c = e & 7;
    float t[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) t[q] = __bfloat162float(a.W[(size_t)(8 * c + q) * kX + i]);
    *reinterpret_cast<uint4*>(WTsm + tile_off(i, c, 1024)) = pack8(t);
  }
  for (int q = tid; q < kH; q += kTile) s_be[q] = a.params[OFF_BE + q];
  for (int q = tid; q < 2 * kH; q += kTile) s_we[q] = a.params[OFF_WE + q];
  if (warp == 0) {
    tc::tmem_alloc(&tbase_s, 256);
    tc::tmem_relinquish();
  }
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tbase_s;
  constexpr uint32_t idx_dx = tc::idesc_bf16_f32(128, 128, 0, 0);
  constexpr uint32_t idx_dw = tc::idesc_bf16_f32(128, 64, 1, 1);
  const uint32_t xs = tc::smem_addr(Xsm), ds = tc::smem_addr(Dsm), wts = tc::smem_addr(WTsm);
  float dbacc[kH];
#pragma unroll
  for (int q = 0; q < kH; ++q) dbacc[q] = 0.f;
  uint32_t phase = 0;
  bool first = true, aborted = false;
  const int ntiles = (a.in.n + kTile - 1) / kTile;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row = tile * kTile + tid;
    {
      float d[kH];
      if (row < a.in.n) {
        const float4* g = reinterpret_cast<const float4*>(a.dh + (size_t)row * kH);
        const uint4* hh = reinterpret_cast<const uint4*>(a.h + (size_t)row * kH);
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          float hv[8];
          unpack8(hh[c], hv);
          const float4 g0 = g[2 * c], g1 = g[2 * c + 1];
          const float gv[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
#pragma unroll
          for (int q = 0; q < 8; ++q) d[8 * c + q] = hv[q] > 0.f ? gv[q] : 0.f;
        }
      } else {
#pragma unroll
        for (int q = 0; q < kH; ++q) d[q] = 0.f;
      }
#pragma unroll
      for (int q = 0; q < kH; ++q) {
        d[q] = __bfloat162float(__float2bfloat16_rn(d[q]));
        dbacc[q] += d[q];
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) *reinterpret_cast<uint4*>(Dsm + tile_off(tid, c, 1024)) = pack8(d + 8 * c);
    }
    build_row<ENC>(a.in, row, Xsm, tid, s_we, s_be);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < 4; ++s)
        tc::mma_bf16(tbase, tc::sdesc(ds + 256 * s, 128, 1024), tc::sdesc(wts + 256 * s, 128, 1024), idx_dx, s > 0);
      // dW^T (M = i, N = o, K = nodes): both operands MN-major views of the tiles
#pragma unroll
      for (int s = 0; s < 8; ++s)
        tc::mma_bf16(tbase + 128, tc::sdesc(xs + 4096 * s, 2048, 128), tc::sdesc(ds + 2048 * s, 1024, 128), idx_dw,
                     (first && s == 0) ? 0u : 1u);
      tc::mma_commit(&mbar);
    }
    first = false;
    const bool ok = tc::mbar_wait_bounded(&mbar, phase, kWaitNs);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(a.err, 1);
      tc::mbar_wait_bounded(&mbar, phase ^ 1u, kWaitNs);
      aborted = true;
      break;
    }
    tc::fence_after_sync();
    // tcgen05.ld is a warp-collective (.sync.aligned): every lane of the warp
    // executes the same loads, rows past n only skip the stores
#pragma unroll
    for (int part = 0; part < 4; ++part) {
      float t[32];
      tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + 32 * part, t);
      if (row < a.in.n) {
        float* dst = part < 2 ? a.dself + (size_t)row * kH + 32 * part : a.dm + (size_t)row * kH + 32 * (part - 2);
#pragma unroll
        for (int q = 0; q < 32; q += 4) *reinterpret_cast<float4*>(dst + q) = make_float4(t[q], t[q + 1], t[q + 2], t[q + 3]);
      }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  // dW^T partial of this CTA: thread (warp, lane) holds row i = 32 warp + lane
  float* wp = a.wpart + (size_t)blockIdx.x * kX * kH;
  if (first || aborted) {
    for (int q = tid; q < kX * kH; q += kTile) wp[q] = 0.f;
  } else {
    float t[32];
    const int i = 32 * warp + (tid & 31);
#pragma unroll
    for (int part = 0; part < 2; ++part) {
      tc::tmem_ld32(tbase + ((uint32_t)(32 * warp) << 16) + 128 + 32 * part, t);
#pragma unroll
      for (int q = 0; q < 32; ++q) wp[(size_t)i * kH + 32 * part + q] = t[q];
    }
  }
  // db partial: block sum of the per-thread sums, fixed order
  {
    __shared__ float red[kTile];
    for (int q = 0; q < kH; ++q) {
      red[tid] = dbacc[q];
      __syncthreads();
      if (tid == 0) {
        float s = 0.f;
        for (int r = 0; r < kTile; ++r) s += red[r];
        a.bpart[(size_t)blockIdx.x * kH + q] = s;
      }
      __syncthreads();
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 256);
}

// dh_prev_i = dself_i + sum_j e_ij dm_j  (the face graph and e are symmetric)
__global__ void scatter_bwd(int n, const int32_t* __restrict__ nbr, const float* __restrict__ ew,
                            const float* __restrict__ dself, const float* __restrict__ dm, float* __restrict__ dh) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t >> 4, c = t & 15;  // 16 threads per row, 4 values each
  if (i >= n) return;
  float4 s = reinterpret_cast<const float4*>(dself + (size_t)i * kH)[c];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int j = nbr[4 * (size_t)i + k];
    if (j < 0 || j >= n) continue;
    const float w = ew[4 * (size_t)i + k];
    const float4 d = reinterpret_cast<const float4*>(dm + (size_t)j * kH)[c];
    s.x = fmaf(w, d.x, s.x);
    s.y = fmaf(w, d.y, s.y);
    s.z = fmaf(w, d.z, s.z);
    s.w = fmaf(w, d.w, s.w);
  }
  reinterpret_cast<float4*>(dh + (size_t)i * kH)[c] = s;
}

// encoder backward: delta0 = dh0 (.) [h0 > 0]; partials of dWe (64 x 2), dbe (64)
__global__ void __launch_bounds__(kBlock) encoder_bwd(int n, const float2* __restrict__ f, const float* __restrict__ dh0,
                                                      const float* __restrict__ params, double* __restrict__ part) {
  __shared__ float s_we[2 * kH], s_be[kH];
  for (int q = threadIdx.x; q < 2 * kH; q += blockDim.x) s_we[q] = params[OFF_WE + q];
  for (int q = threadIdx.x; q < kH; q += blockDim.x) s_be[q] = params[OFF_BE + q];
  __syncthreads();
  double acc[3 * kH];
#pragma unroll
  for (int q = 0; q < 3 * kH; ++q) acc[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float2 fi = f[i];
    for (int k = 0; k < kH; ++k) {
      const float v = fmaf(s_we[2 * k], fi.x, fmaf(s_we[2 * k + 1], fi.y, s_be[k]));
      if (v > 0.f) {
        const double d = dh0[(size_t)i * kH + k];
        acc[2 * k] += d * fi.x;
        acc[2 * k + 1] += d * fi.y;
        acc[2 * kH + k] += d;
      }
    }
  }
  write_partials<3 * kH>(acc, part);
}

// ---------------------------------------------------------------------------
// loss and decoder backward
// ---------------------------------------------------------------------------
// per segment: sum t^2 and sum (out - t)^2 over [lo, hi) with t = x dscale / sigma
__global__ void __launch_bounds__(kBlock) seg_loss(int lo, int hi, const float* __restrict__ out,
                                                   const float* __restrict__ x, const float* __restrict__ dscale,
                                                   const float* __restrict__ sigma, double* __restrict__ part) {
  double acc[2] = {0.0, 0.0};
  const double inv_s = 1.0 / (double)*sigma;
  for (int i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi; i += gridDim.x * blockDim.x) {
    // x / sqrt(a_ii) in the network's scaling: t = x sqrt(a_ii) / sigma = x / (dscale sigma)
    const double t = (double)x[i] / (double)dscale[i] * inv_s;
    const double d = (double)out[i] - t;
    acc[0] += t * t;
    acc[1] += d * d;
  }
  write_partials<2>(acc, part);
}
// dout = coef_s (out - t); partials of dwd (64), dbd, dcs; dh3 = dout wd
__global__ void __launch_bounds__(kBlock) decoder_bwd(int n, const float* __restrict__ out, const float* __restrict__ x,
                                                      const float* __restrict__ dscale, const float* __restrict__ sigma,
                                                      const int32_t* __restrict__ seg_off, int nseg,
                                                      const double* __restrict__ coef, const __nv_bfloat16* __restrict__ h3,
                                                      const float2* __restrict__ f, const float* __restrict__ params,
                                                      float* __restrict__ dh3, double* __restrict__ part) {
  double acc[kH + 2];
#pragma unroll
  for (int q = 0; q < kH + 2; ++q) acc[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int s = seg_of(i, seg_off, nseg);
    const double t = (double)x[i] / ((double)dscale[i] * (double)sigma[s]);
    const float g = (float)(coef[s] * ((double)out[i] - t));
    const uint4* hh = reinterpret_cast<const uint4*>(h3 + (size_t)i * kH);
    float4* d = reinterpret_cast<float4*>(dh3 + (size_t)i * kH);
    for (int c = 0; c < 8; ++c) {
      float hv[8];
      unpack8(hh[c], hv);
      float o[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        acc[8 * c + q] += (double)g * hv[q];
        o[q] = g * params[OFF_WD + 8 * c + q];
      }
      d[2 * c] = make_float4(o[0], o[1], o[2], o[3]);
      d[2 * c + 1] = make_float4(o[4], o[5], o[6], o[7]);
    }
    acc[kH] += g;
    acc[kH + 1] += (double)g * f[i].x;
  }
  write_partials<kH + 2>(acc, part);
}
// the same from a gradient dz with respect to z = out sigma dscale:
// dout = dz sigma dscale
__global__ void __launch_bounds__(kBlock) decoder_bwd_dz(int n, const float* __restrict__ dz,
                                                         const float* __restrict__ dscale,
                                                         const float* __restrict__ sigma,
                                                         const int32_t* __restrict__ seg_off, int nseg,
                                                         const __nv_bfloat16* __restrict__ h3,
                                                         const float2* __restrict__ f, const float* __restrict__ params,
                                                         float* __restrict__ dh3, double* __restrict__ part) {
  double acc[kH + 2];
#pragma unroll
  for (int q = 0; q < kH + 2; ++q) acc[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = dz[i] * sigma[seg_of(i, seg_off, nseg)] * dscale[i];
    const uint4* hh = reinterpret_cast<const uint4*>(h3 + (size_t)i * kH);
    float4* d = reinterpret_cast<float4*>(dh3 + (size_t)i * kH);
    for (int c = 0; c < 8; ++c) {
      float hv[8];
      unpack8(hh[c], hv);
      float o[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        acc[8 * c + q] += (double)g * hv[q];
        o[q] = g * params[OFF_WD + 8 * c + q];
      }
      d[2 * c] = make_float4(o[0], o[1], o[2], o[3]);
      d[2 * c + 1] = make_float4(o[4], o[5], o[6], o[7]);
    }
    acc[kH] += g;
    acc[kH + 1] += (double)g * f[i].x;
  }
  write_partials<kH + 2>(acc, part);
}
// out[c] = sum_r part[r][c] (fixed order), into grad at offset (FP32)
__global__ void reduce_rows_f(const float* __restrict__ part, int rows, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double s = 0.0;
  for (int r = 0; r < rows; ++r) s += part[(size_t)r * cols + c];
  out[c] = (float)s;
}
__global__ void reduce_rows_d(const double* __restrict__ part, int rows, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  double s = 0.0;
  for (int r = 0; r < rows; ++r) s += part[(size_t)r * cols + c];
  out[c] = (float)s;
}
// dW[o][i] = dW^T[i][o]
__global__ void transpose_into(const float* __restrict__ wt, float* __restrict__ w) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= kH * kX) return;
  const int o = e / kX, i = e % kX;
  w[e] = wt[(size_t)i * kH + o];
}

// Adam (bias-corrected), then the BF16 weight copies
__global__ void adam(int np, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                     float* __restrict__ m2, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
}
__global__ void to_bf16(int n, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = __float2bfloat16_rn(a[i]);
}

}  // namespace mp

// ============================================================================
// host side
// ============================================================================
namespace {
template <class T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  Dev() = default;
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  ~Dev() {
    if (p) cudaFree(p);
  }
  void alloc(size_t m) {
    if (p) cudaFree(p);
    p = nullptr;
    n = m;
    if (m) NDS_CUDA(cudaMalloc((void**)&p, m * sizeof(T)));
  }
};
int sm_count() {
  static int n = [] {
    int d = 0, c = 148;
    if (cudaGetDevice(&d) == cudaSuccess) cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, d);
    return c;
  }();
  return n;
}
}  // namespace

// The network's device state: parameters (FP32 master, BF16 weight copies),
// Adam moments, gradients and the work arrays of graphs up to n_max nodes.
struct MpnnImpl {
  int n_max = 0;
  cudaStream_t st = nullptr;
  Dev<float> params, grads, m1, m2;
  Dev<__nv_bfloat16> wbf;              // 3 x [64][128]
  Dev<float> s, out, sigma, dh, dself, dm, wpart, bpart, wtmp;
  Dev<float2> f;
  Dev<__nv_bfloat16> h1, h2, h3;
  Dev<double> dpart, segd;
  Dev<int32_t> seg_dev;
  Dev<int> err;
  int fwd_grid = 0, bwd_grid = 0;
  bool training = false;

  MpnnImpl(int nmax, bool train, cudaStream_t stream) : n_max(nmax), st(stream), training(train) {
    params.alloc(mp::kNParam);
    wbf.alloc(3 * mp::kH * mp::kX);
    const size_t n = (size_t)std::max(nmax, 1);
    s.alloc(n);
    out.alloc(n);
    f.alloc(n);
    h1.alloc(n * mp::kH);
    h2.alloc(n * mp::kH);
    sigma.alloc(64);
    seg_dev.alloc(65);
    segd.alloc(64 * 2);
    dpart.alloc((size_t)kMaxBlocks * (3 * mp::kH));
    err.alloc(1);
    NDS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    fwd_grid = 4 * sm_count();
    bwd_grid = 2 * sm_count();
    if (train) {
      grads.alloc(mp::kNParam);
      m1.alloc(mp::kNParam);
      m2.alloc(mp::kNParam);
      NDS_CUDA(cudaMemsetAsync(m1.p, 0, sizeof(float) * mp::kNParam, st));
      NDS_CUDA(cudaMemsetAsync(m2.p, 0, sizeof(float) * mp::kNParam, st));
      h3.alloc(n * mp::kH);
      dh.alloc(n * mp::kH);
      dself.alloc(n * mp::kH);
      dm.alloc(n * mp::kH);
      wpart.alloc((size_t)bwd_grid * mp::kX * mp::kH);
      bpart.alloc((size_t)bwd_grid * mp::kH);
      wtmp.alloc((size_t)mp::kX * mp::kH);
    }
    NDS_CUDA(cudaFuncSetAttribute(mp::layer_fwd<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mp::kFwdSmem));
    NDS_CUDA(cudaFuncSetAttribute(mp::layer_fwd<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mp::kFwdSmem));
    NDS_CUDA(cudaFuncSetAttribute(mp::layer_fwd<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mp::kFwdSmem));
    NDS_CUDA(cudaFuncSetAttribute(mp::layer_bwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mp::kBwdSmem));
    NDS_CUDA(cudaFuncSetAttribute(mp::layer_bwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mp::kBwdSmem));
  }
  static constexpr int kMaxBlocks = 1184;

  void set_params(const float* host) {
    NDS_CUDA(cudaMemcpyAsync(params.p, host, sizeof(float) * mp::kNParam, cudaMemcpyHostToDevice, st));
    refresh_bf16();
  }
  void refresh_bf16() {
    for (int l = 1; l <= 3; ++l) {
      mp::to_bf16<<<grid_for(mp::kH * mp::kX), kBlock, 0, st>>>(mp::kH * mp::kX, params.p + mp::off_w(l),
                                                               wbf.p + (size_t)(l - 1) * mp::kH * mp::kX);
      NDS_LAUNCH();
    }
  }
  void check_err() {
    int e = 0;
    NDS_CUDA(cudaMemcpyAsync(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    NDS_CUDA(cudaStreamSynchronize(st));
    NDS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    if (e & 2) throw std::runtime_error("learned stage: a neighbour index of the graph is out of range");
    if (e) throw std::runtime_error("learned stage: a tensor-core wait ran out (error flag set)");
  }
  std::vector<int32_t> seg_host;  // segment offsets last uploaded to seg_dev
  int seg_n = -1;
  void upload_segments(const std::vector<int32_t>& seg) {
    if (seg.size() > 65) throw std::runtime_error("learned stage: at most 64 segments");
    seg_host = seg;
    seg_n = seg.back();
    NDS_CUDA(cudaMemcpyAsync(seg_dev.p, seg_host.data(), sizeof(int32_t) * seg_host.size(), cudaMemcpyHostToDevice, st));
    NDS_CUDA(cudaStreamSynchronize(st));
  }
  // sigma per segment and the features f (s kept in this->s); seg must be
  // the offsets in seg_dev
  void inputs(const nds_mpnn_graph& g, const float* v, const std::vector<int32_t>& seg) {
    const int nseg = (int)seg.size() - 1;
    for (int q = 0; q < nseg; ++q) {
      const int lo = seg[(size_t)q], hi = seg[(size_t)q + 1];
      const int gb = std::min(grid_for(std::max(hi - lo, 1)), kMaxBlocks);
      mp::seg_sq<<<gb, kBlock, 0, st>>>(lo, hi, v, g.dscale, dpart.p);
      NDS_LAUNCH();
      mp::seg_sigma<<<1, kBlock, 0, st>>>(dpart.p, gb, hi - lo, sigma.p + q);
      NDS_LAUNCH();
    }
    mp::scaled_input<<<grid_for(g.n), kBlock, 0, st>>>(g.n, v, g.dscale, sigma.p, seg_dev.p, nseg, s.p);
    NDS_LAUNCH();
    mp::features<<<grid_for(g.n), kBlock, 0, st>>>(g.n, s.p, g.nbr, g.ew, f.p, err.p);
    NDS_LAUNCH();
  }
  mp::FwdArgs fwd_args(const nds_mpnn_graph& g, int layer, int nseg) {
    mp::FwdArgs a{};
    a.in = mp::LayerIn{g.n, g.nbr, g.ew, f.p, nullptr};
    a.W = wbf.p + (size_t)(layer - 1) * mp::kH * mp::kX;
    a.params = params.p;
    a.layer = layer;
    a.dscale = g.dscale;
    a.sigma = sigma.p;
    a.seg_off = seg_dev.p;
    a.nseg = nseg;
    a.err = err.p;
    return a;
  }
  int tiles(int n) const { return (n + mp::kTile - 1) / mp::kTile; }
  // z = N(v); with training, h1..h3 and out are kept for backward
  void forward(const nds_mpnn_graph& g, const float* v, float* z, const std::vector<int32_t>& seg, bool upload) {
    if (g.n > n_max) throw std::runtime_error("learned stage: graph larger than the work arrays");
    if (upload && seg != seg_host) upload_segments(seg);
    const int nseg = (int)seg.size() - 1;
    inputs(g, v, seg);
    const int grid = std::max(1, std::min(fwd_grid, tiles(g.n)));
    mp::FwdArgs a1 = fwd_args(g, 1, nseg);
    a1.hout = h1.p;
    mp::layer_fwd<true, false><<<grid, mp::kTile, mp::kFwdSmem, st>>>(a1);
    NDS_LAUNCH();
    mp::FwdArgs a2 = fwd_args(g, 2, nseg);
    a2.in.hin = h1.p;
    a2.hout = h2.p;
    mp::layer_fwd<false, false><<<grid, mp::kTile, mp::kFwdSmem, st>>>(a2);
    NDS_LAUNCH();
    mp::FwdArgs a3 = fwd_args(g, 3, nseg);
    a3.in.hin = h2.p;
    a3.hout = training ? h3.p : nullptr;
    a3.out = out.p;
    a3.z = z;
    mp::layer_fwd<false, true><<<grid, mp::kTile, mp::kFwdSmem, st>>>(a3);
    NDS_LAUNCH();
  }
  // forward, loss, backward: gradients in grads; returns the mean segment loss
  double loss_backward(const nds_mpnn_graph& g, const float* v, const float* x, const std::vector<int32_t>& seg) {
    if (!training) throw std::runtime_error("learned stage: created without training buffers");
    const int nseg = (int)seg.size() - 1;
    forward(g, v, nullptr, seg, true);
    // segment sums of t^2 and (out - t)^2
    std::vector<double> coef((size_t)nseg), sums(2 * (size_t)nseg);
    for (int q = 0; q < nseg; ++q) {
      const int lo = seg[(size_t)q], hi = seg[(size_t)q + 1];
      const int gb = std::min(grid_for(std::max(hi - lo, 1)), kMaxBlocks);
      mp::seg_loss<<<gb, kBlock, 0, st>>>(lo, hi, out.p, x, g.dscale, sigma.p + q, dpart.p);
      NDS_LAUNCH();
      mp::reduce_partials<2><<<1, kBlock, 0, st>>>(dpart.p, gb, segd.p + 2 * q);
      NDS_LAUNCH();
    }
    NDS_CUDA(cudaMemcpyAsync(sums.data(), segd.p, sizeof(double) * 2 * nseg, cudaMemcpyDeviceToHost, st));
    NDS_CUDA(cudaStreamSynchronize(st));
    double loss = 0.0;
    for (int q = 0; q < nseg; ++q) {
      const double tt = std::max(sums[2 * (size_t)q], 1e-300);
      loss += sums[2 * (size_t)q + 1] / tt / nseg;
      coef[(size_t)q] = 2.0 / (tt * nseg);
    }
    NDS_CUDA(cudaMemcpyAsync(segd.p, coef.data(), sizeof(double) * nseg, cudaMemcpyHostToDevice, st));
    const int rg = std::min(grid_for(g.n), kMaxBlocks);
    mp::decoder_bwd<<<rg, kBlock, 0, st>>>(g.n, out.p, x, g.dscale, sigma.p, seg_dev.p, nseg, segd.p, h3.p, f.p,
                                           params.p, dh.p, dpart.p);
    NDS_LAUNCH();
    layers_backward(g, rg);
    return loss;
  }
  // gradients from dL/dz of the last forward (which must have been run on
  // this graph with the training buffers)
  void backward_dz(const nds_mpnn_graph& g, const float* dz) {
    if (!training) throw std::runtime_error("learned stage: created without training buffers");
    const int nseg = (int)seg_host.size() - 1;
    const int rg = std::min(grid_for(g.n), kMaxBlocks);
    mp::decoder_bwd_dz<<<rg, kBlock, 0, st>>>(g.n, dz, g.dscale, sigma.p, seg_dev.p, nseg, h3.p, f.p, params.p, dh.p,
                                              dpart.p);
    NDS_LAUNCH();
    layers_backward(g, rg);
  }
  // decoder partials in dpart and dh3 in dh -> every parameter gradient
  void layers_backward(const nds_mpnn_graph& g, int rg) {
    mp::reduce_rows_d<<<1, 128, 0, st>>>(dpart.p, rg, mp::kH + 2, grads.p + mp::OFF_WD);
    NDS_LAUNCH();
    const int bgrid = std::max(1, std::min(bwd_grid, tiles(g.n)));
    const __nv_bfloat16* hs[4] = {nullptr, h1.p, h2.p, h3.p};
    for (int l = 3; l >= 1; --l) {
      mp::BwdArgs b{};
      b.in = mp::LayerIn{g.n, g.nbr, g.ew, f.p, l >= 2 ? hs[l - 1] : nullptr};
      b.W = wbf.p + (size_t)(l - 1) * mp::kH * mp::kX;
      b.params = params.p;
      b.layer = l;
      b.dh = dh.p;
      b.h = hs[l];
      b.dself = dself.p;
      b.dm = dm.p;
      b.wpart = wpart.p;
      b.bpart = bpart.p;
      b.err = err.p;
      if (l == 1) mp::layer_bwd<true><<<bgrid, mp::kTile, mp::kBwdSmem, st>>>(b);
      else mp::layer_bwd<false><<<bgrid, mp::kTile, mp::kBwdSmem, st>>>(b);
      NDS_LAUNCH();
      mp::reduce_rows_f<<<grid_for(mp::kX * mp::kH), kBlock, 0, st>>>(wpart.p, bgrid, mp::kX * mp::kH, wtmp.p);
      NDS_LAUNCH();
      mp::transpose_into<<<grid_for(mp::kX * mp::kH), kBlock, 0, st>>>(wtmp.p, grads.p + mp::off_w(l));
      NDS_LAUNCH();
      mp::reduce_rows_f<<<1, mp::kH, 0, st>>>(bpart.p, bgrid, mp::kH, grads.p + mp::off_b(l));
      NDS_LAUNCH();
      // gradient into h^{l-1} (h0 for l = 1)
      mp::scatter_bwd<<<grid_for((long long)g.n * 16), kBlock, 0, st>>>(g.n, g.nbr, g.ew, dself.p, dm.p, dh.p);
      NDS_LAUNCH();
    }
    mp::encoder_bwd<<<rg, kBlock, 0, st>>>(g.n, f.p, dh.p, params.p, dpart.p);
    NDS_LAUNCH();
    {
      // partial rows: [dWe (2 per unit, unit-major) ; dbe]
      mp::reduce_rows_d<<<1, 3 * mp::kH, 0, st>>>(dpart.p, rg, 3 * mp::kH, wtmp.p);
      NDS_LAUNCH();
      NDS_CUDA(cudaMemcpyAsync(grads.p + mp::OFF_WE, wtmp.p, sizeof(float) * 3 * mp::kH, cudaMemcpyDeviceToDevice, st));
    }
    check_err();
  }
  void adam_step(float lr, float b1, float b2, float eps, int step) {
    const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
    mp::adam<<<grid_for(mp::kNParam), kBlock, 0, st>>>(mp::kNParam, params.p, grads.p, m1.p, m2.p, lr, b1, b2, eps, c1,
                                                       c2);
    NDS_LAUNCH();
    refresh_bf16();
  }
};

void MpnnDeleter::operator()(MpnnImpl* m) const { delete m; }
MpnnPtr make_mpnn(int n_max, bool training, cudaStream_t st) {
  MpnnPtr m(new MpnnImpl(n_max, training, st));
  m->upload_segments({0, n_max});
  return m;
}
void mpnn_set_params(MpnnImpl& m, const float* host) {
  m.set_params(host);
  NDS_CUDA(cudaStreamSynchronize(m.st));
}
void mpnn_forward(MpnnImpl& m, const nds_mpnn_graph& g, const float* v, float* z) {
  if (g.n != m.seg_n) throw std::runtime_error("learned stage: graph size differs from the solver's");
  m.forward(g, v, z, m.seg_host, false);
}
void mpnn_check(MpnnImpl& m) { m.check_err(); }

}  // namespace nds

// ============================================================== C ABI
struct nds_mpnn {
  nds::MpnnPtr impl;
  cudaStream_t st = nullptr;
};

namespace {
int mfail(int code, const std::string& m) {
  nds::set_error(m);
  return code;
}
template <class F>
int mguard(F&& f) {
  try {
    f();
    return NDS_OK;
  } catch (const nds::CudaError& e) {
    return mfail(NDS_E_CUDA, e.what());
  } catch (const std::exception& e) {
    return mfail(NDS_E_SETUP, e.what());
  }
}
std::vector<int32_t> segs(int n, int nseg, const int32_t* seg_off) {
  std::vector<int32_t> s;
  if (nseg <= 0 || !seg_off) return {0, n};
  s.assign(seg_off, seg_off + nseg + 1);
  if (s.front() != 0 || s.back() != n || nseg > 64) throw std::invalid_argument("bad segment offsets");
  for (int q = 0; q < nseg; ++q)
    if (s[(size_t)q + 1] <= s[(size_t)q]) throw std::invalid_argument("empty or decreasing segment");
  return s;
}
}  // namespace

extern "C" {

int nds_mpnn_param_count(void) { return NDS_MPNN_NPARAM; }

int nds_mpnn_create(int n_max, int training, int device, nds_mpnn** out) {
  if (!out || n_max < 1) return mfail(NDS_E_INVALID, "nds_mpnn_create: bad argument");
  return mguard([&] {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
      throw nds::CudaError("no CUDA device available");
    NDS_CUDA(cudaSetDevice(device));
    auto m = std::make_unique<nds_mpnn>();
    NDS_CUDA(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    m->impl = nds::make_mpnn(n_max, training != 0, m->st);
    *out = m.release();
  });
}
int nds_mpnn_set_params(nds_mpnn* m, const float* host, int count) {
  if (!m || !host || count != NDS_MPNN_NPARAM) return mfail(NDS_E_INVALID, "nds_mpnn_set_params: bad argument");
  return mguard([&] {
    m->impl->set_params(host);
    NDS_CUDA(cudaStreamSynchronize(m->st));
  });
}
int nds_mpnn_get_params(nds_mpnn* m, float* host, int count) {
  if (!m || !host || count != NDS_MPNN_NPARAM) return mfail(NDS_E_INVALID, "nds_mpnn_get_params: bad argument");
  return mguard([&] {
    NDS_CUDA(cudaMemcpyAsync(host, m->impl->params.p, sizeof(float) * NDS_MPNN_NPARAM, cudaMemcpyDeviceToHost, m->st));
    NDS_CUDA(cudaStreamSynchronize(m->st));
  });
}
int nds_mpnn_get_grads(nds_mpnn* m, float* host, int count) {
  if (!m || !host || count != NDS_MPNN_NPARAM || !m->impl->training)
    return mfail(NDS_E_INVALID, "nds_mpnn_get_grads: bad argument");
  return mguard([&] {
    NDS_CUDA(cudaMemcpyAsync(host, m->impl->grads.p, sizeof(float) * NDS_MPNN_NPARAM, cudaMemcpyDeviceToHost, m->st));
    NDS_CUDA(cudaStreamSynchronize(m->st));
  });
}
int nds_mpnn_forward(nds_mpnn* m, const nds_mpnn_graph* g, int nseg, const int32_t* seg_off, const float* v,
                     float* z) {
  if (!m || !g || !v || !z) return mfail(NDS_E_INVALID, "nds_mpnn_forward: null argument");
  return mguard([&] {
    m->impl->forward(*g, v, z, segs(g->n, nseg, seg_off), true);
    m->impl->check_err();
  });
}
int nds_mpnn_loss_backward(nds_mpnn* m, const nds_mpnn_graph* g, int nseg, const int32_t* seg_off, const float* v,
                           const float* x, double* loss) {
  if (!m || !g || !v || !x) return mfail(NDS_E_INVALID, "nds_mpnn_loss_backward: null argument");
  return mguard([&] {
    const double L = m->impl->loss_backward(*g, v, x, segs(g->n, nseg, seg_off));
    if (loss) *loss = L;
  });
}
int nds_mpnn_backward(nds_mpnn* m, const nds_mpnn_graph* g, const float* dz) {
  if (!m || !g || !dz) return mfail(NDS_E_INVALID, "nds_mpnn_backward: null argument");
  return mguard([&] {
    if (g->n != m->impl->seg_n) throw std::invalid_argument("graph differs from the last forward's");
    m->impl->backward_dz(*g, dz);
  });
}
int nds_mpnn_adam_step(nds_mpnn* m, float lr, float beta1, float beta2, float eps, int step) {
  if (!m || step < 1 || !m->impl->training) return mfail(NDS_E_INVALID, "nds_mpnn_adam_step: bad argument");
  return mguard([&] {
    m->impl->adam_step(lr, beta1, beta2, eps, step);
    NDS_CUDA(cudaStreamSynchronize(m->st));
  });
}
int nds_mpnn_activations(nds_mpnn* m, int layer, void* out_dev) {
  if (!m || !out_dev || layer < 1 || layer > 3) return mfail(NDS_E_INVALID, "nds_mpnn_activations: bad argument");
  return mguard([&] {
    const __nv_bfloat16* src = layer == 1 ? m->impl->h1.p : layer == 2 ? m->impl->h2.p : m->impl->h3.p;
    if (!src) throw std::invalid_argument("activation not kept (inference handle)");
    NDS_CUDA(cudaMemcpyAsync(out_dev, src, sizeof(__nv_bfloat16) * (size_t)m->impl->n_max * nds::mp::kH,
                             cudaMemcpyDeviceToDevice, m->st));
    NDS_CUDA(cudaStreamSynchronize(m->st));
  });
}
void nds_mpnn_destroy(nds_mpnn* m) {
  if (!m) return;
  m->impl.reset();
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
}

}  // extern "C"
