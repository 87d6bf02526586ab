// sm_100a kernels of the SIMPLE hot path.  All kernels are deterministic:
// every output element is owned by one thread, group or warp, and every
// reduction goes through fixed-order block partials (no floating atomics).
//
// T is the storage/arithmetic type of states, operators and AMG data
// (double for the FP64 path, float for FP32); reductions and Krylov scalars
// are double in both, as in the reference (gpu/serial_cuda/precision.hpp:7-36).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "common.cuh"

namespace nds {
namespace k {

// ---------------------------------------------------------------------------
// block partial reductions -> out[NV] (single block, fixed order)
// ---------------------------------------------------------------------------
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

template <int NV>
__device__ __forceinline__ void write_partials(double (&v)[NV], double* part) {
  block_sum<NV>(v);
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) part[(size_t)blockIdx.x * NV + k] = v[k];
}

// The velocity state is stored interleaved, component d of dof g at
// u[kVel g + d]: the momentum sweep, the cell pass and the continuity
// residual gather all three components of a dof, which then share a sector.
// Kernels take the three component pointers u, u + 1, u + 2.
constexpr int kVel = 3;

// u[3 i + d] = a_d[i] for the components given (null: left as is)
template <class T>
__global__ void interleave3(int n, const T* __restrict__ a0, const T* __restrict__ a1, const T* __restrict__ a2,
                            T* __restrict__ u) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (a0) u[kVel * (size_t)i] = a0[i];
  if (a1) u[kVel * (size_t)i + 1] = a1[i];
  if (a2) u[kVel * (size_t)i + 2] = a2[i];
}
template <class T>
__global__ void deinterleave3(int n, const T* __restrict__ u, T* __restrict__ a0, T* __restrict__ a1,
                              T* __restrict__ a2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  a0[i] = u[kVel * (size_t)i];
  a1[i] = u[kVel * (size_t)i + 1];
  a2[i] = u[kVel * (size_t)i + 2];
}

// ---------------------------------------------------------------------------
// Momentum assembly (a9 + a10 + a11 + a12) in two passes
//
//   A[i,:]  = K[i,:] + sum_{(c,a) incident to i} C_c[a,:]           (convection, lagged u)
//   conv_i  = - sum C_c[a,b] u_fixed(b)                              (Dirichlet columns)
//   delta_i = (1/alpha_u - 1) sum_k |A[i,k]|, A[i,i] += delta_i     (row-L1 relaxation)
//   diag_i  = A[i,i], rau_i = rau_scale / A[i,i]
//   b_d[i]  = s_d[i] + conv_d[i] + (B^T p)_d[i] + delta_i u_d[i]
// with C_c[a,b] = det_c sum_m sum_j ur[m][j] T[a][m][b][j],
//      ur[m][j] = sum_d u_d(m) invJ_c[j][d].
// Reference: h7_momentum_assembly.cuh:16-85, h4_kernels.cuh:10-56,
// g5e_fp32_kernels.cuh:78-85 and :97-105, h8_precomputed_b.cuh:93-114.
//
// Pass 1 (mom_cell_conv, cell-owned) evaluates each cell's 8x8 convection
// block once.  Pass 2 (mom_assemble, row-owned) builds every velocity row in
// shared memory from K and the blocks of its incident cells, visited in
// ascending cell order, so every A entry is summed in a fixed order (K
// first) with no atomics; relaxation, diag, rAU, B^T p and the RHS follow in
// the same pass.
// ---------------------------------------------------------------------------

// Laminar SUPG terms, implicit form (h7_momentum_assembly.cuh:100-226; host
// twin g4_host.hpp:324-419): column b of the cell block
//   S[a][b] = sum_q tau_q w_q det (adv_q . grad phi_a) strong_b(q),
//   strong_b = adv . grad phi_b (- nu lap phi_b for the bubbles),
//   tau_q = tau_scale / sqrt(max(4 |adv_q|^2 / h^2 + magic (4 nu / h^2)^2, 1e-30)),
// over the 64-point collapsed rule (rule: 64 x (lambda0..3, weight)).
// Lane m of the 8-lane group holds the velocity q of basis m; lane b returns
// S[0..7][b].
struct SupgArgs {
  double nu, tau_scale, magic;
};
template <class T>
__device__ __forceinline__ void supg_column(const T* __restrict__ I, T h2, T dc, T q0, T q1, T q2,
                                            const T* __restrict__ rule, const SupgArgs& sa, int lane8,
                                            unsigned gmask, T S[8]) {
  T gl[4][3], gd[4][4];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    gl[0][d] = -(I[d] + I[3 + d] + I[6 + d]);
    gl[1][d] = I[d];
    gl[2][d] = I[3 + d];
    gl[3][d] = I[6 + d];
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i; j < 4; ++j) {
      T v = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) v += gl[i][d] * gl[j][d];
      gd[i][j] = gd[j][i] = v;
    }
  // this lane's basis function: vertex i = lane8 (< 4) or the bubble on the
  // face opposite vertex i = lane8 - 4, with the other vertices j0 < j1 < j2
  const int i = lane8 & 3;
  const int j0 = i == 0 ? 1 : 0, j1 = i <= 1 ? 2 : 1, j2 = i <= 2 ? 3 : 2;
  const bool bubble = lane8 >= 4;
  const T nu = T(sa.nu), diff = T(4) * nu / h2;
#pragma unroll
  for (int a = 0; a < 8; ++a) S[a] = 0;
  for (int qp = 0; qp < 64; ++qp) {
    const T* lam = rule + 5 * qp;
    const T l0 = lam[j0], l1 = lam[j1], l2 = lam[j2];
    const T phi = bubble ? T(27) * l0 * l1 * l2 : lam[i];
    const T a0 = group_sum<8>(q0 * phi, gmask), a1 = group_sum<8>(q1 * phi, gmask), a2 = group_sum<8>(q2 * phi, gmask);
    T g0, g1, g2, lap = 0;
    if (!bubble) {
      g0 = gl[i][0];
      g1 = gl[i][1];
      g2 = gl[i][2];
    } else {
      g0 = T(27) * (l1 * l2 * gl[j0][0] + l0 * l2 * gl[j1][0] + l0 * l1 * gl[j2][0]);
      g1 = T(27) * (l1 * l2 * gl[j0][1] + l0 * l2 * gl[j1][1] + l0 * l1 * gl[j2][1]);
      g2 = T(27) * (l1 * l2 * gl[j0][2] + l0 * l2 * gl[j1][2] + l0 * l1 * gl[j2][2]);
      lap = T(54) * (l2 * gd[j0][j1] + l1 * gd[j0][j2] + l0 * gd[j1][j2]);
    }
    const T stream = a0 * g0 + a1 * g1 + a2 * g2;
    const T strong = bubble ? -nu * lap + stream : stream;
    const T speed2 = a0 * a0 + a1 * a1 + a2 * a2;
    const T den = fmax(T(4) * speed2 / h2 + T(sa.magic) * diff * diff, T(1e-30));
    const T w = T(sa.tau_scale) / sqrt(den) * lam[4] * dc;
    const T ta = w * stream;
#pragma unroll
    for (int a = 0; a < 8; ++a) S[a] += __shfl_sync(gmask, ta, a, 8) * strong;
  }
}

// 8 lanes per cell; lane b computes column b of the cell's block (convection,
// plus the SUPG terms when SUPG; supg_rule and h2 are read only then).  Row a
// of the block is written to C[8 z + b], z the incidence (c, a) in the
// velocity rows' incidence lists, so that a row's blocks lie contiguous; the
// cell's pressure goes to pz[z] for the B^T p terms of the row pass.
template <class T, bool SUPG>
__global__ void __launch_bounds__(kBlock, SUPG ? 2 : 4) mom_cell_conv(int nc, const int32_t* __restrict__ ref,
                                                        const T* __restrict__ fixed, const T* __restrict__ u0,
                                                        const T* __restrict__ u1, const T* __restrict__ u2,
                                                        const T* __restrict__ invJ, const T* __restrict__ det,
                                                        const T* __restrict__ centT, const int32_t* __restrict__ zpos,
                                                        T* __restrict__ C, const T* __restrict__ p, T* __restrict__ pz,
                                                        const T* __restrict__ supg_rule, const T* __restrict__ h2,
                                                        SupgArgs sa) {
  __shared__ T sT[1536];
  __shared__ T sQ[SUPG ? 320 : 1];
  for (int k = threadIdx.x; k < 1536; k += blockDim.x) sT[k] = centT[k];
  if (SUPG)
    for (int k = threadIdx.x; k < 320; k += blockDim.x) sQ[k] = supg_rule[k];
  __syncthreads();
  const int lane8 = threadIdx.x & 7;
  const int groups = blockDim.x >> 3;
  const unsigned gmask = group8_mask();
  for (int c = blockIdx.x * groups + (threadIdx.x >> 3); c < nc; c += gridDim.x * groups) {
    // lane m: velocity of basis function m of cell c, mapped by J^-1
    const int gm = ref[8 * (size_t)c + lane8];
    T q0, q1, q2;
    if (gm >= 0) {
      q0 = u0[kVel * (size_t)gm];
      q1 = u1[kVel * (size_t)gm];
      q2 = u2[kVel * (size_t)gm];
    } else {
      const T* f = fixed + 3 * (size_t)(-gm - 1);
      q0 = f[0];
      q1 = f[1];
      q2 = f[2];
    }
    const T* I = invJ + 9 * (size_t)c;
    const T r0 = q0 * I[0] + q1 * I[1] + q2 * I[2];
    const T r1 = q0 * I[3] + q1 * I[4] + q2 * I[5];
    const T r2 = q0 * I[6] + q1 * I[7] + q2 * I[8];
    T w[8][3];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      w[m][0] = __shfl_sync(gmask, r0, m, 8);
      w[m][1] = __shfl_sync(gmask, r1, m, 8);
      w[m][2] = __shfl_sync(gmask, r2, m, 8);
    }
    const T dc = det[c];
    // row a of the block goes to the incidence slot zpos[8c + a] (-1: the
    // dof of basis a is fixed and has no momentum row)
    const int zl = zpos[8 * (size_t)c + lane8];
    if (zl >= 0) pz[zl] = p[c];  // the cell's pressure, by the incidences of its bases
    T S[8];
    if (SUPG) supg_column<T>(I, h2[c], dc, q0, q1, q2, sQ, sa, lane8, gmask, S);
#pragma unroll 2
    for (int a = 0; a < 8; ++a) {
      T cv = 0;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        const T* t = sT + ((a * 8 + m) * 8 + lane8) * 3;
        cv += w[m][0] * t[0] + w[m][1] * t[1] + w[m][2] * t[2];
      }
      const int za = __shfl_sync(gmask, zl, a, 8);
      if (za >= 0) C[8 * (size_t)za + lane8] = SUPG ? cv * dc + S[a] : cv * dc;
    }
  }
}

template <class T>
struct MomArgs {
  int nrows;
  const int2* __restrict__ span;        // row i's (begin, end) in the colour-ordered storage
  const int32_t* __restrict__ dpos;     // diagonal position (absolute)
  const T* __restrict__ K;              // persistent diffusion values
  const int32_t* __restrict__ inc_off;  // row -> incident (cell,a)
  const uint32_t* __restrict__ inc;     // (cell << 3) | a
  const int32_t* __restrict__ ref;      // 8 per cell
  const uint8_t* __restrict__ slot;     // 64 per cell
  const T* __restrict__ C;              // 8 per incidence: convection rows from mom_cell_conv
  const uint8_t* __restrict__ slotz;    // 8 per incidence: slot[c][a][b] of incidence (c, a)
  const T* __restrict__ Bz;             // 3 per incidence: B[c][a]
  const T* __restrict__ pz;             // per incidence: p_c (written by the cell pass)
  const uint8_t* __restrict__ fixz;     // per incidence: bit b set when dof b of the cell is fixed
  const T* __restrict__ bco;            // 24 per cell
  const T* __restrict__ fixed;          // 3 per fixed slot
  const T* __restrict__ u0;
  const T* __restrict__ u1;
  const T* __restrict__ u2;
  const T* __restrict__ p;
  const T* __restrict__ s0;
  const T* __restrict__ s1;
  const T* __restrict__ s2;
  // fused form (no cell pass): C rows are evaluated per incidence
  const T* __restrict__ invJ;           // 9 per cell
  const T* __restrict__ det;            // 1 per cell
  const T* __restrict__ centT;          // reference tensor T[8][8][8][3]
  T alpha_u, rau_scale;
  int row_cap;                          // shared row buffer length per group
  T* __restrict__ A;
  T* __restrict__ delta;
  T* __restrict__ diag;
  T* __restrict__ rau;
  T* __restrict__ b0;
  T* __restrict__ b1;
  T* __restrict__ b2;
};

// 8 lanes per velocity row; lane b adds column b of each incident block.
// Convection entries C_c[a][lane8] of one incidence (cell c, basis a), the
// same expression and order as mom_cell_conv: lane m maps the velocity of
// basis m by J^-1, the group shares the eight mapped velocities, lane b sums
// over m.  ga: this lane's DOF of cell c (ref[8 c + lane8]).
template <class T>
__device__ __forceinline__ T conv_entry(const MomArgs<T>& g, const T* __restrict__ sT, int c, int a, int ga,
                                        int lane8, unsigned gmask) {
  T q0, q1, q2;
  if (ga >= 0) {
    q0 = g.u0[kVel * (size_t)ga];
    q1 = g.u1[kVel * (size_t)ga];
    q2 = g.u2[kVel * (size_t)ga];
  } else {
    const T* f = g.fixed + 3 * (size_t)(-ga - 1);
    q0 = f[0];
    q1 = f[1];
    q2 = f[2];
  }
  const T* I = g.invJ + 9 * (size_t)c;
  const T r0 = q0 * I[0] + q1 * I[1] + q2 * I[2];
  const T r1 = q0 * I[3] + q1 * I[4] + q2 * I[5];
  const T r2 = q0 * I[6] + q1 * I[7] + q2 * I[8];
  T cv = 0;
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const T w0 = __shfl_sync(gmask, r0, m, 8), w1 = __shfl_sync(gmask, r1, m, 8), w2 = __shfl_sync(gmask, r2, m, 8);
    const T* t = sT + ((a * 8 + m) * 8 + lane8) * 3;
    cv += w0 * t[0] + w1 * t[1] + w2 * t[2];
  }
  return cv * g.det[c];
}

// FUSED 0: the row pass of the two-pass assembly; each velocity row reads
// its incident cells' convection rows, which the cell pass wrote contiguous
// in incidence order, kAsmAhead at a time.  FUSED 1: C rows evaluated per
// incidence (conv_entry) instead, with the reference tensor staged in shared
// memory after the row buffers (no cell pass).  Both add the same values in
// the same order.
constexpr int kAsmAhead = 4;
template <class T, int FUSED = 0>
__global__ void __launch_bounds__(kBlock) mom_assemble(MomArgs<T> g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sRow = reinterpret_cast<T*>(smem_raw);  // groups * row_cap
  const int tid = threadIdx.x;
  const int lane8 = tid & 7;
  const int grp = tid >> 3;
  const int groups = blockDim.x >> 3;
  T* buf = sRow + (size_t)grp * g.row_cap;
  T* sT = sRow + (size_t)groups * g.row_cap;
  if (FUSED) {
    for (int k = tid; k < 1536; k += blockDim.x) sT[k] = g.centT[k];
    __syncthreads();
  }
  const unsigned gmask = group8_mask();
  for (int i = blockIdx.x * groups + grp; i < g.nrows; i += gridDim.x * groups) {
    const int2 sp = g.span[i];
    const int rb = sp.x, len = sp.y - sp.x;
    for (int k = lane8; k < len; k += 8) buf[k] = g.K[rb + k];
    __syncwarp(gmask);
    T conv0 = 0, conv1 = 0, conv2 = 0, bt0 = 0, bt1 = 0, bt2 = 0;
    const int z0 = g.inc_off[i], z1 = g.inc_off[i + 1];
    if (FUSED == 1) {
      for (int z = z0; z < z1; ++z) {
        const uint32_t pa = g.inc[z];
        const int ca = (int)(pa >> 3), aa = (int)(pa & 7u);
        const int ga = g.ref[8 * (size_t)ca + lane8];
        const int sa = g.slot[64 * (size_t)ca + 8 * aa + lane8];
        const T va = conv_entry<T>(g, sT, ca, aa, ga, lane8, gmask);
        if (ga >= 0) {
          buf[sa] += va;
        } else {
          const T* f = g.fixed + 3 * (size_t)(-ga - 1);
          conv0 -= va * f[0];
          conv1 -= va * f[1];
          conv2 -= va * f[2];
        }
        if (lane8 == 0) {
          const T pv = g.p[ca];
          const T* B = g.bco + 24 * (size_t)ca + 3 * aa;
          bt0 += B[0] * pv;
          bt1 += B[1] * pv;
          bt2 += B[2] * pv;
        }
        __syncwarp(gmask);
      }
    }
    if (FUSED == 0) {
      // B^T p: lane d < 3 sums component d over the row's incidences in
      // incidence order (B and p contiguous per row); lane 0 then takes the
      // other two components
      {
        T btd = 0;
        if (lane8 < 3)
          for (int z = z0; z < z1; ++z) btd += g.Bz[3 * (size_t)z + lane8] * g.pz[z];
        const T t1 = __shfl_sync(gmask, btd, 1, 8), t2 = __shfl_sync(gmask, btd, 2, 8);
        if (lane8 == 0) {
          bt0 = btd;
          bt1 = t1;
          bt2 = t2;
        }
      }
      // the row's convection rows, contiguous in incidence order, kAsmAhead
      // at a time; added in incidence order
      for (int zb = z0; zb < z1; zb += kAsmAhead) {
        T cz[kAsmAhead];
        int sz[kAsmAhead];
        uint32_t fm[kAsmAhead];
#pragma unroll
        for (int u = 0; u < kAsmAhead; ++u) {
          const int z = zb + u;
          const bool ok = z < z1;
          cz[u] = ok ? g.C[8 * (size_t)z + lane8] : T(0);
          sz[u] = ok ? g.slotz[8 * (size_t)z + lane8] : 0;
          fm[u] = ok ? g.fixz[z] : 0u;
        }
#pragma unroll
        for (int u = 0; u < kAsmAhead; ++u) {
          if (zb + u < z1) {
            if ((fm[u] >> lane8) & 1u) {
              const uint32_t pa = g.inc[zb + u];
              const int ga = g.ref[8 * (size_t)(pa >> 3) + lane8];
              const T* f = g.fixed + 3 * (size_t)(-ga - 1);
              conv0 -= cz[u] * f[0];
              conv1 -= cz[u] * f[1];
              conv2 -= cz[u] * f[2];
            } else {
              buf[sz[u]] += cz[u];
            }
          }
          __syncwarp(gmask);
        }
      }
    }
    conv0 = group_sum<8>(conv0, gmask);
    conv1 = group_sum<8>(conv1, gmask);
    conv2 = group_sum<8>(conv2, gmask);
    T l1 = 0;
    for (int k = lane8; k < len; k += 8) l1 += fabs(buf[k]);
    l1 = group_sum<8>(l1, gmask);
    const int dl = g.dpos[i] - rb;
    const T de = (T(1) / g.alpha_u - T(1)) * l1;
    __syncwarp(gmask);
    if (lane8 == 0) buf[dl] += de;
    __syncwarp(gmask);
    for (int k = lane8; k < len; k += 8) g.A[rb + k] = buf[k];
    if (lane8 == 0) {
      const T d = buf[dl];
      g.delta[i] = de;
      g.diag[i] = d;
      g.rau[i] = (T(1) / d) * g.rau_scale;
      g.b0[i] = g.s0[i] + conv0 + bt0 + de * g.u0[kVel * (size_t)i];
      g.b1[i] = g.s1[i] + conv1 + bt1 + de * g.u1[kVel * (size_t)i];
      g.b2[i] = g.s2[i] + conv2 + bt2 + de * g.u2[kVel * (size_t)i];
    }
    __syncwarp(gmask);
  }
}

// One multicolour Gauss-Seidel colour pass on the shared momentum matrix,
// three right-hand sides (g5e_fp32_kernels.cuh:106-116).  8 lanes per row.
// The matrix is stored colour by colour (the rows of one colour contiguous,
// each colour's rows in ascending order), so one pass streams one block of
// the matrix; span: the storage range of each of the colour's rows (pad
// entries have the row's own column), rows: their natural indices (their
// right-hand sides, diagonals and unknowns).
// Each lane takes its entries kGsAhead at a time: it loads their columns and
// values, then gathers their unknowns, so a batch's loads are in flight
// together; the diagonal entry and the padding of a batch contribute 0.
// Per lane the entries are summed in the order of the storage, then over
// the 8 lanes.
constexpr int kGsAhead = 2;
template <class T>
__global__ void __launch_bounds__(kBlock, 6) mom_gs_color(int count, const int32_t* __restrict__ rows,
                                                       const int2* __restrict__ span, const int32_t* __restrict__ ci,
                                                       const T* __restrict__ av, const T* __restrict__ diag,
                                                       const T* __restrict__ b0, const T* __restrict__ b1,
                                                       const T* __restrict__ b2, T* __restrict__ x0, T* __restrict__ x1,
                                                       T* __restrict__ x2, T omega) {
  const int lane8 = threadIdx.x & 7;
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
  if (q >= count) return;
  const unsigned gmask = group8_mask();
  const int i = rows[q];
  const int2 sp = span[q];
  const int kb = sp.x, ke = sp.y;
  T d = 0, c0 = 0, c1 = 0, c2 = 0, y0 = 0, y1 = 0, y2 = 0;
  const size_t vi = kVel * (size_t)i;
  if (lane8 == 0) {
    d = diag[i];
    c0 = b0[i];
    c1 = b1[i];
    c2 = b2[i];
    y0 = x0[vi];
    y1 = x1[vi];
    y2 = x2[vi];
  }
  T s0 = 0, s1 = 0, s2 = 0;
  for (int k0 = kb + lane8; k0 < ke; k0 += 8 * kGsAhead) {
    int jj[kGsAhead];
    T aa[kGsAhead];
#pragma unroll
    for (int u = 0; u < kGsAhead; ++u) {
      const int k = k0 + 8 * u;
      jj[u] = k < ke ? ci[k] : i;
      aa[u] = k < ke ? av[k] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kGsAhead; ++u) {
      const T a = jj[u] == i ? T(0) : aa[u];
      const size_t vj = kVel * (size_t)jj[u];
      s0 += a * x0[vj];
      s1 += a * x1[vj];
      s2 += a * x2[vj];
    }
  }
  s0 = group_sum<8>(s0, gmask);
  s1 = group_sum<8>(s1, gmask);
  s2 = group_sum<8>(s2, gmask);
  if (lane8 == 0) {
    const T iv = T(1) / d;
    x0[vi] = (T(1) - omega) * y0 + omega * ((c0 - s0) * iv);
    x1[vi] = (T(1) - omega) * y1 + omega * ((c1 - s1) * iv);
    x2[vi] = (T(1) - omega) * y2 + omega * ((c2 - s2) * iv);
  }
}

// ||b_d||^2 and ||b_d - A u_d||^2 (g5e_fp32_kernels.cuh:117-126); 6 partials per block.
template <class T>
__global__ void __launch_bounds__(kBlock) mom_audit(int n, const int2* __restrict__ span, const int32_t* __restrict__ ci,
                                                    const T* __restrict__ av, const T* __restrict__ b0,
                                                    const T* __restrict__ b1, const T* __restrict__ b2,
                                                    const T* __restrict__ x0, const T* __restrict__ x1,
                                                    const T* __restrict__ x2, double* __restrict__ part) {
  const int lane8 = threadIdx.x & 7;
  const unsigned gmask = group8_mask();
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int groups_total = (gridDim.x * blockDim.x) >> 3;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 3; i < n; i += groups_total) {
    T a0 = 0, a1 = 0, a2 = 0;
    const int2 sp = span[i];
    for (int k = sp.x + lane8; k < sp.y; k += 8) {
      const size_t vj = kVel * (size_t)ci[k];
      const T a = av[k];
      a0 += a * x0[vj];
      a1 += a * x1[vj];
      a2 += a * x2[vj];
    }
    a0 = group_sum<8>(a0, gmask);
    a1 = group_sum<8>(a1, gmask);
    a2 = group_sum<8>(a2, gmask);
    if (lane8 == 0) {
      const double db0 = (double)b0[i], db1 = (double)b1[i], db2 = (double)b2[i];
      const double r0 = (double)(b0[i] - a0), r1 = (double)(b1[i] - a1), r2 = (double)(b2[i] - a2);
      acc[0] += db0 * db0;
      acc[1] += db1 * db1;
      acc[2] += db2 * db2;
      acc[3] += r0 * r0;
      acc[4] += r1 * r1;
      acc[5] += r2 * r2;
    }
  }
  write_partials<6>(acc, part);
}

// ---------------------------------------------------------------------------
// Continuity r_c = fixedDiv_c + sum_a B[c][a] . u(ref a)  (h8_precomputed_b.cuh:140-163),
// stored negated as the pressure right-hand side, with sum r^2 partials.
// Component d of velocity dof g is ud[VS g]: VS = kVel for the solver's
// interleaved state, 1 for three separate arrays.
// ---------------------------------------------------------------------------
template <class T, int VS = kVel>
__global__ void __launch_bounds__(kBlock) continuity(int nc, const int32_t* __restrict__ ref, const T* __restrict__ bco,
                                                     const T* __restrict__ fixed_div, const T* __restrict__ u0,
                                                     const T* __restrict__ u1, const T* __restrict__ u2,
                                                     T* __restrict__ rhs, double* __restrict__ part) {
  double acc[1] = {0.0};
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
    T s = fixed_div[c];
    // the cell's 8 dofs and 24 coefficients in 16-byte loads (the records
    // are 32 and 24 * sizeof(T) bytes, so 16-byte aligned)
    int rf[8];
    T B[24];
    {
      const int4* r4 = reinterpret_cast<const int4*>(ref + 8 * (size_t)c);
      const int4 q0 = r4[0], q1 = r4[1];
      rf[0] = q0.x; rf[1] = q0.y; rf[2] = q0.z; rf[3] = q0.w;
      rf[4] = q1.x; rf[5] = q1.y; rf[6] = q1.z; rf[7] = q1.w;
      if constexpr (sizeof(T) == 8) {
        const double2* b2 = reinterpret_cast<const double2*>(bco + 24 * (size_t)c);
#pragma unroll
        for (int k = 0; k < 12; ++k) {
          const double2 v = b2[k];
          B[2 * k] = v.x;
          B[2 * k + 1] = v.y;
        }
      } else {
#pragma unroll
        for (int k = 0; k < 24; ++k) B[k] = bco[24 * (size_t)c + k];
      }
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int g = rf[a];
      if (g < 0) continue;
      const size_t vg = (size_t)VS * g;
      s += B[3 * a] * u0[vg] + B[3 * a + 1] * u1[vg] + B[3 * a + 2] * u2[vg];
    }
    const T sr = s;
    acc[0] += (double)sr * (double)sr;
    rhs[c] = -s;
  }
  write_partials<1>(acc, part);
}

// ---------------------------------------------------------------------------
// CSR SpMV family, warp per row (h2b_fine_csr.cuh:579-596, h6_coarse_spmv.cuh:10-32)
// ---------------------------------------------------------------------------
// Lane l of a G-lane group sums entries rb+l, rb+l+G, ... in that order;
// the loads of eight entries are issued before their products are added
// (same order, an eighth of the dependent memory round trips).
// Coarse-level CSR rows (one to a few hundred entries) go to a warp each
// (G = 32), or to 16 lanes on the FP16 copies of the mixed path.  Lane l
// takes entries rb + l + G u; one round of predicated loads (eight per lane:
// columns and values, then the x gathers) covers a row of up to 8 G entries,
// so a row costs three dependent round trips (row bounds, columns and
// values, gathers).  Longer rows take further rounds.
// MT: the stored value type (T, or __half for an FP16 copy of a level whose
// values are scaled by a power of two; the caller multiplies the row sum back).
// CT: the column type (int32 absolute, or int16 deltas to the row).
template <class T, class MT>
__device__ __forceinline__ T load_val(const MT* __restrict__ v, int k) {
  if constexpr (std::is_same<MT, __half>::value) return (T)__half2float(v[k]);
  else return v[k];
}
// column of entry k of row i: absolute (int32) or a 16-bit delta to the row
__device__ __forceinline__ int col_at(const int32_t* __restrict__ ci, int k, int) { return ci[k]; }
__device__ __forceinline__ int col_at(const int16_t* __restrict__ ci, int k, int i) { return i + ci[k]; }
template <int G, class T, class MT = T, class CT = int32_t>
__device__ __forceinline__ T lane_batched_dot(int rb, int re, const CT* __restrict__ ci, const MT* __restrict__ v,
                                              const T* __restrict__ x, int lane, int i = 0) {
  T s = 0;
  for (int k0 = rb + lane; k0 < re; k0 += 8 * G) {
    int c[8];
    T a[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u * G;
      c[u] = k < re ? col_at(ci, k, i) : -1;
      a[u] = k < re ? load_val<T, MT>(v, k) : T(0);
    }
    T xv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) xv[u] = c[u] >= 0 ? x[c[u]] : T(0);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (c[u] >= 0) s += a[u] * xv[u];
  }
  return s;
}
constexpr int kRowLanes = 32;
template <class T, class MT = T, class CT = int32_t, int GL = kRowLanes>
__device__ __forceinline__ T group_row_dot(const int32_t* __restrict__ rp, const CT* __restrict__ ci,
                                           const MT* __restrict__ v, const T* __restrict__ x, int i, int lane,
                                           unsigned mask, T vinv = T(1)) {
  T s = group_sum<GL>(lane_batched_dot<GL, T, MT, CT>(rp[i], rp[i + 1], ci, v, x, lane, i), mask);
  if constexpr (!std::is_same<MT, T>::value) s *= vinv;
  return s;
}

// y = A x (GL lanes per row)
template <class T, class MT = T, class CT = int32_t, int GL = kRowLanes>
__global__ void __launch_bounds__(kBlock) spmv(int n, const int32_t* __restrict__ rp, const CT* __restrict__ ci,
                                               const MT* __restrict__ v, const T* __restrict__ x, T* __restrict__ y,
                                               T vinv = T(1)) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / GL, lane = t % GL;
  if (i >= n) return;
  const T s = group_row_dot<T, MT, CT, GL>(rp, ci, v, x, i, lane, group_mask<GL>(), vinv);
  if (lane == 0) y[i] = s;
}

// r = b - A x  (optionally also r2 = r)
template <class T, class MT = T, class CT = int32_t, int GL = kRowLanes>
__global__ void __launch_bounds__(kBlock) spmv_resid(int n, const int32_t* __restrict__ rp, const CT* __restrict__ ci,
                                                     const MT* __restrict__ v, const T* __restrict__ x,
                                                     const T* __restrict__ b, T* __restrict__ r, T* __restrict__ r2,
                                                     const T* __restrict__ den, T w, T vinv = T(1)) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / GL, lane = t % GL;
  if (i >= n) return;
  const T s = group_row_dot<T, MT, CT, GL>(rp, ci, v, x, i, lane, group_mask<GL>(), vinv);
  if (lane == 0) {
    // r; r2 = r (den null) or the first Jacobi step w r / den
    const T q = b[i] - s;
    r[i] = q;
    if (den) r2[i] = w * q / den[i];
    else if (r2) r2[i] = q;
  }
}

// Jacobi-type smoothing step: x_out = x_in + w (b - A x_in) / den
template <class T, class MT = T, class CT = int32_t, int GL = kRowLanes>
__global__ void __launch_bounds__(kBlock) spmv_smooth(int n, const int32_t* __restrict__ rp,
                                                      const CT* __restrict__ ci, const MT* __restrict__ v,
                                                      const T* __restrict__ xin, const T* __restrict__ b,
                                                      const T* __restrict__ den, T w, T* __restrict__ xout,
                                                      T* __restrict__ add_to, T vinv = T(1)) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = t / GL, lane = t % GL;
  if (i >= n) return;
  const T s = group_row_dot<T, MT, CT, GL>(rp, ci, v, xin, i, lane, group_mask<GL>(), vinv);
  if (lane == 0) {
    // with add_to the step is added to add_to instead of stored in xout
    const T r = b[i] - s;
    const T val = xin[i] + w * r / den[i];
    if (add_to) add_to[i] += val;
    else xout[i] = val;
  }
}

// ---------------------------------------------------------------------------
// vector kernels (g5e_fp32_kernels.cuh:132-150, vector_kernels.cuh)
// ---------------------------------------------------------------------------
template <class T>
__global__ void jacobi_zero(int n, T w, const T* __restrict__ b, const T* __restrict__ d, T* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] = w * b[i] / d[i];
}
template <class T>
__global__ void axpy(int n, T a, const T* __restrict__ x, T* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}
template <class T>
__global__ void copy(int n, const T* __restrict__ a, T* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = a[i];
}
template <class T>
__global__ void scale(int n, T s, T* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}
template <class T>
__global__ void div_sqrt(int n, const T* __restrict__ x, const T* __restrict__ d, T* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i] / sqrt(d[i]);
}
template <class T>
__global__ void power_init(int n, T* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const T g = T(i + 1);
    v[i] = sin(T(0.731) * g) + T(0.27) * cos(T(1.117) * g);
  }
}

// partial sums of x.y
template <class T>
__global__ void __launch_bounds__(kBlock) dot(int n, const T* __restrict__ x, const T* __restrict__ y,
                                              double* __restrict__ part) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    acc[0] += (double)x[i] * (double)y[i];
  write_partials<1>(acc, part);
}
// x += a p; r -= a q; partial r.r.  a = alpha_dev ? *alpha_dev : alpha
// With x1: also the first (diagonal) step of the next preconditioner
// application's fine pre-smoother on the new r, x1 = w0 r / den0 (the
// expression of jacobi_zero).
template <class T>
__global__ void __launch_bounds__(kBlock) xr_update(int n, double alpha, const double* __restrict__ alpha_dev,
                                                    const T* __restrict__ p, const T* __restrict__ q,
                                                    T* __restrict__ x, T* __restrict__ r, double* __restrict__ part,
                                                    const T* __restrict__ den0 = nullptr, T w0 = T(0),
                                                    T* __restrict__ x1 = nullptr) {
  const T a = T(alpha_dev ? *alpha_dev : alpha);
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    const T rr = r[i] - a * q[i];
    r[i] = rr;
    if (x1) x1[i] = w0 * rr / den0[i];
    acc[0] += (double)rr * (double)rr;
  }
  write_partials<1>(acc, part);
}

// p = z + beta p, beta = *beta_dev
template <class T>
__global__ void p_update(int n, const double* __restrict__ beta_dev, const T* __restrict__ z, T* __restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = z[i] + T(*beta_dev) * p[i];
}

// PCG scalar steps on device.  flags bit 1: pAp <= 0 or non-finite; bit 2: rho <= 0 or non-finite.
// sc layout: [0] rho  [1] pq  [2] alpha  [3] rn2  [4] rhon  [5] beta
__device__ __forceinline__ void pcg_alpha_step(double* __restrict__ sc, int* __restrict__ flags) {
  const double pq = sc[1];
  if (!(pq > 0.0) || !isfinite(pq)) {
    *flags |= 1;
    sc[2] = 0.0;
    return;
  }
  sc[2] = sc[0] / pq;
}
__global__ void pcg_alpha(double* __restrict__ sc, int* __restrict__ flags) { pcg_alpha_step(sc, flags); }
__global__ void pcg_beta(double* __restrict__ sc, int* __restrict__ flags) {
  const double rhon = sc[4];
  if (!(rhon > 0.0) || !isfinite(rhon)) {
    *flags |= 2;
    sc[5] = 0.0;
    return;
  }
  sc[5] = rhon / sc[0];
  sc[0] = rhon;
}

// Device-resident PCG loop (one CUDA graph with a conditional while node).
// ctl: [0] iterations done, [1] converged, [2] first iteration pending.
// flags bit 8: initial rho <= 0 or non-finite; bit 4: residual non-finite.
//
// rho step of the loop body: on the first iteration rho = r.z (p = z follows),
// afterwards beta = rho_new / rho as pcg_beta.
__device__ __forceinline__ void pcg_rho_step(double* __restrict__ sc, int* __restrict__ flags,
                                             const int* __restrict__ ctl) {
  const double rhon = sc[4];
  if (ctl[2]) {
    if (!(rhon > 0.0) || !isfinite(rhon)) *flags |= 8;
    sc[0] = rhon;
    sc[5] = 0.0;
    return;
  }
  if (!(rhon > 0.0) || !isfinite(rhon)) {
    *flags |= 2;
    sc[5] = 0.0;
    return;
  }
  sc[5] = rhon / sc[0];
  sc[0] = rhon;
}
__global__ void pcg_rho_dev(double* __restrict__ sc, int* __restrict__ flags, const int* __restrict__ ctl) {
  pcg_rho_step(sc, flags, ctl);
}
// p = z on the first iteration, else p = z + beta p
template <class T>
__global__ void p_update_dev(int n, const double* __restrict__ beta_dev, const int* __restrict__ ctl,
                             const T* __restrict__ z, T* __restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  p[i] = ctl[2] ? z[i] : z[i] + T(*beta_dev) * p[i];
}
// End of the loop body: count the iteration and test ||r|| <= target the way
// the host loop does (sqrt, then compare); stop on convergence, on any flag
// or at max_its.  The loop always ends: every body pass runs this kernel and
// the count reaches max_its.
// max_its < 0: the cap is ctl[3] (set per solve by the host).  in_graph = 0:
// launched outside a graph (host-driven loop), no condition to set.
__device__ __forceinline__ void pcg_check_step(const double* __restrict__ sc, int rn2_slot, int r0_slot,
                                               int target_slot, int* __restrict__ flags, int* __restrict__ ctl,
                                               int max_its, cudaGraphConditionalHandle loop, int in_graph) {
  if (max_its < 0) max_its = ctl[3];
  const int it = ++ctl[0];
  ctl[2] = 0;
  const double rn = sqrt(sc[rn2_slot]);
  if (!isfinite(rn / fmax(sc[r0_slot], 1e-300))) *flags |= 4;
  const int conv = rn <= sc[target_slot];
  ctl[1] = conv;
  const bool stop = conv || *flags != 0 || it >= max_its;
  if (in_graph) cudaGraphSetConditional(loop, stop ? 0u : 1u);
}
__global__ void pcg_check(const double* __restrict__ sc, int rn2_slot, int r0_slot, int target_slot,
                          int* __restrict__ flags, int* __restrict__ ctl, int max_its,
                          cudaGraphConditionalHandle loop, int in_graph = 1) {
  pcg_check_step(sc, rn2_slot, r0_slot, target_slot, flags, ctl, max_its, loop, in_graph);
}

// A reduction of one value's block partials (as reduce_partials<1>) whose
// thread 0 then takes the next scalar step of the device PCG: rho and beta
// (PCG_RHO), alpha (PCG_ALPHA) or the stopping test (PCG_CHECK).  One launch
// instead of two; the same sums and the same scalar arithmetic.
enum { PCG_RHO = 1, PCG_ALPHA = 2, PCG_CHECK = 3 };
struct PcgScalars {
  double* sc;
  int* flags;
  int* ctl;
  int rn2_slot, r0_slot, target_slot, max_its;
  cudaGraphConditionalHandle loop;
  int in_graph;
};
template <int STEP>
__global__ void reduce_pcg(const double* __restrict__ part, int nblocks, double* __restrict__ out, PcgScalars s) {
  double v[1] = {0.0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v[0] += part[b];
  block_sum<1>(v);
  if (threadIdx.x == 0) {
    out[0] = v[0];
    if (STEP == PCG_RHO) pcg_rho_step(s.sc, s.flags, s.ctl);
    else if (STEP == PCG_ALPHA) pcg_alpha_step(s.sc, s.flags);
    else pcg_check_step(s.sc, s.rn2_slot, s.r0_slot, s.target_slot, s.flags, s.ctl, s.max_its, s.loop, s.in_graph);
  }
}

// ---------------------------------------------------------------------------
// transfers and terminal solve (g5e_fp32_kernels.cuh:140-150)
// ---------------------------------------------------------------------------
// f += P c (one thread per fine row; P in ELL with entry k of row i at
// k nf + i, so a warp's loads of P are coalesced).  Sequential sum over k
// with the loads of four entries issued ahead; padding adds 0 c[0].
template <class T>
__global__ void prolong_add(int nf, int pw, const int32_t* __restrict__ pc, const T* __restrict__ pv,
                            const T* __restrict__ c, T* __restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  T s = 0;
  int k = 0;
  const size_t n = (size_t)nf;
  for (; k + 3 < pw; k += 4) {
    const size_t o = (size_t)k * n + i;
    const int c0 = pc[o], c1 = pc[o + n], c2 = pc[o + 2 * n], c3 = pc[o + 3 * n];
    const T a0 = pv[o], a1 = pv[o + n], a2 = pv[o + 2 * n], a3 = pv[o + 3 * n];
    const T x0 = c[c0], x1 = c[c1], x2 = c[c2], x3 = c[c3];
    s += a0 * x0;
    s += a1 * x1;
    s += a2 * x2;
    s += a3 * x3;
  }
  for (; k < pw; ++k) {
    const size_t o = (size_t)k * n + i;
    s += pv[o] * c[pc[o]];
  }
  f[i] += s;
}
// x = Ainv b, dense row-major, warp per row
template <class T>
__global__ void __launch_bounds__(kBlock) dense_mv(int n, const T* __restrict__ A, const T* __restrict__ b,
                                                   T* __restrict__ x) {
  const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (i >= n) return;
  const T* a = A + (size_t)i * n;
  T s = 0;
  for (int j = lane; j < n; j += 32) s += a[j] * b[j];
  s = warp_sum(s);
  if (lane == 0) x[i] = s;
}

// multicolour GS colour pass on an AMG level (h8_main_base.cu:205-223)
template <class T>
__global__ void amg_gs_color(int count, const int32_t* __restrict__ rows, const int32_t* __restrict__ rp,
                             const int32_t* __restrict__ ci, const T* __restrict__ v, const T* __restrict__ diag,
                             const T* __restrict__ b, T* __restrict__ x, T omega) {
  const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (q >= count) return;
  const int i = rows[q];
  T off = 0;
  for (int k = rp[i] + lane; k < rp[i + 1]; k += 32) {
    const int j = ci[k];
    if (j != i) off += v[k] * x[j];
  }
  off = warp_sum(off);
  if (lane == 0) {
    const T old = x[i];
    const T gs = (b[i] - off) / diag[i];
    x[i] = old + omega * (gs - old);
  }
}

}  // namespace k
}  // namespace nds

namespace nds {
namespace k {

// ---------------------------------------------------------------------------
// Fine Schur operator in sliced ELL with 4-wide lanes (SELL-32x4): rows are
// grouped in slices of 32 (one warp); each row's entries are padded to a
// multiple of 4 and entry k of row i (slice s = i/32, lane l = i%32) lives at
//   base[s] + 128 (k/4) + 4 l + (k%4),
// so every thread reads four consecutive entries of its own row with one
// vector load while the warp's loads stay fully coalesced (512 B of FP32
// values per instruction).  width[s] is the slice's longest row; padding
// entries carry value 0 and the row's own column.  One thread owns a row.
// ---------------------------------------------------------------------------
struct Sell {
  int n;
  const int32_t* __restrict__ base;
  const int32_t* __restrict__ width;
  const int32_t* __restrict__ col;   // absolute columns (used when dcol is null)
  const int16_t* __restrict__ dcol;  // column - row, when every |column - row| < 2^15
};

__device__ __forceinline__ int sell_offset(int base, int lane, int k) { return base + 128 * (k >> 2) + 4 * lane + (k & 3); }

// the four column indices of entries o..o+3 of row i (o a multiple of 4)
template <bool D16>
__device__ __forceinline__ void sell_col4(const Sell& A, int o, int i, int j[4]) {
  if (D16) {
    const short4 d = *reinterpret_cast<const short4*>(A.dcol + o);
    j[0] = i + d.x;
    j[1] = i + d.y;
    j[2] = i + d.z;
    j[3] = i + d.w;
  } else {
    const int4 c = *reinterpret_cast<const int4*>(A.col + o);
    j[0] = c.x;
    j[1] = c.y;
    j[2] = c.z;
    j[3] = c.w;
  }
}
template <class T>
__device__ __forceinline__ void sell_val4(const T* __restrict__ v, int o, T a[4]);
template <>
__device__ __forceinline__ void sell_val4<float>(const float* __restrict__ v, int o, float a[4]) {
  const float4 q = *reinterpret_cast<const float4*>(v + o);
  a[0] = q.x;
  a[1] = q.y;
  a[2] = q.z;
  a[3] = q.w;
}
template <>
__device__ __forceinline__ void sell_val4<double>(const double* __restrict__ v, int o, double a[4]) {
  const double2 p = *reinterpret_cast<const double2*>(v + o);
  const double2 q = *reinterpret_cast<const double2*>(v + o + 2);
  a[0] = p.x;
  a[1] = p.y;
  a[2] = q.x;
  a[3] = q.y;
}
// FP16 operator copy (values scaled by a power of two into FP16 range): four
// values of one 8-byte load, widened
__device__ __forceinline__ void sell_val4h(const __half* __restrict__ v, int o, float a[4]) {
  const uint2 q = *reinterpret_cast<const uint2*>(v + o);
  const float2 lo = __half22float2(*reinterpret_cast<const __half2*>(&q.x));
  const float2 hi = __half22float2(*reinterpret_cast<const __half2*>(&q.y));
  a[0] = lo.x;
  a[1] = lo.y;
  a[2] = hi.x;
  a[3] = hi.y;
}
template <class T, class MT>
__device__ __forceinline__ void sell_vals4(const MT* __restrict__ v, int o, T a[4]) {
  if constexpr (std::is_same<MT, __half>::value) sell_val4h(v, o, a);
  else sell_val4<T>(v, o, a);
}
template <bool D16>
__device__ __forceinline__ int sell_col(const Sell& A, int o, int i) {
  if (D16) return i + (int)A.dcol[o];
  return A.col[o];
}

enum SellMode { SELL_Y = 0, SELL_RESID = 1, SELL_SMOOTH = 2, SELL_DOT = 3 };

// Row dot product: entries in batches of 8 (two vector loads of values and
// of columns, then the 8 x gathers), even entries into s0 and odd ones into
// s1; the last w mod 8 entries (and the zero padding) go to s0 in order.
// Fixed order -> deterministic.
template <class T, bool D16, class MT = T>
__device__ __forceinline__ T sell_row(const Sell& A, const MT* __restrict__ v, const T* __restrict__ x, int i) {
  const int s = i >> 5, lane = i & 31;
  const int b = A.base[s];
  const int w = A.width[s];
  const int w8 = w & ~7, wp = (w + 3) & ~3;
  T s0 = 0, s1 = 0;
  int k = 0;
  if constexpr (std::is_same<MT, __half>::value) {
    // the FP16 copy moves 4 B per entry: 16 entries in flight per thread
    // keep as many bytes in flight as 8 entries of the wider formats
    const int w16 = w & ~15;
    for (; k < w16; k += 16) {
      int j[16];
      T a[16];
#pragma unroll
      for (int g4 = 0; g4 < 4; ++g4) {
        const int o = sell_offset(b, lane, k + 4 * g4);
        sell_col4<D16>(A, o, i, j + 4 * g4);
        sell_vals4<T, MT>(v, o, a + 4 * g4);
      }
      T xv[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) xv[u] = x[j[u]];
#pragma unroll
      for (int u = 0; u < 16; u += 2) {
        s0 += a[u] * xv[u];
        s1 += a[u + 1] * xv[u + 1];
      }
    }
  }
  for (; k < w8; k += 8) {
    int j[8];
    T a[8];
    const int o0 = sell_offset(b, lane, k), o1 = o0 + 128;
    sell_col4<D16>(A, o0, i, j);
    sell_col4<D16>(A, o1, i, j + 4);
    sell_vals4<T, MT>(v, o0, a);
    sell_vals4<T, MT>(v, o1, a + 4);
    T xv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) xv[u] = x[j[u]];
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
      s0 += a[u] * xv[u];
      s1 += a[u + 1] * xv[u + 1];
    }
  }
  for (; k < wp; k += 4) {
    int j[4];
    T a[4];
    const int o = sell_offset(b, lane, k);
    sell_col4<D16>(A, o, i, j);
    sell_vals4<T, MT>(v, o, a);
#pragma unroll
    for (int u = 0; u < 4; ++u) s0 += a[u] * x[j[u]];
  }
  return s0 + s1;
}

// MODE SELL_Y:      y = A x
// MODE SELL_RESID:  y = b - A x (and y2 = y when y2 != null)
// MODE SELL_SMOOTH: y = x + w (b - A x) / den
// MODE SELL_DOT:    y = A x, partials of x.y (grid-stride; blockDim = kBlock)
// MT: the operator's value type (T, or __half for the FP16 copy whose values
// are a s, with vinv = 1 / s: a power of two, so the product is exact)
template <class T, int MODE, bool D16, class MT = T>
__global__ void __launch_bounds__(kBlock, 8) sell_spmv(Sell A, const MT* __restrict__ v, const T* __restrict__ x,
                                                    const T* __restrict__ b, const T* __restrict__ den, T w,
                                                    T* __restrict__ y, T* __restrict__ y2, double* __restrict__ part,
                                                    T vinv = T(1)) {
  if (MODE == SELL_DOT) {
    double acc[1] = {0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
      T s = sell_row<T, D16, MT>(A, v, x, i);
      if constexpr (!std::is_same<MT, T>::value) s *= vinv;
      y[i] = s;
      acc[0] += (double)x[i] * (double)s;
    }
    write_partials<1>(acc, part);
    return;
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  T s = sell_row<T, D16, MT>(A, v, x, i);
  if constexpr (!std::is_same<MT, T>::value) s *= vinv;
  if (MODE == SELL_Y) {
    y[i] = s;
  } else if (MODE == SELL_RESID) {
    // y = r; y2 = r (den null) or the first Jacobi step w r / den
    const T q = b[i] - s;
    y[i] = q;
    if (den) y2[i] = w * q / den[i];
    else if (y2) y2[i] = q;
  } else {
    // smoothing step; with y2 the step is added to y2 instead of stored
    const T val = x[i] + w * (b[i] - s) / den[i];
    if (y2) y2[i] += val;
    else y[i] = val;
  }
}

// Static part of the fine Schur refresh: for every directed contribution q of
// row c (basis a of c, incidence (c2, b) of the shared velocity dof), the
// geometric factor G_q = B[c][a] . B[c2][b].  Evaluated once at setup.
// cs[q]: basis a in bits 0-2 (0xFFFF: pad entry, G = 0); cpk[q] = c2 << 3 | b.
template <class T>
__global__ void refresh_geometry(int nc, const int32_t* __restrict__ coff, const uint32_t* __restrict__ cpk,
                                 const uint16_t* __restrict__ cs, const T* __restrict__ bco, T* __restrict__ G) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const T* Bc = bco + 24 * (size_t)c;
  for (int q = coff[c]; q < coff[c + 1]; ++q) {
    if (cs[q] == 0xFFFFu) {
      G[q] = T(0);
      continue;
    }
    const int a = cs[q] & 7;
    const uint32_t pk = cpk[q];
    const T* bb = bco + 24 * (size_t)(pk >> 3) + 3 * (pk & 7u);
    G[q] = Bc[3 * a] * bb[0] + Bc[3 * a + 1] * bb[1] + Bc[3 * a + 2] * bb[2];
  }
}

// Fine Schur numeric refresh A_p = B diag(rau) B^T (h8_precomputed_b.cuh:37-91)
// into the SELL layout.  Each value is sum_q rau_{g(c,a_q)} G_q over the
// row's contributions to that entry, in the reference's (basis, incidence)
// order (h2b_fine_csr.cuh:480-520), each product rounded on its own.  The
// contributions of a row are stored as runs, one per fine entry (the row's
// longest runs first), that never straddle a 32-entry chunk; the code word
// cs gives the basis a (bits 0-2), the position in the run (bits 3-5), the
// run's last entry (bit 6) and the entry's slot (bits 7-15); pads are
// 0xFFFF.  The next chunk's code words and factors are loaded before the
// current chunk is summed.
//
// One block of 32 warps per SELL slice, a warp per row, a lane per
// contribution: a shuffle chain sums every run sequentially (the lane at
// position j adds its product to the finished sum of position j-1), so each
// value is the reference's serial sum; no atomics.  The run's last lane
// puts the value into the slice's shared-memory image ([entry][row], row
// stride 33 against bank conflicts), which the block then writes out
// contiguously in SELL order (padding as zeros).  Values go to val
// (operator precision T) and, in the mixed modes, also to valA (AMG precision
// TA) and valH (FP16, scaled by hscale and saturated); the diagonal and L1
// row sums feed the AMG smoothers.
// Launch: blockDim 1024; dynamic shared memory 33 * padded max width * sizeof(T).
constexpr int kRefreshBlock = 1024;
template <class T>
__device__ __forceinline__ T mul_rn(T a, T b);
template <>
__device__ __forceinline__ double mul_rn<double>(double a, double b) { return __dmul_rn(a, b); }
template <>
__device__ __forceinline__ float mul_rn<float>(float a, float b) { return __fmul_rn(a, b); }
template <class T, class TA>
__global__ void __launch_bounds__(kRefreshBlock) sell_refresh(int nc, const int32_t* __restrict__ coff,
                                                              const uint16_t* __restrict__ cs, const T* __restrict__ G,
                                                              const int32_t* __restrict__ ref, const T* __restrict__ rau,
                                                              const int32_t* __restrict__ dslot,
                                                              const int32_t* __restrict__ sbase,
                                                              const int32_t* __restrict__ swidth, T* __restrict__ val,
                                                              TA* __restrict__ valA, TA* __restrict__ diag,
                                                              TA* __restrict__ l1, __half* __restrict__ valH = nullptr,
                                                              float hscale = 1.f) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sv = reinterpret_cast<T*>(smem_raw);
  __shared__ T sR[32][8];
  const int slice = blockIdx.x;
  const int width = (swidth[slice] + 3) & ~3;  // padded to the 4-wide lanes
  for (int t = threadIdx.x; t < 33 * width; t += blockDim.x) sv[t] = T(0);
  const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
  const int c = slice * 32 + r;
  const bool live_row = c < nc;
  int qb = 0, qe = 0, ds = -1;
  // the code word and factor of this lane's contribution in the next chunk,
  // loaded one chunk ahead (the first chunk's loads overlap the rAU staging)
  unsigned vn = 0xFFFFu;
  T gn = 0;
  if (live_row) {
    if (lane < 8) {
      const int g = ref[8 * (size_t)c + lane];
      sR[r][lane] = g >= 0 ? rau[g] : T(0);
    }
    qb = coff[c];
    qe = coff[c + 1];
    ds = dslot[c];
    if (qb + lane < qe) {
      vn = cs[qb + lane];
      gn = G[qb + lane];
    }
  }
  __syncthreads();  // image zeroed, rAU of every row staged
  T asum = 0;
  for (int q0 = qb; q0 < qe; q0 += 32) {  // warp-uniform bounds
    const unsigned v = vn;
    const T gq = gn;
    vn = 0xFFFFu;
    gn = 0;
    if (q0 + 32 + lane < qe) {
      vn = cs[q0 + 32 + lane];
      gn = G[q0 + 32 + lane];
    }
    // each product rounded on its own, then summed serially along the run
    const T p = v != 0xFFFFu ? mul_rn<T>(sR[r][v & 7u], gq) : T(0);
    const bool real = v != 0xFFFFu;
    const int pos = real ? (int)((v >> 3) & 7u) : 0;
    const int maxpos = __reduce_max_sync(0xffffffffu, pos);
    T acc = p;
    for (int j = 1; j <= maxpos; ++j) {
      const T up = __shfl_up_sync(0xffffffffu, acc, 1);
      if (pos == j) acc = up + p;
    }
    if (real && (v & 64u)) {
      const int sl = (int)(v >> 7);
      sv[sl * 33 + r] = acc;
      if (sl == ds) diag[c] = TA(acc);
      asum += fabs(acc);
    }
  }
  if (l1 && live_row) {
    asum = warp_sum(asum);
    if (lane == 0) l1[c] = TA(asum);
  }
  __syncthreads();
  const size_t base = (size_t)sbase[slice];
  for (int t = threadIdx.x; t < 32 * width; t += blockDim.x) {
    // element t of the slice is entry 4 (t/128) + t%4 of row (t/4)%32
    const T v = sv[(4 * (t >> 7) + (t & 3)) * 33 + ((t >> 2) & 31)];
    val[base + t] = v;
    if (valA) valA[base + t] = TA(v);
    if (valH) valH[base + t] = __float2half_rn(fminf(fmaxf((float)v * hscale, -65504.f), 65504.f));
  }
}

template <class Tin, class Tout>
__global__ void cast_copy(int n, const Tin* __restrict__ a, Tout* __restrict__ b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = Tout(a[i]);
}
// b = a in the other precision, and the fine pre-smoother's diagonal step
// x1 = w0 b / den0
template <class Tin, class Tout>
__global__ void cast_jacobi(int n, const Tin* __restrict__ a, Tout* __restrict__ b, Tout w0,
                            const Tout* __restrict__ den0, Tout* __restrict__ x1) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Tout v = Tout(a[i]);
  b[i] = v;
  x1[i] = w0 * v / den0[i];
}

// multicolour GS colour pass on the SELL fine operator (thread per row)
template <class T, bool D16>
__global__ void sell_gs_color(int count, const int32_t* __restrict__ rows, Sell A, const T* __restrict__ v,
                              const T* __restrict__ diag, const T* __restrict__ b, T* __restrict__ x, T omega) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int i = rows[q];
  const int s = i >> 5;
  const int base = A.base[s];
  T off = 0;
  for (int k = 0; k < A.width[s]; ++k) {
    const int o = sell_offset(base, i & 31, k);
    const int j = sell_col<D16>(A, o, i);
    if (j != i) off += v[o] * x[j];
  }
  const T old = x[i];
  const T gs = (b[i] - off) / diag[i];
  x[i] = old + omega * (gs - old);
}

// c = P^T f, a kRowLanes group per coarse row over R = P^T (deterministic
// tree per row)
template <class T, int GL = kRowLanes>
__global__ void __launch_bounds__(kBlock) restrict_rows(int nc, const int32_t* __restrict__ rr,
                                                        const int32_t* __restrict__ rc, const T* __restrict__ rv,
                                                        const T* __restrict__ f, T* __restrict__ c,
                                                        const T* __restrict__ den0, T w0, T* __restrict__ x1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int I = t / GL, lane = t % GL;
  if (I >= nc) return;
  const T s = group_row_dot<T, T, int32_t, GL>(rr, rc, rv, f, I, lane, group_mask<GL>());
  if (lane == 0) {
    c[I] = s;
    // with x1: the coarse pre-smoother's diagonal step w0 c / den0
    if (x1) x1[I] = w0 * s / den0[I];
  }
}

}  // namespace k
}  // namespace nds
