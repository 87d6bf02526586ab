// Shared device helpers for the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace nds {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess)
    throw CudaError(std::string("CUDA failure ") + what + " at " + file + ":" + std::to_string(line) + ": " +
                    cudaGetErrorString(e));
}
#define NDS_CUDA(call) ::nds::cuda_check((call), #call, __FILE__, __LINE__)
// every kernel launch of the library goes through NDS_LAUNCH, which also
// counts launches (nds_launch_count)
extern unsigned long long g_launches;
#define NDS_LAUNCH() (++::nds::g_launches, ::nds::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__))

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;

inline int grid_for(long long n, int per_block = kBlock) {
  long long g = (n + per_block - 1) / per_block;
  return (int)(g < 1 ? 1 : g);
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// sum over an aligned group of G lanes (G a power of two <= 32); mask names
// exactly the lanes of the calling group, which may have diverged from the
// other groups of its warp
template <int G, class T>
__device__ __forceinline__ T group_sum(T v, unsigned mask) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
  return v;
}
// lanes of the aligned 8-lane group of the calling thread
__device__ __forceinline__ unsigned group8_mask() { return 0xffu << (threadIdx.x & 24); }
// lanes of the aligned G-lane group of the calling thread (G = 8, 16 or 32)
template <int G>
__device__ __forceinline__ unsigned group_mask() {
  return G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (threadIdx.x & (32 - G)));
}

// Deterministic block reduction of NV doubles; thread 0 holds the sums.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double red[kWarps][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) red[w][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0;
      for (int q = 0; q < kWarps; ++q) s += red[q][k];
      v[k] = s;
    }
  }
  __syncthreads();
}

}  // namespace nds
