// Deterministic block/grid reductions shared by the vector kernels.
//
// Every reduction kernel runs on a fixed grid; each block reduces its values
// with warp shuffles, stores one partial per value, and the last block to
// arrive (atomic ticket) sums the partials in index order.  The result is
// independent of scheduling, so repeated solves are bitwise reproducible as
// far as the reductions are concerned.
#pragma once
#include <cuda_runtime.h>

namespace dp {

constexpr int kRedBlocks = 592;   // 4 x 148 SMs
constexpr int kRedThreads = 256;

__device__ inline double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int NV>
__device__ inline void block_sum_n(double (&v)[NV], double (*sh)[32]) {
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) sh[j][wid] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = (threadIdx.x < (blockDim.x >> 5)) ? sh[j][threadIdx.x] : 0.0;
  if (wid == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum(v[j]);
  }
  __syncthreads();
}

// partial: NV * gridDim.x doubles; out[j] receives the total of value j.
template <int NV>
__device__ inline bool grid_finish(double (&v)[NV], double* partial, unsigned int* counter, double* const* out) {
  __shared__ double sh[NV][32];
  __shared__ bool last;
  block_sum_n<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) partial[j * gridDim.x + blockIdx.x] = v[j];
    __threadfence();
    const unsigned int ticket = atomicInc(counter, gridDim.x);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double s[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) s[j] = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
#pragma unroll
    for (int j = 0; j < NV; ++j) s[j] += ((volatile double*)partial)[j * gridDim.x + i];
  }
  block_sum_n<NV>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) *out[j] = s[j];
    *counter = 0;
  }
  return true;  // in every thread of the last block (thread 0 holds the sums)
}

inline int red_grid(long long n) {
  long long b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
  if (b > kRedBlocks) b = kRedBlocks;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace dp
