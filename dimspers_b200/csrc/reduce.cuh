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

constexpr int kRedBlocks = 1184;  // 8 x 148 SMs: 64 resident warps per SM keep enough loads in flight
constexpr int kRedThreads = 256;
// per-context partials: room for two double-double values (4 doubles) per block
constexpr int kPartialDoubles = 8 * 1024;
static_assert(4 * kRedBlocks <= kPartialDoubles, "reduction partial buffer too small for the grid");

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

// ---- compensated (double-double) accumulation ---------------------------------
// The Schur-complement dots, norms and means accumulate error-free: each thread
// keeps a (hi, lo) pair updated with Knuth's TwoSum and the FMA TwoProduct
// (the Dot2 / Sum2 algorithms of Ogita, Rump and Oishi, "Accurate sum and dot
// product", SIAM J. Sci. Comput. 26(6), 2005), and the block and grid
// combinations merge pairs with TwoSum followed by a renormalisation.  The
// result is as accurate as a plain sum carried out in twice the working
// precision and then rounded to double; the combination order is fixed, so it
// is bitwise reproducible like the plain reductions above.
struct DD {
  double hi, lo;
};

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
__device__ __forceinline__ void dd_add(DD& x, double v) {
  double s, e;
  two_sum(x.hi, v, s, e);
  x.hi = s;
  x.lo += e;
}
__device__ __forceinline__ void dd_add_prod(DD& x, double a, double b) {
  const double p = a * b;
  const double pe = fma(a, b, -p);   // exact: a*b = p + pe
  double s, e;
  two_sum(x.hi, p, s, e);
  x.hi = s;
  x.lo += e + pe;
}
__device__ __forceinline__ DD dd_merge(DD x, DD y) {
  double s, e;
  two_sum(x.hi, y.hi, s, e);
  e += x.lo + y.lo;
  DD r;
  r.hi = s + e;                       // renormalise (|s| >= |e| after TwoSum)
  r.lo = e - (r.hi - s);
  return r;
}
__device__ __forceinline__ DD warp_sum_dd(DD v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    DD w;
    w.hi = __shfl_down_sync(0xffffffffu, v.hi, o);
    w.lo = __shfl_down_sync(0xffffffffu, v.lo, o);
    v = dd_merge(v, w);
  }
  return v;
}

template <int NV>
__device__ inline void block_sum_dd(DD (&v)[NV], DD (*sh)[32]) {
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = warp_sum_dd(v[j]);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) sh[j][wid] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) v[j] = (threadIdx.x < (blockDim.x >> 5)) ? sh[j][threadIdx.x] : DD{0.0, 0.0};
  if (wid == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) v[j] = warp_sum_dd(v[j]);
  }
  __syncthreads();
}

// Compensated grid_finish: partial holds 2 * NV * gridDim.x doubles (hi and
// lo per block and value); out[j] receives hi + lo of the total of value j.
template <int NV>
__device__ inline bool grid_finish_dd(DD (&v)[NV], double* partial, unsigned int* counter, double* const* out) {
  __shared__ DD sh[NV][32];
  __shared__ bool last;
  block_sum_dd<NV>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      partial[2 * (j * gridDim.x + blockIdx.x)] = v[j].hi;
      partial[2 * (j * gridDim.x + blockIdx.x) + 1] = v[j].lo;
    }
    __threadfence();
    const unsigned int ticket = atomicInc(counter, gridDim.x);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  DD s[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) s[j] = DD{0.0, 0.0};
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      DD w;
      w.hi = ((volatile double*)partial)[2 * (j * gridDim.x + i)];
      w.lo = ((volatile double*)partial)[2 * (j * gridDim.x + i) + 1];
      s[j] = dd_merge(s[j], w);
    }
  }
  block_sum_dd<NV>(s, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) *out[j] = s[j].hi + s[j].lo;
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
