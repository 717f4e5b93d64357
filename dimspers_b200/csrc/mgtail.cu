// The small end of the V-cycle in one launch (option mg_tail, off by default).
//
// Below about 16k elements a multigrid level is too small to fill the GPU: each
// of its kernels (Chebyshev steps, applies, transfers) runs for ~1 us but costs
// ~2.5 us of launch and drain, and a V-cycle has ~13 of them per level.  This
// kernel runs every level from the first small one down to the coarsest, and
// back up, as ONE thread-block cluster (up to 16 CTAs, one GPC): the phases
// are the same per-element / per-node operations as the separate kernels, in
// the same order, separated by cluster barriers (barrier.cluster with release /
// acquire semantics) instead of kernel boundaries.  Vectors rewritten inside
// the kernel are read with ld.global.cg (L2, coherent across the cluster's
// SMs); element matrices and block inverses are constant during the kernel.
//
// Control flow is uniform: every thread walks the same phase sequence and
// reaches every barrier (no early return), so the cluster cannot deadlock.
//
// Measured on B200 it does not pay: a phase still waits for one L2 round trip
// and for the release of its stores and atomics before the barrier, on 16 SMs
// instead of all of them, so it costs as much as the separate launch it
// replaces (128x1024: 400 us per inner iteration with separate kernels, 445-
// 470 us with the tail from 8x64 or 16x128 down).  It stays as an option.
#include <cooperative_groups.h>

#include <cstring>

#include "kernels.cuh"
#include "mg.cuh"

namespace cg = cooperative_groups;

namespace dp {

constexpr int kTailMaxLevels = 8;
constexpr int kTailThreads = 512;

template <typename T>
struct TailLevel {
  const T* K;           // packed element matrices (AoSoA)
  const T* dinv;        // 2x2 nodal block inverses (3 per node)
  const double* cheb;   // Chebyshev recurrence coefficients
  T *x, *b, *r, *d, *t; // level vectors (2 per node)
  int ncr, nct, pin, nel, nnod, A, B;
  int degree;           // Chebyshev steps on this level
};

template <typename T>
struct TailArgs {
  TailLevel<T> L[kTailMaxLevels];
  int nlev;            // tail levels; the last is the coarsest
  int first_done;      // top level: the first smoothing step was fused into the restriction
  const double* inv;   // dense inverse of the coarsest level (ninv x ninv), or null
  int ninv;
  int coarse_sweeps;   // Chebyshev sweeps on the coarsest when it is not solved densely
};

template <typename T>
__device__ __forceinline__ T ld2(const T* p) { return __ldcg(p); }

// y += K x over the level's elements
template <typename T>
__device__ __forceinline__ void tail_apply(const TailLevel<T>& L, const T* x, T* y, int tid, int nth) {
  for (int e = tid; e < L.nel; e += nth) apply_element<T, T, true>(L.K, x, y, e, L.ncr, L.A, L.B);
}

// The tail's smoother keeps A d in the accumulator t (zeroed by each step)
// rather than subtracting it from r in the apply as the separate kernels do:
// the form is older, and the tail is an option that measured slower anyway.
// First step per node: r = b, d = x = coef[0] D^-1 b, t = 0
template <typename T>
__device__ __forceinline__ void tail_cheb_first(const TailLevel<T>& L, int tid, int nth) {
  const double it = L.cheb[0];
  for (int n = tid; n < L.nnod; n += nth) {
    const double b0 = (double)ld2(L.b + 2 * n), b1 = (double)ld2(L.b + 2 * n + 1);
    double z0, z1;
    bj_apply<T>(L.dinv, n, b0, b1, z0, z1);
    L.t[2 * n] = (T)0; L.t[2 * n + 1] = (T)0;
    L.r[2 * n] = (T)b0; L.r[2 * n + 1] = (T)b1;
    L.d[2 * n] = (T)(it * z0); L.d[2 * n + 1] = (T)(it * z1);
    L.x[2 * n] = (T)(it * z0); L.x[2 * n + 1] = (T)(it * z1);
  }
}

// First step from a given x, per node: r = b - (A x held in r), d = coef[0] D^-1 r, x += d, t = 0
template <typename T>
__device__ __forceinline__ void tail_cheb_first_x(const TailLevel<T>& L, int tid, int nth) {
  const double it = L.cheb[0];
  for (int n = tid; n < L.nnod; n += nth) {
    const double r0 = (double)ld2(L.b + 2 * n) - (double)ld2(L.r + 2 * n);
    const double r1 = (double)ld2(L.b + 2 * n + 1) - (double)ld2(L.r + 2 * n + 1);
    double z0, z1;
    bj_apply<T>(L.dinv, n, r0, r1, z0, z1);
    L.t[2 * n] = (T)0; L.t[2 * n + 1] = (T)0;
    L.r[2 * n] = (T)r0; L.r[2 * n + 1] = (T)r1;
    L.d[2 * n] = (T)(it * z0); L.d[2 * n + 1] = (T)(it * z1);
    L.x[2 * n] = ld2(L.x + 2 * n) + (T)(it * z0);
    L.x[2 * n + 1] = ld2(L.x + 2 * n + 1) + (T)(it * z1);
  }
}

// Chebyshev step per node: r -= t; d = c1 d + c2 D^-1 r; x += d; t = 0
template <typename T>
__device__ __forceinline__ void tail_cheb_step(const TailLevel<T>& L, const double* coef, int tid, int nth) {
  const double c1 = coef[0], c2 = coef[1];
  for (int n = tid; n < L.nnod; n += nth) {
    const double r0 = (double)ld2(L.r + 2 * n) - (double)ld2(L.t + 2 * n);
    const double r1 = (double)ld2(L.r + 2 * n + 1) - (double)ld2(L.t + 2 * n + 1);
    L.t[2 * n] = (T)0; L.t[2 * n + 1] = (T)0;
    double z0, z1;
    bj_apply<T>(L.dinv, n, r0, r1, z0, z1);
    const double d0 = c1 * (double)ld2(L.d + 2 * n) + c2 * z0;
    const double d1 = c1 * (double)ld2(L.d + 2 * n + 1) + c2 * z1;
    L.r[2 * n] = (T)r0; L.r[2 * n + 1] = (T)r1;
    L.d[2 * n] = (T)d0; L.d[2 * n + 1] = (T)d1;
    L.x[2 * n] = ld2(L.x + 2 * n) + (T)d0;
    L.x[2 * n + 1] = ld2(L.x + 2 * n + 1) + (T)d1;
  }
}

// Chebyshev smoothing on level L (the phases of chebyshev() in mg.cu).
// mode 0: from x = 0; 1: from x = 0, first step already taken; 2: from x (r zero on entry).
template <typename T>
__device__ void tail_smooth(const TailLevel<T>& L, int mode, cg::cluster_group& cl, int tid, int nth) {
  if (mode == 0) {
    tail_cheb_first(L, tid, nth);
    cl.sync();
  } else if (mode == 2) {
    tail_apply(L, L.x, L.r, tid, nth);
    cl.sync();
    tail_cheb_first_x(L, tid, nth);
    cl.sync();
  }
  for (int k = 1; k < L.degree; ++k) {
    tail_apply(L, L.d, L.t, tid, nth);
    cl.sync();
    tail_cheb_step(L, L.cheb + 2 * k, tid, nth);
    cl.sync();
  }
}

// bc = P^T (r - t) of the fine level F into the coarse level C (k_restrict_g),
// optionally with C's first Chebyshev step from x = 0.
template <typename T>
__device__ void tail_restrict(const TailLevel<T>& F, const TailLevel<T>& C, int first, int tid, int nth) {
  typedef typename V2<T>::T X2;
  const X2* r2 = reinterpret_cast<const X2*>(F.r);
  const X2* t2 = reinterpret_cast<const X2*>(F.t);
  const int Af = F.A, Bf = F.B, Ac = C.A, Bc = C.B, pin = C.pin;
  // the four parity classes run side by side on quarters of the cluster's
  // threads (nth / 4 is a multiple of 32, so every warp has one class and the
  // stencil reads are constant-cache broadcasts)
  const int q = nth >> 2;
  const int cls = tid / q, qtid = tid - cls * q;
  const int pa = cls & 1, pb = cls >> 1;
  const int nA = (Ac - pa + 1) >> 1;
  const int cnt = nA * (Bc >> 1);
  const int m = c_rtab.n[cls];
  for (int idx = qtid; idx < cnt; idx += q) {
    const int ac = 2 * (idx % nA) + pa, bcn = 2 * (idx / nA) + pb;
    double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
    for (int j = 0; j < m; ++j) {
      const int a = 2 * ac + c_rtab.da[cls][j];
      int b = 2 * bcn + c_rtab.db[cls][j];
      b += (b < 0) ? Bf : 0;
      b -= (b >= Bf) ? Bf : 0;
      const bool in = a >= 0 && a < Af;
      const int f = in ? a + Af * b : 0;
      const X2 rv = __ldcg(r2 + f), tv = __ldcg(t2 + f);
      const double w = c_rtab.w[cls][j];
      const double w0 = (in && !dof_fixed(a, b, 0, Af - 1, pin)) ? w : 0.0;
      const double w1 = (in && !dof_fixed(a, b, 1, Af - 1, pin)) ? w : 0.0;
      s0 += w0 * ((double)rv.x - (double)tv.x);
      s1 += w1 * ((double)rv.y - (double)tv.y);
    }
    const int n = ac + Ac * bcn;
    const double b0 = dof_fixed(ac, bcn, 0, Ac - 1, pin) ? 0.0 : s0;
    const double b1 = dof_fixed(ac, bcn, 1, Ac - 1, pin) ? 0.0 : s1;
    C.b[2 * n] = (T)b0;
    C.b[2 * n + 1] = (T)b1;
    if (first) {
      const double it = C.cheb[0];
      double z0, z1;
      bj_apply<T>(C.dinv, n, b0, b1, z0, z1);
      C.t[2 * n] = (T)0; C.t[2 * n + 1] = (T)0;
      C.r[2 * n] = (T)b0; C.r[2 * n + 1] = (T)b1;
      C.d[2 * n] = (T)(it * z0); C.d[2 * n + 1] = (T)(it * z1);
      C.x[2 * n] = (T)(it * z0); C.x[2 * n + 1] = (T)(it * z1);
    }
  }
}

// F.x += P C.x and F.r = 0 (the prolongation of k_prolong_add)
template <typename T>
__device__ void tail_prolong(const TailLevel<T>& F, const TailLevel<T>& C, int tid, int nth) {
  const int Af = F.A, pin = F.pin;
  for (int n = tid; n < F.nnod; n += nth) {
    const int a = n % Af, b = n / Af;
    int cn[6];
    double w[6];
    fine_node_weights(a, b, C.ncr, C.A, C.B, cn, w);
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if (w[k] != 0.0) {
        s0 += w[k] * (double)ld2(C.x + 2 * cn[k]);
        s1 += w[k] * (double)ld2(C.x + 2 * cn[k] + 1);
      }
    }
    if (!dof_fixed(a, b, 0, Af - 1, pin)) F.x[2 * n] = ld2(F.x + 2 * n) + (T)s0;
    if (!dof_fixed(a, b, 1, Af - 1, pin)) F.x[2 * n + 1] = ld2(F.x + 2 * n + 1) + (T)s1;
    F.r[2 * n] = (T)0;
    F.r[2 * n + 1] = (T)0;
  }
}

// x = Inv b on the coarsest level: each row is summed by a group of g lanes
// (g = 32, 16, 8 or 4: the widest that still gives every row its own group)
template <typename T>
__device__ void tail_dense(const TailLevel<T>& L, const double* inv, int n, int tid, int nth) {
  int g = 32;
  while (g > 4 && (nth / g) < n) g >>= 1;
  const int lane = tid & (g - 1);
  const int groups = nth / g;
  const int rounds = (n + groups - 1) / groups;  // same for every thread: the shuffles see full warps
  for (int k = 0; k < rounds; ++k) {
    const int row = tid / g + k * groups;
    double s = 0.0;
    if (row < n) {
      const double* a = inv + (size_t)row * n;
#pragma unroll 4
      for (int j = lane; j < n; j += g) s += a[j] * (double)ld2(L.b + j);
    }
    for (int o = g >> 1; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, g);
    if (row < n && lane == 0) L.x[row] = (T)s;
  }
}

template <typename T>
__device__ void tail_zero(T* v, int n, int tid, int nth) {
  for (int i = tid; i < n; i += nth) v[i] = (T)0;
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads) k_vcycle_tail(const TailArgs<T> a) {
  grid_dep_wait();
  cg::cluster_group cl = cg::this_cluster();
  const int tid = (int)cl.block_rank() * kTailThreads + (int)threadIdx.x;
  const int nth = (int)cl.num_blocks() * kTailThreads;
  const int last = a.nlev - 1;
  // down: pre-smoothing, residual, restriction (+ the coarse first step)
  for (int l = 0; l < last; ++l) {
    const TailLevel<T>& L = a.L[l];
    tail_smooth(L, (l > 0 || a.first_done) ? 1 : 0, cl, tid, nth);
    tail_apply(L, L.d, L.t, tid, nth);
    cl.sync();
    const bool first = !(l + 1 == last && a.inv);
    tail_restrict(L, a.L[l + 1], first ? 1 : 0, tid, nth);
    cl.sync();
  }
  // coarsest
  const TailLevel<T>& Lc = a.L[last];
  if (a.inv) {
    tail_dense(Lc, a.inv, a.ninv, tid, nth);
    cl.sync();
  } else {
    tail_smooth(Lc, (last > 0 || a.first_done) ? 1 : 0, cl, tid, nth);
    for (int s = 1; s < a.coarse_sweeps; ++s) {
      tail_zero(Lc.r, 2 * Lc.nnod, tid, nth);
      cl.sync();
      tail_smooth(Lc, 2, cl, tid, nth);
    }
  }
  // up: prolongation and post-smoothing
  for (int l = last - 1; l >= 0; --l) {
    tail_prolong(a.L[l], a.L[l + 1], tid, nth);
    cl.sync();
    tail_smooth(a.L[l], 2, cl, tid, nth);
  }
}

// ---- host side -----------------------------------------------------------------
template <typename T>
static const T* tail_K(const MGLevel& L);
template <>
const double* tail_K<double>(const MGLevel& L) { return L.K64; }
template <>
const float* tail_K<float>(const MGLevel& L) { return L.K32; }
template <typename T>
static const T* tail_dinv(const MGLevel& L);
template <>
const double* tail_dinv<double>(const MGLevel& L) { return L.dinv64; }
template <>
const float* tail_dinv<float>(const MGLevel& L) { return L.dinv32; }

// Cluster size for the tail kernel on this device (16 where the GPU can place a
// 16-CTA cluster of this kernel, else 8), cached per device and precision.
template <typename T>
static int tail_cluster_size() {
  static int cached[64] = {0};
  int dev = 0;
  DP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return 8;
  if (cached[dev]) return cached[dev];
  int size = 8;
  if (cudaFuncSetAttribute(k_vcycle_tail<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 16;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(kTailThreads);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, k_vcycle_tail<T>, &cfg) == cudaSuccess && nclusters >= 1) size = 16;
  }
  cudaGetLastError();  // a refused query leaves no sticky error
  cached[dev] = size;
  return size;
}

// First level that the tail kernel runs (the V-cycle from there down is one
// launch); c.mg.size() when the tail is off or no level is small enough.
size_t tail_start(const Ctx& c, const MGOptions& o) {
  const size_t n = c.mg.size();
  if (o.tail_max_el <= 0 || n == 0) return n;
  size_t s = n;
  for (size_t l = 0; l < n; ++l)
    if (c.mg[l].g.nel <= o.tail_max_el) { s = l; break; }
  if (s < n && n - s > (size_t)kTailMaxLevels) s = n - kTailMaxLevels;
  return s;
}

template <typename T>
void launch_vcycle_tail(Ctx& c, size_t l0, const T* b, T* x, bool first_done, const MGOptions& o) {
  TailArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  a.nlev = (int)(c.mg.size() - l0);
  a.first_done = first_done ? 1 : 0;
  a.coarse_sweeps = o.coarse_sweeps;
  a.inv = c.coarse_n > 0 ? c.coarse_inv + (size_t)c.coarse_n * c.coarse_n : nullptr;
  a.ninv = (int)c.coarse_n;
  for (int i = 0; i < a.nlev; ++i) {
    const MGLevel& M = c.mg[l0 + i];
    TailLevel<T>& L = a.L[i];
    L.K = tail_K<T>(M);
    L.dinv = tail_dinv<T>(M);
    L.cheb = M.cheb;
    L.x = (T*)M.x; L.b = (T*)M.b; L.r = (T*)M.r; L.d = (T*)M.d; L.t = (T*)M.t;
    L.ncr = M.g.ncr; L.nct = M.g.nct; L.pin = M.g.pin;
    L.degree = M.degree;
    L.nel = (int)M.g.nel; L.nnod = (int)M.g.nnod; L.A = (int)M.g.A(); L.B = (int)M.g.B();
  }
  // the top level's b and x are the caller's vectors
  a.L[0].b = const_cast<T*>(b);
  a.L[0].x = x;
  const int cs = tail_cluster_size<T>();
  cudaLaunchAttribute attr[3];
  unsigned na = 0;
  attr[na].id = cudaLaunchAttributeClusterDimension;
  attr[na].val.clusterDim.x = (unsigned)cs;
  attr[na].val.clusterDim.y = 1;
  attr[na].val.clusterDim.z = 1;
  ++na;
  if (g_pdl) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  if (g_prio != kNoPriority) {
    attr[na].id = cudaLaunchAttributePriority;
    attr[na].val.priority = g_prio;
    ++na;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cs);
  cfg.blockDim = dim3(kTailThreads);
  cfg.stream = c.stream;
  cfg.attrs = attr;
  cfg.numAttrs = na;
  ++g_klaunch;
  DP_CUDA(cudaLaunchKernelEx(&cfg, k_vcycle_tail<T>, a));
}

template void launch_vcycle_tail<float>(Ctx&, size_t, const float*, float*, bool, const MGOptions&);
template void launch_vcycle_tail<double>(Ctx&, size_t, const double*, double*, bool, const MGOptions&);

}  // namespace dp
