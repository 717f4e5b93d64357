// Operator applies, reductions and vector kernels.
//
// A-apply (K x): element-by-element from the stored packed polar element
// matrices (the element blocks of StokesSolver.jl:688-810 after the rotation
// of :192-201), gathering the 12 element DOFs through the analytic lattice
// connectivity and scatter-adding the 12 results.
// G / G^T applies: element-local 12x3 blocks (StokesSolver.jl:812-823), as the
// SpMVs GG*q and GG'*z of IterativeSolvers.jl:142,144.
// Dots: deterministic two-level reduction (warp shuffles -> block -> fixed-order
// sum of the per-block partials by the last block), the role of mydot /
// mynorm / vmean in Algebra.jl:104-113 and IterativeSolvers.jl:179-186.
#include <stdexcept>

#include "kernels.cuh"
#include "reduce.cuh"

namespace dp {

// ---- element-by-element K apply -------------------------------------------
// Loads the element's packed matrix as 16-byte vectors (all issued before the
// arithmetic, so each thread keeps 20-39 loads in flight), gathers x as one
// 8/16-byte load per node and scatter-adds y per node (float2 vector atomics
// for FP32).
template <typename Tm>
struct KVec;
template <>
struct KVec<float> { typedef float4 V; static constexpr int n = 20; };
template <>
struct KVec<double> { typedef double2 V; static constexpr int n = 39; };

__device__ inline void vec_to(const float4& v, float* k) { k[0] = v.x; k[1] = v.y; k[2] = v.z; k[3] = v.w; }
__device__ inline void vec_to(const double2& v, double* k) { k[0] = v.x; k[1] = v.y; }

__device__ inline void atomic_add2(float* y, float a, float b) { atomicAdd(reinterpret_cast<float2*>(y), make_float2(a, b)); }
__device__ inline void atomic_add2(double* y, double a, double b) { atomicAdd(y, a); atomicAdd(y + 1, b); }

template <typename Tv>
struct V2;
template <>
struct V2<float> { typedef float2 T; };
template <>
struct V2<double> { typedef double2 T; };

// Element of this thread.  wt == 1: linear order (CTA = blockDim consecutive
// elements).  wt > 1: the CTA is a tile of (blockDim/32/wt) x 16 radial cells by
// wt theta columns; each warp still reads one contiguous 32-element block of K
// (e = 2 (ir + ncr it) + t with ir = 16 m + lane/2, t = lane & 1).
__device__ inline int tile_element(int ncr, int wt) {
  if (wt == 1) return blockIdx.x * blockDim.x + threadIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wr = (blockDim.x >> 5) / wt;       // warps along r
  const int nbr = (ncr >> 4) / wr;              // CTAs along r
  const int br = blockIdx.x % nbr, bt = blockIdx.x / nbr;
  const int m = br * wr + w % wr, it = bt * wt + w / wr;
  return 32 * m + 2 * ncr * it + lane;
}

// ye = K_e x_e for element e, with the lattice index of each of its 6 nodes.
// kL2: read x with ld.global.cg (L2 only), for callers where other CTAs
// rewrite x during the same kernel.
template <typename Tm, typename Tv, bool kL2>
__device__ __forceinline__ void element_product(const Tm* __restrict__ K, const Tv* x, int e, int ncr, int A, int B,
                                                int nd[6], Tv ye[12]) {
  typedef typename KVec<Tm>::V VT;
  constexpr int NV = KVec<Tm>::n;
  constexpr int PER = sizeof(VT) / sizeof(Tm);
  const VT* Kb = reinterpret_cast<const VT*>(K + (int64_t)(e >> 5) * (32 * NV * PER)) + (e & 31);
  Tm kk[NV * PER];
#pragma unroll
  for (int j = 0; j < NV; ++j) vec_to(Kb[j * 32], kk + j * PER);
  const int q = e >> 1, t = e & 1;
  const int ir = q % ncr, it = q / ncr;
  const int a0 = 2 * ir, b0 = 2 * it;
  {
    int bb[6], aa[6];
    if (t == 0) {
      aa[0] = a0; aa[1] = a0; aa[2] = a0 + 2; aa[3] = a0; aa[4] = a0 + 1; aa[5] = a0 + 1;
      bb[0] = b0; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 1; bb[4] = b0 + 1; bb[5] = b0;
    } else {
      aa[0] = a0; aa[1] = a0 + 2; aa[2] = a0 + 2; aa[3] = a0 + 1; aa[4] = a0 + 2; aa[5] = a0 + 1;
      bb[0] = b0 + 2; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 2; bb[4] = b0 + 1; bb[5] = b0 + 1;
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) nd[k] = aa[k] + A * (bb[k] >= B ? bb[k] - B : bb[k]);
  }
  typedef typename V2<Tv>::T X2;
  const X2* x2 = reinterpret_cast<const X2*>(x);
  Tv xe[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const X2 v = kL2 ? __ldcg(x2 + nd[k]) : x2[nd[k]];
    xe[2 * k] = v.x;
    xe[2 * k + 1] = v.y;
    ye[2 * k] = 0;
    ye[2 * k + 1] = 0;
  }
#pragma unroll
  for (int C = 0; C < 12; ++C) {
#pragma unroll
    for (int R = C; R < 12; ++R) {
      const Tv kv = (Tv)kk[packed_index12(R, C)];
      ye[R] += kv * xe[C];
      if (R != C) ye[C] += kv * xe[R];
    }
  }
}

// y += K_e x_e for element e (kSub: y -= K_e x_e), scatter-added with atomics.
template <typename Tm, typename Tv, bool kL2, bool kSub = false>
__device__ __forceinline__ void apply_element(const Tm* __restrict__ K, const Tv* x, Tv* y, int e, int ncr, int A,
                                              int B) {
  int nd[6];
  Tv ye[12];
  element_product<Tm, Tv, kL2>(K, x, e, ncr, A, B, nd, ye);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    if (kSub) atomic_add2(&y[2 * nd[k]], -ye[2 * k], -ye[2 * k + 1]);
    else atomic_add2(&y[2 * nd[k]], ye[2 * k], ye[2 * k + 1]);
  }
}

template <typename Tm, typename Tv, bool kSub = false>
__global__ void __launch_bounds__(256) k_apply_K(const Tm* __restrict__ K, const Tv* __restrict__ x,
                                                 Tv* __restrict__ y, int nel, int ncr, int A, int B, int wt) {
  grid_dep_wait();
  const int e = tile_element(ncr, wt);
  if (e >= nel) return;
  apply_element<Tm, Tv, false, kSub>(K, x, y, e, ncr, A, B);
}

// Deterministic form, pass 1: E[(2k + c) nel + e] = (K_e x_e) of local node k,
// component c (no atomics; k_node_gather sums the nodes in a fixed order).
template <typename Tm, typename Tv>
__global__ void __launch_bounds__(256) k_apply_K_elem(const Tm* __restrict__ K, const Tv* __restrict__ x,
                                                      Tv* __restrict__ E, int nel, int ncr, int A, int B) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int nd[6];
  Tv ye[12];
  element_product<Tm, Tv, false>(K, x, e, ncr, A, B, nd, ye);
#pragma unroll
  for (int d = 0; d < 12; ++d) E[(int64_t)d * nel + e] = ye[d];
}

// Local node k of triangle type t sits at lattice offset (kLocA, kLocB) from
// its cell origin (2 ir, 2 it): the node order of element_product.
__host__ __device__ constexpr int loc_a(int t, int k) {
  return t == 0 ? (k == 2 ? 2 : (k >= 4 ? 1 : 0)) : (k == 0 ? 0 : (k == 3 || k == 5 ? 1 : 2));
}
__host__ __device__ constexpr int loc_b(int t, int k) {
  return t == 0 ? (k == 1 ? 2 : (k == 3 || k == 4 ? 1 : 0)) : (k == 2 ? 0 : (k >= 4 ? 1 : 2));
}

// Deterministic form, pass 2: per lattice node n, the sum of E over the
// elements that contain it, taken in a fixed order (triangle type t = 0, 1,
// then local node k = 0..5), so the result is the same bit for bit in every
// run.  E[(NC k + c) nel + e] holds element e's value c at its local node k.
// MODE 0: y[NC n + c] += s; 1: y -= s; 2: y = s.
// One thread owns the 2x2 node block a = 2i + pa, b = 2j + pb (i <= ncr,
// j < nct): for each parity class (pa, pb) the elements holding the node are
// fixed at compile time (local node k of type t holds it iff loc_a(t, k) has
// the parity of a and loc_b(t, k) that of b; the element's cell is then
// (i + (pa - loc_a) / 2, j + (pb - loc_b) / 2), theta periodic), so a warp
// never diverges on them, and neighbouring lanes write neighbouring nodes.
template <int PA, int PB, typename T, int NC>
__device__ __forceinline__ void gather_class(const T* __restrict__ E, int i, int j, int ncr, int nct, int64_t nel,
                                             T s[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) s[c] = (T)0;
#pragma unroll
  for (int t = 0; t < 2; ++t) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      if ((loc_a(t, k) & 1) != PA || (loc_b(t, k) & 1) != PB) continue;   // resolved at compile time
      const int ir = i + ((PA - loc_a(t, k)) >> 1);
      int it = j + ((PB - loc_b(t, k)) >> 1);
      if (ir < 0 || ir >= ncr) continue;
      if (it < 0) it += nct;
      const int64_t e = 2 * ((int64_t)ir + (int64_t)ncr * it) + t;
#pragma unroll
      for (int c = 0; c < NC; ++c) s[c] += E[(int64_t)(NC * k + c) * nel + e];
    }
  }
}

template <int PA, int PB, typename T, int NC, int MODE>
__device__ __forceinline__ void gather_node(const T* __restrict__ E, T* __restrict__ y, int i, int j, int ncr, int nct,
                                            int64_t nel) {
  const int a = 2 * i + PA;
  if (a > 2 * ncr) return;
  T s[NC];
  gather_class<PA, PB, T, NC>(E, i, j, ncr, nct, nel, s);
  const int64_t n = a + (int64_t)(2 * ncr + 1) * (2 * j + PB);
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    T* p = y + NC * n + c;
    if (MODE == 0) *p += s[c];
    else if (MODE == 1) *p -= s[c];
    else *p = s[c];
  }
}

template <typename T, int NC, int MODE>
__global__ void __launch_bounds__(256) k_node_gather(const T* __restrict__ E, T* __restrict__ y, int ncr, int nct,
                                                     int64_t nel) {
  grid_dep_wait();
  const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (q >= (int64_t)(ncr + 1) * nct) return;
  const int j = (int)(q / (ncr + 1)), i = (int)(q - (int64_t)j * (ncr + 1));
  gather_node<0, 0, T, NC, MODE>(E, y, i, j, ncr, nct, nel);
  gather_node<1, 0, T, NC, MODE>(E, y, i, j, ncr, nct, nel);
  gather_node<0, 1, T, NC, MODE>(E, y, i, j, ncr, nct, nel);
  gather_node<1, 1, T, NC, MODE>(E, y, i, j, ncr, nct, nel);
}

template <typename T>
void launch_node_gather(const Level& L, const T* E, T* y, int nc, int mode, cudaStream_t s) {
  const int grid = (int)div_up((int64_t)(L.ncr + 1) * L.nct, 256);
#define DP_GATHER(NC, M) \
  klaunch(k_node_gather<T, NC, M>, grid, 256, 0, s, E, y, L.ncr, L.nct, (int64_t)L.nel)
  if (nc == 2) {
    if (mode == 0) DP_GATHER(2, 0);
    else if (mode == 1) DP_GATHER(2, 1);
    else DP_GATHER(2, 2);
  } else if (nc == 3 && mode == 2) {
    DP_GATHER(3, 2);
  } else {
    throw std::runtime_error("launch_node_gather: unsupported layout");
  }
#undef DP_GATHER
  DP_LAUNCH_CHECK();
}
template void launch_node_gather<double>(const Level&, const double*, double*, int, int, cudaStream_t);
template void launch_node_gather<float>(const Level&, const float*, float*, int, int, cudaStream_t);

// ---- matrix-free element-by-element K apply (fine level) -------------------------
// K_e (polar DOFs, constrained rows/columns masked) = sum_ip B0^T Dw_ip B0, with
// B0 = B_cart(ref) T(ref) of the ring's reference element (it = 0) and Dw_ip =
// om Q^T D Q the element's viscous tensor rotated into that reference frame
// (written by the assembly).  Per element the apply reads 36 Dw values (144 B
// in FP32 instead of 312 B of packed matrix) and does ~400 FMA: node DOFs to
// the reference Cartesian frame, strain (exx, ezz, gxz) per IP, stress = Dw
// strain, back-projection, back to polar.  Threads run along r (the element
// order of the packed apply), so node gathers and atomics are contiguous; the
// per-ring table is value-major, so the lanes of a warp (consecutive rings)
// read it with coalesced loads.
template <typename T, bool kSub = false>
__global__ void __launch_bounds__(256) k_apply_K_mf(const T* __restrict__ Dw, const T* __restrict__ tab,
                                                    const T* __restrict__ x, T* __restrict__ y, int ncr, int nct,
                                                    int A, int B, int pin) {
  grid_dep_wait();
  const int nel = 2 * ncr * nct;
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= nel) return;
  const int q = gid >> 1, t = gid & 1;
  const int ir = q % ncr, it = q / ncr;
  const int ring = 2 * ir + t, nring = 2 * ncr;
  const int a0 = 2 * ir, b0 = 2 * it;
  int aa[6], bb[6];
  if (t == 0) {
    aa[0] = a0; aa[1] = a0; aa[2] = a0 + 2; aa[3] = a0; aa[4] = a0 + 1; aa[5] = a0 + 1;
    bb[0] = b0; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 1; bb[4] = b0 + 1; bb[5] = b0;
  } else {
    aa[0] = a0; aa[1] = a0 + 2; aa[2] = a0 + 2; aa[3] = a0 + 1; aa[4] = a0 + 2; aa[5] = a0 + 1;
    bb[0] = b0 + 2; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 2; bb[4] = b0 + 1; bb[5] = b0 + 1;
  }
  const T* tb = tab + ring;
  typedef typename V2<T>::T X2;
  const X2* x2 = reinterpret_cast<const X2*>(x);
  const int amax = 2 * ncr;
  int nd[6];
  bool ft[6], fr[6];
  T ux[6], uz[6], fx[6], fz[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int b = bb[k] >= B ? bb[k] - B : bb[k];
    nd[k] = aa[k] + A * b;
    ft[k] = dof_fixed(aa[k], b, 0, amax, pin);
    fr[k] = dof_fixed(aa[k], b, 1, amax, pin);
    const X2 v = x2[nd[k]];
    const T x0 = ft[k] ? (T)0 : v.x, x1 = fr[k] ? (T)0 : v.y;
    const T c = __ldg(tb + (72 + 2 * k) * nring), s = __ldg(tb + (73 + 2 * k) * nring);
    ux[k] = c * x0 + s * x1;
    uz[k] = c * x1 - s * x0;
    fx[k] = (T)0;
    fz[k] = (T)0;
  }
  const size_t st = (size_t)nel;
  const T* D = Dw + gid;
  // the IP loop stays rolled (the table is read per IP, warp-uniform, from
  // L1) and the next IP's six tensor values are loaded one IP ahead
  T dn[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) dn[v] = D[v * st];
#pragma unroll 1
  for (int ip = 0; ip < 6; ++ip) {
    const T d11 = dn[0], d12 = dn[1], d13 = dn[2], d22 = dn[3], d23 = dn[4], d33 = dn[5];
    if (ip < 5) {
      const T* Dn = D + (size_t)((ip + 1) * 6) * st;
#pragma unroll
      for (int v = 0; v < 6; ++v) dn[v] = Dn[v * st];
    }
    const T* tq = tb + ip * 12 * nring;
    T exx = 0, ezz = 0, gxz = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const T dxk = __ldg(tq + k * nring), dzk = __ldg(tq + (6 + k) * nring);
      exx += dxk * ux[k];
      ezz += dzk * uz[k];
      gxz += dzk * ux[k] + dxk * uz[k];
    }
    const T sxx = d11 * exx + d12 * ezz + d13 * gxz;
    const T szz = d12 * exx + d22 * ezz + d23 * gxz;
    const T sxz = d13 * exx + d23 * ezz + d33 * gxz;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const T dxk = __ldg(tq + k * nring), dzk = __ldg(tq + (6 + k) * nring);
      fx[k] += dxk * sxx + dzk * sxz;
      fz[k] += dzk * szz + dxk * sxz;
    }
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const T c = __ldg(tb + (72 + 2 * k) * nring), s = __ldg(tb + (73 + 2 * k) * nring);
    const T y0 = ft[k] ? (T)0 : c * fx[k] - s * fz[k];
    const T y1 = fr[k] ? (T)0 : s * fx[k] + c * fz[k];
    if (kSub) atomic_add2(&y[2 * nd[k]], -y0, -y1);
    else atomic_add2(&y[2 * nd[k]], y0, y1);
  }
}

template <typename T>
static inline const T* mf_data(const Level& L);
template <>
inline const double* mf_data<double>(const Level& L) { return L.mfD64; }
template <>
inline const float* mf_data<float>(const Level& L) { return L.mfD32; }
template <typename T>
static inline const T* mf_table(const Level& L);
template <>
inline const double* mf_table<double>(const Level& L) { return L.mfT64; }
template <>
inline const float* mf_table<float>(const Level& L) { return L.mfT32; }

// Grid of the tiled apply; the stacked tile only where it divides the lattice
// exactly (ncr % (16 wr) == 0, nct % wt == 0), else the linear order.
static void apply_tile(const Level& L, int& blocks, int& threads, int& wt) {
  threads = 32 * L.warps;
  wt = L.warps_t;
  const int wr = L.warps / std::max(wt, 1);
  if (wt > 1 && wr >= 1 && L.warps % wt == 0 && L.ncr % (16 * wr) == 0 && L.nct % wt == 0) {
    blocks = (L.ncr / (16 * wr)) * (L.nct / wt);
  } else {
    wt = 1;
    blocks = (int)div_up(L.nel, threads);
  }
}

// kMode 0: y += K x, 1: y -= K x, 2: y = K x (the atomic form zeroes y
// first).  With L.det set the apply runs as two passes without atomics
// (element results, then the fixed-order node gather).
template <int kMode, typename Tm, typename Tv>
static void apply_K_into(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s) {
  constexpr bool kSub = kMode == 1;
  if (L.det) {
    Tv* E = static_cast<Tv*>(L.det);
    klaunch(k_apply_K_elem<Tm, Tv>, (int)div_up(L.nel, 256), 256, 0, s, K, x, E, (int)L.nel, L.ncr, (int)L.A(),
            (int)L.B());
    DP_LAUNCH_CHECK();
    launch_node_gather<Tv>(L, E, y, 2, kMode, s);
    return;
  }
  if (kMode == 2) DP_CUDA(cudaMemsetAsync(y, 0, sizeof(Tv) * 2 * L.nnod, s));
  if (std::is_same<Tm, Tv>::value && mf_data<Tv>(L) && mf_table<Tv>(L)) {
    klaunch(k_apply_K_mf<Tv, kSub>, (int)div_up(L.nel, 256), 256, 0, s, mf_data<Tv>(L), mf_table<Tv>(L), x, y, L.ncr,
            L.nct, (int)L.A(), (int)L.B(), L.pin);
    DP_LAUNCH_CHECK();
    return;
  }
  int blocks, threads, wt;
  apply_tile(L, blocks, threads, wt);
  klaunch(k_apply_K<Tm, Tv, kSub>, blocks, threads, 0, s, K, x, y, (int)L.nel, L.ncr, (int)L.A(), (int)L.B(), wt);
  DP_LAUNCH_CHECK();
}

template <typename Tm, typename Tv>
void launch_apply_K(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s) {
  apply_K_into<2>(L, K, x, y, s);
}
template void launch_apply_K<double, double>(const Level&, const double*, const double*, double*, cudaStream_t);
template void launch_apply_K<float, float>(const Level&, const float*, const float*, float*, cudaStream_t);

// y += K x (the caller has zeroed y, typically inside the preceding vector kernel)
template <typename Tm, typename Tv>
void launch_apply_K_acc(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s) {
  apply_K_into<0>(L, K, x, y, s);
}
template void launch_apply_K_acc<double, double>(const Level&, const double*, const double*, double*, cudaStream_t);
template void launch_apply_K_acc<float, float>(const Level&, const float*, const float*, float*, cudaStream_t);

// y -= K x: the smoother keeps its residual in y and lets the apply update it
// in place (no accumulator to zero and re-read)
template <typename Tm, typename Tv>
void launch_apply_K_sub(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s) {
  apply_K_into<1>(L, K, x, y, s);
}
template void launch_apply_K_sub<double, double>(const Level&, const double*, const double*, double*, cudaStream_t);
template void launch_apply_K_sub<float, float>(const Level&, const float*, const float*, float*, cudaStream_t);

// ---- G / G^T ----------------------------------------------------------------
__device__ inline void element_nodes_dev(int e, int ncr, int A, int B, int nd[6]) {
  const int q = e >> 1, t = e & 1;
  const int ir = q % ncr, it = q / ncr;
  const int a0 = 2 * ir, b0 = 2 * it;
  int aa[6], bb[6];
  if (t == 0) {
    aa[0] = a0; aa[1] = a0; aa[2] = a0 + 2; aa[3] = a0; aa[4] = a0 + 1; aa[5] = a0 + 1;
    bb[0] = b0; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 1; bb[4] = b0 + 1; bb[5] = b0;
  } else {
    aa[0] = a0; aa[1] = a0 + 2; aa[2] = a0 + 2; aa[3] = a0 + 1; aa[4] = a0 + 2; aa[5] = a0 + 1;
    bb[0] = b0 + 2; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 2; bb[4] = b0 + 1; bb[5] = b0 + 1;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) nd[k] = aa[k] + A * (bb[k] >= B ? bb[k] - B : bb[k]);
}

__device__ inline void element_pdofs_dev(int e, int ncr, int nct, int pressure, int pd[3]) {
  if (pressure == 1) {
    pd[0] = 3 * e; pd[1] = 3 * e + 1; pd[2] = 3 * e + 2;
    return;
  }
  const int q = e >> 1, t = e & 1;
  const int ir = q % ncr, it = q / ncr;
  const int nr = ncr + 1;
  const int it1 = (it + 1 == nct) ? 0 : it + 1;
  const int v1 = ir + nr * it, v2 = ir + nr * it1, v3 = ir + 1 + nr * it1, v4 = ir + 1 + nr * it;
  if (t == 0) { pd[0] = v1; pd[1] = v2; pd[2] = v4; }
  else        { pd[0] = v2; pd[1] = v3; pd[2] = v4; }
}

__global__ void k_apply_G(const double* __restrict__ G, const double* __restrict__ p, double* __restrict__ y,
                          int nel, int ncr, int nct, int A, int B, int pressure) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int nd[6], pd[3];
  element_nodes_dev(e, ncr, A, B, nd);
  element_pdofs_dev(e, ncr, nct, pressure, pd);
  const double p0 = p[pd[0]], p1 = p[pd[1]], p2 = p[pd[2]];
#pragma unroll
  for (int d = 0; d < 12; ++d) {
    const double v = G[(size_t)d * nel + e] * p0 + G[(size_t)(12 + d) * nel + e] * p1 +
                     G[(size_t)(24 + d) * nel + e] * p2;
    atomicAdd(&y[2 * nd[d >> 1] + (d & 1)], v);
  }
}

// Deterministic form of the G apply, pass 1: element e's 12 values of G_e p_e
// into E[d nel + e] (k_node_gather sums them per node).
__global__ void k_apply_G_elem(const double* __restrict__ G, const double* __restrict__ p, double* __restrict__ E,
                               int nel, int ncr, int nct, int pressure) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int pd[3];
  element_pdofs_dev(e, ncr, nct, pressure, pd);
  const double p0 = p[pd[0]], p1 = p[pd[1]], p2 = p[pd[2]];
#pragma unroll
  for (int d = 0; d < 12; ++d)
    E[(size_t)d * nel + e] = G[(size_t)d * nel + e] * p0 + G[(size_t)(12 + d) * nel + e] * p1 +
                             G[(size_t)(24 + d) * nel + e] * p2;
}

__global__ void k_apply_GT(const double* __restrict__ G, const double* __restrict__ x, double* __restrict__ p,
                           int nel, int ncr, int nct, int A, int B, int pressure) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int nd[6], pd[3];
  element_nodes_dev(e, ncr, A, B, nd);
  element_pdofs_dev(e, ncr, nct, pressure, pd);
  double xe[12];
#pragma unroll
  for (int k = 0; k < 6; ++k) { xe[2 * k] = x[2 * nd[k]]; xe[2 * k + 1] = x[2 * nd[k] + 1]; }
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < 12; ++d) s += G[(size_t)(i * 12 + d) * nel + e] * xe[d];
    if (pressure == 1) p[pd[i]] = s;
    else atomicAdd(&p[pd[i]], s);
  }
}

// y = G p with the scatter pre-summed per warp: with ncr a multiple of 16 the 32
// elements of a warp are the two triangles of 16 consecutive cells of one theta
// column, which share 33 x 3 = 99 lattice nodes.  The warp adds its 384 values
// into a shared-memory copy of those nodes first and then issues one global FP64
// atomic per node and component (198), since sm_100a has no vector FP64 reduction.
constexpr int kGWarpNodes = 99;
__global__ void __launch_bounds__(128) k_apply_G_warp(const double* __restrict__ G, const double* __restrict__ p,
                                                      double* __restrict__ y, int nel, int ncr, int nct, int A, int B,
                                                      int pressure) {
  grid_dep_wait();
  __shared__ double acc[4][2 * kGWarpNodes];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int e0 = e - lane;                        // first element of the warp (nel is a multiple of 32)
  if (e0 >= nel) return;                          // whole warps past the last element (tail block)
  const int q0 = e0 >> 1, ir0 = q0 % ncr, it = q0 / ncr;
  double* s = acc[w];
  for (int k = lane; k < 2 * kGWarpNodes; k += 32) s[k] = 0.0;
  __syncwarp();
  {
    const int q = e >> 1, t = e & 1;
    const int ir = q % ncr;
    int pd[3];
    element_pdofs_dev(e, ncr, nct, pressure, pd);
    const double p0 = p[pd[0]], p1 = p[pd[1]], p2 = p[pd[2]];
    // local lattice offsets (a relative to 2 ir0, b relative to 2 it) of the 6 nodes
    const int la0 = 2 * (ir - ir0);
    int la[6], lb[6];
    if (t == 0) {
      la[0] = la0; la[1] = la0; la[2] = la0 + 2; la[3] = la0; la[4] = la0 + 1; la[5] = la0 + 1;
      lb[0] = 0; lb[1] = 2; lb[2] = 0; lb[3] = 1; lb[4] = 1; lb[5] = 0;
    } else {
      la[0] = la0; la[1] = la0 + 2; la[2] = la0 + 2; la[3] = la0 + 1; la[4] = la0 + 2; la[5] = la0 + 1;
      lb[0] = 2; lb[1] = 2; lb[2] = 0; lb[3] = 2; lb[4] = 1; lb[5] = 1;
    }
#pragma unroll
    for (int d = 0; d < 12; ++d) {
      const double v = G[(size_t)d * nel + e] * p0 + G[(size_t)(12 + d) * nel + e] * p1 +
                       G[(size_t)(24 + d) * nel + e] * p2;
      const int k = d >> 1;
      atomicAdd(&s[2 * (la[k] + 33 * lb[k]) + (d & 1)], v);
    }
  }
  __syncwarp();
  for (int k = lane; k < kGWarpNodes; k += 32) {
    const int a = 2 * ir0 + k % 33, bl = 2 * it + k / 33;
    const int64_t n = a + (int64_t)A * (bl >= B ? bl - B : bl);
    atomicAdd(&y[2 * n], s[2 * k]);
    atomicAdd(&y[2 * n + 1], s[2 * k + 1]);
  }
}

void launch_apply_G(Ctx& c, const double* p, double* y) {
  const Level& L = c.fine;
  if (L.det) {
    double* E = static_cast<double*>(L.det);
    klaunch(k_apply_G_elem, (int)div_up(L.nel, 128), 128, 0, c.stream, c.Gp, p, E, (int)L.nel, L.ncr, L.nct,
            c.mesh.pressure);
    DP_LAUNCH_CHECK();
    launch_node_gather<double>(L, E, y, 2, 2, c.stream);
    return;
  }
  DP_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * 2 * L.nnod, c.stream));
  if (L.ncr % 16 == 0) {
    // nel = 2 ncr nct is then a multiple of 32 and every warp is whole
    klaunch(k_apply_G_warp, (int)div_up(L.nel, 128), 128, 0, c.stream, c.Gp, p, y, (int)L.nel, L.ncr, L.nct,
            (int)L.A(), (int)L.B(), c.mesh.pressure);
  } else {
    klaunch(k_apply_G, (int)div_up(L.nel, 128), 128, 0, c.stream, c.Gp, p, y, (int)L.nel, L.ncr, L.nct, (int)L.A(),
            (int)L.B(), c.mesh.pressure);
  }
  DP_LAUNCH_CHECK();
}

void launch_apply_GT(Ctx& c, const double* x, double* p) {
  const Level& L = c.fine;
  if (c.mesh.pressure == 0) DP_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * c.mesh.npres, c.stream));
  klaunch(k_apply_GT, (int)div_up(L.nel, 128), 128, 0, c.stream, c.Gp, x, p, (int)L.nel, L.ncr, L.nct, (int)L.A(),
                                                            (int)L.B(), c.mesh.pressure);
  DP_LAUNCH_CHECK();
}

// ---- deterministic reductions ---------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_dot(const T* __restrict__ a, const T* __restrict__ b, int64_t n,
                                                     double* partial, unsigned int* counter, double* out) {
  grid_dep_wait();
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads)
    s += (double)a[i] * (double)b[i];
  double v[1] = {s};
  double* o[1] = {out};
  grid_finish<1>(v, partial, counter, o);
}

__global__ void __launch_bounds__(kRedThreads) k_sum(const double* __restrict__ a, int64_t n, double* partial,
                                                     unsigned int* counter, double* out) {
  grid_dep_wait();
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads)
    s += a[i];
  double v[1] = {s};
  double* o[1] = {out};
  grid_finish<1>(v, partial, counter, o);
}

// compensated variants (double-double accumulation) for the Schur-complement loop
__global__ void __launch_bounds__(kRedThreads) k_dot_c(const double* __restrict__ a, const double* __restrict__ b,
                                                       int64_t n, double* partial, unsigned int* counter, double* out) {
  grid_dep_wait();
  DD s{0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads)
    dd_add_prod(s, a[i], b[i]);
  DD v[1] = {s};
  double* o[1] = {out};
  grid_finish_dd<1>(v, partial, counter, o);
}

__global__ void __launch_bounds__(kRedThreads) k_sum_c(const double* __restrict__ a, int64_t n, double* partial,
                                                       unsigned int* counter, double* out) {
  grid_dep_wait();
  DD s{0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads)
    dd_add(s, a[i]);
  DD v[1] = {s};
  double* o[1] = {out};
  grid_finish_dd<1>(v, partial, counter, o);
}

static int red_blocks(int64_t n) { return red_grid(n); }

void launch_dot_c(Ctx& c, const double* a, const double* b, int64_t n, int slot) {
  klaunch(k_dot_c, red_blocks(n), kRedThreads, 0, c.stream, a, b, n, c.partial, c.counter, c.scal + slot);
  DP_LAUNCH_CHECK();
}
void launch_sum_c(Ctx& c, const double* a, int64_t n, int slot) {
  klaunch(k_sum_c, red_blocks(n), kRedThreads, 0, c.stream, a, n, c.partial, c.counter, c.scal + slot);
  DP_LAUNCH_CHECK();
}

void launch_dot(Ctx& c, const double* a, const double* b, int64_t n, int slot) {
  klaunch(k_dot<double>, red_blocks(n), kRedThreads, 0, c.stream, a, b, n, c.partial, c.counter, c.scal + slot);
  DP_LAUNCH_CHECK();
}
void launch_dot_f(Ctx& c, const float* a, const float* b, int64_t n, int slot) {
  klaunch(k_dot<float>, red_blocks(n), kRedThreads, 0, c.stream, a, b, n, c.partial, c.counter, c.scal + slot);
  DP_LAUNCH_CHECK();
}
void launch_sum(Ctx& c, const double* a, int64_t n, int slot) {
  klaunch(k_sum, red_blocks(n), kRedThreads, 0, c.stream, a, n, c.partial, c.counter, c.scal + slot);
  DP_LAUNCH_CHECK();
}

// ---- permutations between reference numbering and the lattice -------------
__global__ void k_gather_ref2lat(const int64_t* __restrict__ ref2lat, const double* __restrict__ ref,
                                 double* __restrict__ lat, int64_t nnod, int comps) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  const int64_t l = ref2lat[n];
  for (int c = 0; c < comps; ++c) lat[comps * l + c] = ref[comps * n + c];
}
__global__ void k_scatter_lat2ref(const int64_t* __restrict__ ref2lat, const double* __restrict__ lat,
                                  double* __restrict__ ref, int64_t nnod, int comps) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  const int64_t l = ref2lat[n];
  for (int c = 0; c < comps; ++c) ref[comps * n + c] = lat[comps * l + c];
}
void launch_gather_ref2lat(Ctx& c, const double* ref, double* lat, int comps) {
  const int64_t n = c.fine.nnod;
  klaunch(k_gather_ref2lat, (int)div_up(n, 256), 256, 0, c.stream, c.ref2lat, ref, lat, n, comps);
  DP_LAUNCH_CHECK();
}
void launch_scatter_lat2ref(Ctx& c, const double* lat, double* ref, int comps) {
  const int64_t n = c.fine.nnod;
  klaunch(k_scatter_lat2ref, (int)div_up(n, 256), 256, 0, c.stream, c.ref2lat, lat, ref, n, comps);
  DP_LAUNCH_CHECK();
}

__global__ void k_pc_invert(double* pc, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) pc[i] = 1.0 / pc[i];
}
void launch_pc_invert(Ctx& c, double* pc, int64_t n) {
  klaunch(k_pc_invert, (int)div_up(n, 256), 256, 0, c.stream, pc, n);
  DP_LAUNCH_CHECK();
}

}  // namespace dp
