// Geometric multigrid preconditioner for the velocity block K (free DOFs).
//
// The reference inverts K[ifree, ifree] with a sparse LU once per solve and
// back-substitutes per outer iteration (src/PardisoSolvers.jl:247-256,
// :274-278).  On the device the inner solve is PCG preconditioned by one
// V-cycle of this hierarchy.
//
// Hierarchy.  The split-1 annulus with (ncr, nct) cells is nested in the one
// with (ncr/2, nct/2) cells: every coarse triangle is the union of 4 fine
// triangles and the fine diagonals continue the coarse ones, so coarse P2 is a
// subspace of fine P2 in (theta, r).  Prolongation P interpolates each polar
// component with the coarse P2 basis.  Coarse operators are Galerkin,
// A_c = P^T A P, computed element by element: K_E = sum_{children f}
// P_f^T K_f P_f with the 6x6 local interpolation P_f of each child position,
// followed by the coarse free-slip mask.  This keeps every level in the same
// packed element-by-element form as the fine level.
// Smoother: Chebyshev polynomial in D^-1 A (point Jacobi), bounds from a
// 10-step CG-Lanczos estimate of lambda_max.  Coarsest level: assembled densely,
// inverted once per setup by block Gauss-Jordan (32 pivots per panel) and
// applied as a dense mat-vec.
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "kernels.cuh"
#include "mg.cuh"

namespace dp {

// ---- host-side constant tables ---------------------------------------------
struct ChildTable {
  int dr[2][4], dt[2][4], tf[2][4];  // child cell offset (radial, angular) and type
  double P[2][4][6][6];              // P[coarse type][child][fine local][coarse local]
};
__constant__ ChildTable c_child;

static void p2_values(double xi, double eta, double N[6]) {
  const double t = 1.0 - xi - eta;
  N[0] = t * (2.0 * t - 1.0);
  N[1] = xi * (2.0 * xi - 1.0);
  N[2] = eta * (2.0 * eta - 1.0);
  N[3] = 4.0 * xi * t;
  N[4] = 4.0 * xi * eta;
  N[5] = 4.0 * eta * t;
}

// Local node offsets (radial a, angular b) of the 6 nodes of a triangle of type t
// inside its cell, in units of the P2 lattice of that level.
static const int kLocA[2][6] = {{0, 0, 2, 0, 1, 1}, {0, 2, 2, 1, 2, 1}};
static const int kLocB[2][6] = {{0, 2, 0, 1, 1, 0}, {2, 2, 0, 2, 1, 1}};

// Coarse reference coordinates of a point given in fine-lattice offsets
// (alpha radial, beta angular) from the coarse cell origin (coarse cell = 4x4).
static void coarse_ref(int type, double alpha, double beta, double* xi, double* eta) {
  if (type == 0) {  // v1 (0,0), v2 (0,4), v3 (4,0): point = (4 eta, 4 xi)
    *xi = beta / 4.0;
    *eta = alpha / 4.0;
  } else {          // v1 (0,4), v2 (4,4), v3 (4,0): point = (4 xi + 4 eta, 4 - 4 eta)
    *eta = (4.0 - beta) / 4.0;
    *xi = (alpha + beta - 4.0) / 4.0;
  }
}

// Restriction stencils.  R = P^T is translation invariant on the structured
// lattice: the fine nodes inside the support of a coarse basis function, and
// their weights, depend only on the parity class (a_c mod 2, b_c mod 2) of the
// coarse node.  The table is built once from the prolongation rule on an
// interior node of each class; at the walls the fine nodes outside the annulus
// are simply absent.  This turns the restriction into a gather (no atomics,
// no zeroing pass, deterministic).
constexpr int kRMax = 64;
constexpr int kRTaps = 25;  // largest stencil (vertex class)
struct RestrictTable {
  int n[4];
  signed char da[4][kRMax], db[4][kRMax];
  double w[4][kRMax];
};
__constant__ RestrictTable c_rtab;

static void host_fine_weights(int a, int b, int ncrc, int Ac, int Bc, int cn[6], double w[6]) {
  int IR = a >> 2;
  if (IR >= ncrc) IR = ncrc - 1;
  const int IT = b >> 2;
  const int alpha = a - 4 * IR, beta = b - 4 * IT;
  const int ct = (alpha + beta <= 4) ? 0 : 1;
  double xi, eta;
  coarse_ref(ct, alpha, beta, &xi, &eta);
  p2_values(xi, eta, w);
  for (int k = 0; k < 6; ++k) {
    const int ac = 2 * IR + kLocA[ct][k];
    int bc = 2 * IT + kLocB[ct][k];
    if (bc >= Bc) bc -= Bc;
    cn[k] = ac + Ac * bc;
  }
}

static void upload_restriction_table() {
  RestrictTable R{};
  const int ncrc = 8, nctc = 16, Ac = 2 * ncrc + 1, Bc = 2 * nctc, Af = 4 * ncrc + 1, Bf = 4 * nctc;
  for (int cls = 0; cls < 4; ++cls) {
    const int ac = 8 + (cls & 1), bc = 12 + (cls >> 1);
    const int target = ac + Ac * bc;
    int m = 0;
    for (int da = -4; da <= 4; ++da)
      for (int db = -4; db <= 4; ++db) {
        const int a = 2 * ac + da, b = 2 * bc + db;
        if (a < 0 || a >= Af || b < 0 || b >= Bf) continue;
        int cn[6];
        double w[6];
        host_fine_weights(a, b, ncrc, Ac, Bc, cn, w);
        double wt = 0.0;
        for (int k = 0; k < 6; ++k)
          if (cn[k] == target) wt += w[k];
        if (wt != 0.0) {
          if (m >= kRMax) throw std::runtime_error("restriction table overflow");
          R.da[cls][m] = (signed char)da;
          R.db[cls][m] = (signed char)db;
          R.w[cls][m] = wt;
          ++m;
        }
      }
    if (m > kRTaps) throw std::runtime_error("restriction stencil larger than expected");
    R.n[cls] = m;
  }
  DP_CUDA(cudaMemcpyToSymbol(c_rtab, &R, sizeof(R)));
}

void upload_mg_constants() {
  ChildTable T{};
  // coarse A children: (0,0,A) (0,0,B) (0,1,A) (1,0,A); coarse B: (0,1,B) (1,0,B) (1,1,A) (1,1,B)
  const int dr[2][4] = {{0, 0, 0, 1}, {0, 1, 1, 1}};
  const int dt[2][4] = {{0, 0, 1, 0}, {1, 0, 1, 1}};
  const int tf[2][4] = {{0, 1, 0, 0}, {1, 1, 0, 1}};
  for (int ct = 0; ct < 2; ++ct)
    for (int ch = 0; ch < 4; ++ch) {
      T.dr[ct][ch] = dr[ct][ch];
      T.dt[ct][ch] = dt[ct][ch];
      T.tf[ct][ch] = tf[ct][ch];
      for (int i = 0; i < 6; ++i) {
        const double alpha = 2 * dr[ct][ch] + kLocA[tf[ct][ch]][i];
        const double beta = 2 * dt[ct][ch] + kLocB[tf[ct][ch]][i];
        double xi, eta, N[6];
        coarse_ref(ct, alpha, beta, &xi, &eta);
        p2_values(xi, eta, N);
        for (int k = 0; k < 6; ++k) T.P[ct][ch][i][k] = N[k];
      }
    }
  DP_CUDA(cudaMemcpyToSymbol(c_child, &T, sizeof(T)));
  upload_restriction_table();
}

// ---- Galerkin coarsening: one thread per (coarse element, packed entry) ------
template <typename T>
__global__ void k_galerkin(const T* __restrict__ Kf, T* __restrict__ Kc, int nelc, int ncrc, int nctc, int nelf,
                           int ncrf, int pin) {
  grid_dep_wait();
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (gid >= (int64_t)nelc * kKe) return;
  const int E = (int)(gid % nelc);
  const int pidx = (int)(gid / nelc);
  // decode packed index -> (R, C)
  int C = 0, off = 0;
  while (off + (12 - C) <= pidx) { off += 12 - C; ++C; }
  const int R = C + (pidx - off);
  const int k = R >> 1, alpha = R & 1, l = C >> 1, beta = C & 1;
  const int Q = E >> 1, ct = E & 1;
  const int IR = Q % ncrc, IT = Q / ncrc;
  double acc = 0.0;
#pragma unroll
  for (int ch = 0; ch < 4; ++ch) {
    const int fr = 2 * IR + c_child.dr[ct][ch], ft = 2 * IT + c_child.dt[ct][ch];
    const int ef = 2 * (fr + ncrf * ft) + c_child.tf[ct][ch];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const double pik = c_child.P[ct][ch][i][k];
      if (pik == 0.0) continue;
      double s = 0.0;
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const double pjl = c_child.P[ct][ch][j][l];
        if (pjl == 0.0) continue;
        const int r = 2 * i + alpha, cc = 2 * j + beta;
        const int pi = r >= cc ? packed_index12(r, cc) : packed_index12(cc, r);
        s += pjl * (double)Kf[kidx<T>(pi, ef)];
      }
      acc += pik * s;
    }
  }
  // coarse constraint mask (free slip + optional tangential pin)
  const int a0 = 2 * IR, b0 = 2 * IT, Bc = 2 * nctc;
  const int ak = a0 + kLocA_dev(ct, k), al = a0 + kLocA_dev(ct, l);
  int bk = b0 + kLocB_dev(ct, k), bl = b0 + kLocB_dev(ct, l);
  if (bk >= Bc) bk -= Bc;
  if (bl >= Bc) bl -= Bc;
  const int amax = 2 * ncrc;
  if (dof_fixed(ak, bk, alpha, amax, pin) || dof_fixed(al, bl, beta, amax, pin)) acc = 0.0;
  Kc[kidx<T>(pidx, E)] = (T)acc;
}

// ---- nodal 2x2 diagonal blocks and their inverses ----------------------------
template <typename T>
__global__ void k_diag_blocks(const T* __restrict__ K, double* __restrict__ diag, int nel, int ncr, int A, int B) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int nd[6];
  element_nodes_mg(e, ncr, A, B, nd);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    atomicAdd(&diag[3 * nd[k] + 0], (double)K[kidx<T>(packed_index12(2 * k, 2 * k), e)]);
    atomicAdd(&diag[3 * nd[k] + 1], (double)K[kidx<T>(packed_index12(2 * k + 1, 2 * k), e)]);
    atomicAdd(&diag[3 * nd[k] + 2], (double)K[kidx<T>(packed_index12(2 * k + 1, 2 * k + 1), e)]);
  }
}

// Deterministic form: element e's three block entries at its local node k into
// E[(3k + c) nel + e], summed per node by k_node_gather.
template <typename T>
__global__ void k_diag_blocks_elem(const T* __restrict__ K, double* __restrict__ E, int nel) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    E[(size_t)(3 * k + 0) * nel + e] = (double)K[kidx<T>(packed_index12(2 * k, 2 * k), e)];
    E[(size_t)(3 * k + 1) * nel + e] = (double)K[kidx<T>(packed_index12(2 * k + 1, 2 * k), e)];
    E[(size_t)(3 * k + 2) * nel + e] = (double)K[kidx<T>(packed_index12(2 * k + 1, 2 * k + 1), e)];
  }
}

// Inverse of the nodal block (block = 1) or of its diagonal (block = 0);
// constrained DOFs get zero rows/columns so the smoother never touches them.
template <typename T>
__global__ void k_block_invert(const double* __restrict__ diag, T* __restrict__ dinv, int64_t nnod, int A, int pin,
                               int block) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  const int a = (int)(n % A), b = (int)(n / A);
  const bool f0 = dof_fixed(a, b, 0, A - 1, pin), f1 = dof_fixed(a, b, 1, A - 1, pin);
  const double d00 = diag[3 * n], d11 = diag[3 * n + 2];
  double d01 = block ? diag[3 * n + 1] : 0.0;
  double i00 = 0.0, i01 = 0.0, i11 = 0.0;
  if (f0 || f1 || d01 == 0.0) {
    i00 = (!f0 && d00 > 0.0) ? 1.0 / d00 : 0.0;
    i11 = (!f1 && d11 > 0.0) ? 1.0 / d11 : 0.0;
  } else {
    const double det = d00 * d11 - d01 * d01;
    if (det > 0.0) {
      i00 = d11 / det;
      i01 = -d01 / det;
      i11 = d00 / det;
    } else {
      i00 = d00 > 0.0 ? 1.0 / d00 : 0.0;
      i11 = d11 > 0.0 ? 1.0 / d11 : 0.0;
    }
  }
  dinv[3 * n] = (T)i00;
  dinv[3 * n + 1] = (T)i01;
  dinv[3 * n + 2] = (T)i11;
}

template <typename T>
__device__ inline void bj_apply(const T* __restrict__ dinv, int64_t n, double r0, double r1, double& z0, double& z1) {
  const double a = (double)dinv[3 * n], b = (double)dinv[3 * n + 1], c = (double)dinv[3 * n + 2];
  z0 = a * r0 + b * r1;
  z1 = b * r0 + c * r1;
}

// ---- transfers ---------------------------------------------------------------
// Fine node (a, b) -> containing coarse element and the 6 coarse P2 weights.
__device__ inline void fine_node_weights(int a, int b, int ncrc, int Ac, int Bc, int cn[6], double w[6]) {
  int IR = a >> 2;
  if (IR >= ncrc) IR = ncrc - 1;
  const int IT = b >> 2;
  const int alpha = a - 4 * IR, beta = b - 4 * IT;
  const int ct = (alpha + beta <= 4) ? 0 : 1;
  double xi, eta;
  if (ct == 0) { xi = beta * 0.25; eta = alpha * 0.25; }
  else { eta = (4 - beta) * 0.25; xi = (alpha + beta - 4) * 0.25; }
  const double t = 1.0 - xi - eta;
  w[0] = t * (2.0 * t - 1.0);
  w[1] = xi * (2.0 * xi - 1.0);
  w[2] = eta * (2.0 * eta - 1.0);
  w[3] = 4.0 * xi * t;
  w[4] = 4.0 * xi * eta;
  w[5] = 4.0 * eta * t;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const int ac = 2 * IR + kLocA_dev(ct, k);
    int bc = 2 * IT + kLocB_dev(ct, k);
    if (bc >= Bc) bc -= Bc;
    cn[k] = ac + Ac * bc;
  }
}

// xf += P xc (per fine node, gather); also sets rf = bf (the fine level's
// residual buffer, from which the next apply subtracts A xf)
template <typename T>
__global__ void k_prolong_add(const T* __restrict__ xc, T* __restrict__ xf, const T* __restrict__ bf,
                              T* __restrict__ rf, int Af, int Bf, int ncrc, int Ac, int Bc, int pin) {
  grid_dep_wait();
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= Af * Bf) return;
  const int b = n / Af, a = n - b * Af;
  int cn[6];
  double w[6];
  fine_node_weights(a, b, ncrc, Ac, Bc, cn, w);
  // the 6 nodes of the containing coarse element are always valid: gather them
  // all unconditionally (zero weights included) so the loads issue together
  typedef typename V2<T>::T X2;
  const X2* xc2 = reinterpret_cast<const X2*>(xc);
  X2 v[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) v[k] = xc2[cn[k]];
  X2 xv = reinterpret_cast<const X2*>(xf)[n];
  const X2 bv = reinterpret_cast<const X2*>(bf)[n];
  T s0 = (T)0, s1 = (T)0;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    s0 += (T)w[k] * v[k].x;
    s1 += (T)w[k] * v[k].y;
  }
  if (!dof_fixed(a, b, 0, Af - 1, pin)) xv.x += s0;
  if (!dof_fixed(a, b, 1, Af - 1, pin)) xv.y += s1;
  reinterpret_cast<X2*>(xf)[n] = xv;
  reinterpret_cast<X2*>(rf)[n] = bv;
}

// bc = P^T (r - t) per coarse node (t = null: P^T r; gather over the class
// stencil); constrained DOFs of either level are excluded.  blockIdx.y is the parity class, so the
// stencil reads are uniform across a warp (constant-cache broadcast), and the
// stencil loop is unrolled with its loads predicated rather than branched, so
// a thread keeps several gathers in flight.
// first != 0 also takes the coarse level's first Chebyshev step from x = 0
// (the work of k_cheb_first): rc = bc, dc = xc = coef[0] D^-1 bc, and tc = 0
// when tc is given (the cluster tail's levels accumulate into t).
template <typename T, int LPN>
__global__ void __launch_bounds__(256) k_restrict_g(const T* __restrict__ r, const T* __restrict__ t, T* __restrict__ bc,
                                                    int Af, int Bf, int Ac, int Bc, int pin, int first,
                                                    const T* __restrict__ dinv_c, T* __restrict__ xc, T* __restrict__ rc,
                                                    T* __restrict__ dc, T* __restrict__ tc,
                                                    const double* __restrict__ coef_c) {
  grid_dep_wait();
  const int cls = blockIdx.y;
  const int pa = cls & 1, pb = cls >> 1;
  const int nA = (Ac - pa + 1) >> 1;  // coarse a = pa, pa + 2, ... <= Ac - 1
  // LPN lanes per coarse node, each gathering every LPN-th tap (LPN = 4 on
  // small levels: <= 7 taps per lane, all in flight; LPN = 1 on large levels,
  // where the grid alone keeps the memory system busy), combined by shuffles
  const int gidx = blockIdx.x * blockDim.x + threadIdx.x;
  const int idx = gidx / LPN, sub = gidx % LPN;
  const bool live = idx < nA * (Bc >> 1);
  const int ac = live ? 2 * (idx % nA) + pa : pa, bcn = live ? 2 * (idx / nA) + pb : pb;
  typedef typename V2<T>::T X2;
  const X2* r2 = reinterpret_cast<const X2*>(r);
  const X2* t2 = reinterpret_cast<const X2*>(t);
  const int m = live ? c_rtab.n[cls] : 0;
  double s0 = 0.0, s1 = 0.0;
#pragma unroll 8
  for (int j = sub; j < m; j += LPN) {
    const int jj = j;
    const int a = 2 * ac + c_rtab.da[cls][jj];
    int b = 2 * bcn + c_rtab.db[cls][jj];
    b += (b < 0) ? Bf : 0;
    b -= (b >= Bf) ? Bf : 0;
    const bool in = a >= 0 && a < Af;
    const int f = in ? a + Af * b : 0;
    const X2 rv = r2[f];
    X2 tv;
    if (t2) tv = t2[f];
    else { tv.x = (T)0; tv.y = (T)0; }
    const double w = c_rtab.w[cls][jj];
    const double w0 = (in && !dof_fixed(a, b, 0, Af - 1, pin)) ? w : 0.0;
    const double w1 = (in && !dof_fixed(a, b, 1, Af - 1, pin)) ? w : 0.0;
    s0 += w0 * ((double)rv.x - (double)tv.x);
    s1 += w1 * ((double)rv.y - (double)tv.y);
  }
  // every lane of the warp takes part in the shuffles (dead lanes add zeros)
#pragma unroll
  for (int o = 1; o < LPN; o <<= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  if (!live || sub != 0) return;
  const int n = ac + Ac * bcn;
  const double b0 = dof_fixed(ac, bcn, 0, Ac - 1, pin) ? 0.0 : s0;
  const double b1 = dof_fixed(ac, bcn, 1, Ac - 1, pin) ? 0.0 : s1;
  bc[2 * n] = (T)b0;
  bc[2 * n + 1] = (T)b1;
  if (first) {
    const double it = coef_c[0];
    double z0, z1;
    bj_apply<T>(dinv_c, n, b0, b1, z0, z1);
    if (tc) { tc[2 * n] = (T)0; tc[2 * n + 1] = (T)0; }
    rc[2 * n] = (T)b0; rc[2 * n + 1] = (T)b1;
    dc[2 * n] = (T)(it * z0); dc[2 * n + 1] = (T)(it * z1);
    xc[2 * n] = (T)(it * z0); xc[2 * n + 1] = (T)(it * z1);
  }
}

// Tiled form of the same restriction for the large levels.  One CTA = 16 x 16
// coarse nodes; the fine values r - t of the CTA's stencil footprint (a 39 x 39
// patch of fine nodes, constrained fine DOFs zeroed) are read from global
// memory once into shared memory, and each coarse node gathers its class
// stencil from there (the gather form reads every fine value ~4 times through
// L2).  Warps are class-uniform (64 coarse nodes of each parity class), so the
// stencil table reads are constant-cache broadcasts.  Arithmetic in the level's
// precision (the stencil weights are dyadic fractions, exact in FP32).
constexpr int kRTile = 16;
constexpr int kRPatch = 2 * (kRTile - 1) + 1 + 8;   // 39: stencil offsets reach 4 fine nodes each way
template <typename T>
__global__ void __launch_bounds__(256) k_restrict_tile(const T* __restrict__ r, const T* __restrict__ t,
                                                       T* __restrict__ bc, int Af, int Bf, int Ac, int Bc, int pin,
                                                       int first, const T* __restrict__ dinv_c, T* __restrict__ xc,
                                                       T* __restrict__ rc, T* __restrict__ dc, T* __restrict__ tc,
                                                       const double* __restrict__ coef_c) {
  grid_dep_wait();
  typedef typename V2<T>::T X2;
  __shared__ X2 sp[kRPatch][kRPatch + 1];    // [b][a]
  const int ac0 = blockIdx.x * kRTile, bc0 = blockIdx.y * kRTile;
  const int fa0 = 2 * ac0 - 4, fb0 = 2 * bc0 - 4;
  const X2* r2 = reinterpret_cast<const X2*>(r);
  const X2* t2 = reinterpret_cast<const X2*>(t);
  for (int k = threadIdx.x; k < kRPatch * kRPatch; k += blockDim.x) {
    const int la = k % kRPatch, lb = k / kRPatch;
    const int a = fa0 + la;
    int b = fb0 + lb;
    b += (b < 0) ? Bf : 0;                   // the patch reaches at most 4 nodes past either end
    b -= (b >= Bf) ? Bf : 0;
    X2 v;
    v.x = (T)0;
    v.y = (T)0;
    if (a >= 0 && a < Af) {
      const int64_t f = a + (int64_t)Af * b;
      X2 rv = r2[f];
      if (t2) {
        const X2 tv = t2[f];
        rv.x -= tv.x;
        rv.y -= tv.y;
      }
      if (!dof_fixed(a, b, 0, Af - 1, pin)) v.x = rv.x;
      if (!dof_fixed(a, b, 1, Af - 1, pin)) v.y = rv.y;
    }
    sp[lb][la] = v;
  }
  __syncthreads();
  const int cls = threadIdx.x >> 6, loc = threadIdx.x & 63;
  const int pa = cls & 1, pb = cls >> 1;
  const int ac = ac0 + 2 * (loc & 7) + pa, bcn = bc0 + 2 * (loc >> 3) + pb;
  if (ac >= Ac || bcn >= Bc) return;
  const int m = c_rtab.n[cls];
  T s0 = (T)0, s1 = (T)0;
  for (int j = 0; j < m; ++j) {
    const int la = 2 * (ac - ac0) + 4 + c_rtab.da[cls][j];
    const int lb = 2 * (bcn - bc0) + 4 + c_rtab.db[cls][j];
    const X2 v = sp[lb][la];
    const T w = (T)c_rtab.w[cls][j];
    s0 += w * v.x;
    s1 += w * v.y;
  }
  const int n = ac + Ac * bcn;
  const T b0 = dof_fixed(ac, bcn, 0, Ac - 1, pin) ? (T)0 : s0;
  const T b1 = dof_fixed(ac, bcn, 1, Ac - 1, pin) ? (T)0 : s1;
  X2 bv;
  bv.x = b0;
  bv.y = b1;
  reinterpret_cast<X2*>(bc)[n] = bv;
  if (first) {
    const T it = (T)coef_c[0];
    T z0, z1;
    const T a = dinv_c[3 * (int64_t)n], bb = dinv_c[3 * (int64_t)n + 1], c = dinv_c[3 * (int64_t)n + 2];
    z0 = a * b0 + bb * b1;
    z1 = bb * b0 + c * b1;
    X2 dv;
    dv.x = it * z0;
    dv.y = it * z1;
    if (tc) {
      X2 zero;
      zero.x = (T)0;
      zero.y = (T)0;
      reinterpret_cast<X2*>(tc)[n] = zero;
    }
    reinterpret_cast<X2*>(rc)[n] = bv;
    reinterpret_cast<X2*>(dc)[n] = dv;
    reinterpret_cast<X2*>(xc)[n] = dv;
  }
}

// ---- Chebyshev smoother vector steps (per node, coefficients read from device) --
// The residual r lives in one buffer that the applies between the steps update
// in place (r -= A d, launch_apply_K_sub), so a step reads r, d, x and the
// block inverse and writes only d and x: no accumulator is zeroed, re-read or
// subtracted (52 instead of 76 bytes per FP32 node).
// The three kernels compute in the precision of the level (FP32 on the FP32
// hierarchy) and move each node's pair of components with one 8/16-byte
// access, all loads issued before the arithmetic.
template <typename T>
__device__ __forceinline__ void bj_apply_t(const T* __restrict__ dinv, int64_t n, T r0, T r1, T& z0, T& z1) {
  const T a = dinv[3 * n], b = dinv[3 * n + 1], c = dinv[3 * n + 2];
  z0 = a * r0 + b * r1;
  z1 = b * r0 + c * r1;
}

// first step from x = 0: r = b, d = (1/theta) D^-1 b, x = d
template <typename T>
__global__ void k_cheb_first(const T* __restrict__ b, const T* __restrict__ dinv, T* __restrict__ x,
                             T* __restrict__ r, T* __restrict__ d, const double* __restrict__ coef, int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  typedef typename V2<T>::T X2;
  const X2 bv = reinterpret_cast<const X2*>(b)[n];
  const T it = (T)coef[0];
  T z0, z1;
  bj_apply_t<T>(dinv, n, bv.x, bv.y, z0, z1);
  X2 dv;
  dv.x = it * z0; dv.y = it * z1;
  reinterpret_cast<X2*>(r)[n] = bv;
  reinterpret_cast<X2*>(d)[n] = dv;
  reinterpret_cast<X2*>(x)[n] = dv;
}
// first step from a given x (r = b - Ax on entry): d = (1/theta) D^-1 r, x += d
template <typename T>
__global__ void k_cheb_first_x(const T* __restrict__ r, const T* __restrict__ dinv, T* __restrict__ x,
                               T* __restrict__ d, const double* __restrict__ coef, int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  typedef typename V2<T>::T X2;
  const X2 rv = reinterpret_cast<const X2*>(r)[n];
  const X2 xv = reinterpret_cast<const X2*>(x)[n];
  const T it = (T)coef[0];
  X2 dv;
  T z0, z1;
  bj_apply_t<T>(dinv, n, rv.x, rv.y, z0, z1);
  dv.x = it * z0; dv.y = it * z1;
  reinterpret_cast<X2*>(d)[n] = dv;
  X2 xn;
  xn.x = xv.x + dv.x; xn.y = xv.y + dv.y;
  reinterpret_cast<X2*>(x)[n] = xn;
}
// d = c1 d + c2 D^-1 r; x += d  (c1, c2 = coef[0], coef[1]; r already holds r - A d_prev)
template <typename T>
__global__ void k_cheb_step(const T* __restrict__ r, const T* __restrict__ dinv, T* __restrict__ x,
                            T* __restrict__ d, const double* __restrict__ coef, int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  typedef typename V2<T>::T X2;
  const X2 rv = reinterpret_cast<const X2*>(r)[n];
  const X2 dv = reinterpret_cast<const X2*>(d)[n];
  const X2 xv = reinterpret_cast<const X2*>(x)[n];
  const T c1 = (T)coef[0], c2 = (T)coef[1];
  X2 dn, xn;
  T z0, z1;
  bj_apply_t<T>(dinv, n, rv.x, rv.y, z0, z1);
  dn.x = c1 * dv.x + c2 * z0; dn.y = c1 * dv.y + c2 * z1;
  xn.x = xv.x + dn.x; xn.y = xv.y + dn.y;
  reinterpret_cast<X2*>(d)[n] = dn;
  reinterpret_cast<X2*>(x)[n] = xn;
}
// z = D^-1 r (nodal blocks)
template <typename T>
__global__ void k_bj(const T* __restrict__ dinv, const T* __restrict__ r, T* __restrict__ z, int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  double z0, z1;
  bj_apply<T>(dinv, n, (double)r[2 * n], (double)r[2 * n + 1], z0, z1);
  z[2 * n] = (T)z0;
  z[2 * n + 1] = (T)z1;
}

// ---- coarse dense solve --------------------------------------------------------
template <typename T>
__global__ void k_dense_assemble(const T* __restrict__ K, double* __restrict__ D, int nel, int ncr, int A, int B, int n) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int nd[6];
  element_nodes_mg(e, ncr, A, B, nd);
  for (int C = 0; C < 12; ++C)
    for (int R = C; R < 12; ++R) {
      const double v = (double)K[kidx<T>(packed_index12(R, C), e)];
      const int gr = 2 * nd[R >> 1] + (R & 1), gc = 2 * nd[C >> 1] + (C & 1);
      atomicAdd(&D[(size_t)gr * n + gc], v);
      if (R != C) atomicAdd(&D[(size_t)gc * n + gr], v);
    }
}

// Deterministic form: one CTA walks the elements in order, its threads taking
// the 78 packed entries of one element at a time.  The entries of one element
// land on distinct matrix positions (its 12 DOFs are distinct), so the threads
// never collide, and every position receives its contributions in element
// order.  The coarsest level has a few hundred elements.
template <typename T>
__global__ void __launch_bounds__(128) k_dense_assemble_seq(const T* __restrict__ K, double* __restrict__ D, int nel,
                                                            int ncr, int A, int B, int n) {
  grid_dep_wait();
  const int i = threadIdx.x;
  int R = 0, C = 0;
  if (i < kKe) {   // packed entry i -> (R, C), R >= C, column-major lower triangle
    int c0 = 0, rem = i;
    while (rem >= 12 - c0) { rem -= 12 - c0; ++c0; }
    C = c0;
    R = c0 + rem;
  }
  for (int e = 0; e < nel; ++e) {
    if (i < kKe) {
      int nd[6];
      element_nodes_mg(e, ncr, A, B, nd);
      const double v = (double)K[kidx<T>(packed_index12(R, C), e)];
      const int gr = 2 * nd[R >> 1] + (R & 1), gc = 2 * nd[C >> 1] + (C & 1);
      D[(size_t)gr * n + gc] += v;
      if (R != C) D[(size_t)gc * n + gr] += v;
    }
    __syncthreads();
  }
}

// Identity on the diagonal of fixed (all-zero) rows, so the matrix stays SPD.
__global__ void k_dense_fix_diag(double* __restrict__ D, int n) {
  grid_dep_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && D[(size_t)i * n + i] == 0.0) D[(size_t)i * n + i] = 1.0;
}

// Block Gauss-Jordan inversion of the SPD coarsest matrix, one panel of up to
// kGJPanel pivots K = [k0, k0 + b) at a time (no pivoting: the pivot blocks of an
// SPD matrix are SPD).  With W = A_KK^-1 and T = A_{:,K} W, the panel step maps A
// (old) to B (new):
//   B_KK = W,   B_Kj = W A_Kj,   B_iK = -T_iK,   B_ij = A_ij - T_iK A_Kj
// (i, j outside K).  After all panels B = A^-1.  Three launches per panel: the
// pivot-block inverse (one CTA, shared memory), T (one thread per (row, pivot))
// and the update (one thread per entry, coalesced along rows, ping-pong buffers).
constexpr int kGJPanel = 32;

__global__ void __launch_bounds__(kGJPanel * kGJPanel) k_gj_panel_inverse(const double* __restrict__ A,
                                                                          double* __restrict__ W, int n, int k0,
                                                                          int b) {
  grid_dep_wait();
  __shared__ double s[kGJPanel][kGJPanel + 1];
  const int r = threadIdx.y, c = threadIdx.x;
  s[r][c] = (r < b && c < b) ? A[(size_t)(k0 + r) * n + k0 + c] : (r == c ? 1.0 : 0.0);
  __syncthreads();
  for (int k = 0; k < b; ++k) {
    const double ip = 1.0 / s[k][k];
    const double akc = s[k][c], ark = s[r][k];
    __syncthreads();                       // every read of pivot row/column before any write
    double v;
    if (r == k) v = (c == k) ? ip : akc * ip;
    else if (c == k) v = -ark * ip;
    else v = s[r][c] - ark * akc * ip;
    s[r][c] = v;
    __syncthreads();
  }
  W[r * kGJPanel + c] = s[r][c];
}

// T[i][m] = sum_l A[i][k0 + l] W[l][m]  (i < n, m < b; row stride kGJPanel)
__global__ void k_gj_panel_cols(const double* __restrict__ A, const double* __restrict__ W, double* __restrict__ T,
                                int n, int k0, int b) {
  grid_dep_wait();
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * kGJPanel) return;
  const int i = (int)(idx / kGJPanel), m = (int)(idx % kGJPanel);
  double t = 0.0;
  if (m < b)
    for (int l = 0; l < b; ++l) t += A[(size_t)i * n + k0 + l] * W[l * kGJPanel + m];
  T[idx] = t;
}

__global__ void k_gj_panel_update(const double* __restrict__ A, double* __restrict__ B, const double* __restrict__ W,
                                  const double* __restrict__ T, int n, int k0, int b) {
  grid_dep_wait();
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx % n);
  const bool ik = i >= k0 && i < k0 + b, jk = j >= k0 && j < k0 + b;
  double v;
  if (ik && jk) {
    v = W[(i - k0) * kGJPanel + (j - k0)];
  } else if (ik) {
    v = 0.0;
    for (int m = 0; m < b; ++m) v += W[(i - k0) * kGJPanel + m] * A[(size_t)(k0 + m) * n + j];
  } else if (jk) {
    v = -T[(size_t)i * kGJPanel + (j - k0)];
  } else {
    v = A[idx];
    for (int m = 0; m < b; ++m) v -= T[(size_t)i * kGJPanel + m] * A[(size_t)(k0 + m) * n + j];
  }
  B[idx] = v;
}

// A = (A + A^T) / 2 in place (one thread per pair i < j): the inverse of the SPD
// coarse matrix is symmetric in exact arithmetic; the elimination's rounding is
// not, and a symmetric coarse solve keeps the V-cycle a symmetric preconditioner.
__global__ void k_symmetrize(double* __restrict__ A, int n) {
  grid_dep_wait();
  const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx % n);
  if (i >= j) return;
  const double v = 0.5 * (A[(size_t)i * n + j] + A[(size_t)j * n + i]);
  A[(size_t)i * n + j] = v;
  A[(size_t)j * n + i] = v;
}

// x = Inv b, one CTA per row: each thread reads a few entries of the row (all
// loads in flight at once), then a block reduction.
template <typename T>
__global__ void __launch_bounds__(128) k_dense_apply(const double* __restrict__ Inv, const T* __restrict__ b,
                                                     T* __restrict__ x, int n) {
  grid_dep_wait();
  const int row = blockIdx.x;
  const double* a = Inv + (size_t)row * n;
  double s = 0.0;
#pragma unroll 4
  for (int j = threadIdx.x; j < n; j += 128) s += a[j] * (double)b[j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double part[4];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) x[row] = (T)(part[0] + part[1] + part[2] + part[3]);
}

// ---- host side ---------------------------------------------------------------
static int tpb(int64_t n) { return (int)div_up(n, 256); }

template <typename T>
static T* level_K(MGLevel& L);
template <>
double* level_K<double>(MGLevel& L) { return L.K64; }
template <>
float* level_K<float>(MGLevel& L) { return L.K32; }
template <typename T>
static T* level_dinv(MGLevel& L);
template <>
double* level_dinv<double>(MGLevel& L) { return L.dinv64; }
template <>
float* level_dinv<float>(MGLevel& L) { return L.dinv32; }

void mg_free(Ctx& c) {
  ++c.alloc_gen;
  for (size_t l = 0; l < c.mg.size(); ++l) {
    MGLevel& L = c.mg[l];
    if (l > 0) { cudaFree(L.K64); cudaFree(L.K32); }
    cudaFree(L.dinv64); cudaFree(L.dinv32); cudaFree(L.cheb);
    cudaFree(L.x); cudaFree(L.b); cudaFree(L.r); cudaFree(L.d); cudaFree(L.t);
  }
  c.mg.clear();
  cudaFree(c.coarse_inv);
  c.coarse_inv = nullptr;
  c.coarse_n = 0;
  c.mg_prec = -1;
}

// Largest eigenvalue of a symmetric tridiagonal matrix (Sturm bisection).
static double tridiag_lmax(const std::vector<double>& a, const std::vector<double>& b) {
  const int m = (int)a.size();
  double lo = 0.0, hi = 0.0;
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i < m - 1 ? std::fabs(b[i]) : 0.0);
    hi = std::max(hi, a[i] + r);
    lo = std::min(lo, a[i] - r);
  }
  auto count_below = [&](double x) {
    int cnt = 0;
    double d = 1.0;
    for (int i = 0; i < m; ++i) {
      d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0.0);
      if (d == 0.0) d = 1e-300;
      if (d < 0) ++cnt;
    }
    return cnt;
  };
  for (int it = 0; it < 100; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= m) hi = mid; else lo = mid;
  }
  return hi;
}

template <typename T>
static void apply_level(Ctx& c, MGLevel& L, const T* x, T* y) {
  launch_apply_K<T, T>(L.g, level_K<T>(L), x, y, c.stream);
}

template <typename T>
static void dot_level(Ctx& c, const T* a, const T* b, int64_t n, int slot);
template <>
void dot_level<double>(Ctx& c, const double* a, const double* b, int64_t n, int slot) { launch_dot(c, a, b, n, slot); }
template <>
void dot_level<float>(Ctx& c, const float* a, const float* b, int64_t n, int slot) { launch_dot_f(c, a, b, n, slot); }

template <typename T>
__global__ void k_fill_pattern(T* v, int64_t n, int A, int pin) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  // deterministic pseudo-random start vector, zero on fixed DOFs
  uint64_t z = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  const int64_t node = i >> 1;
  const int a = (int)(node % A), b = (int)(node / A);
  const bool fixed = dof_fixed(a, b, (int)(i & 1), A - 1, pin);
  v[i] = fixed ? (T)0 : (T)u;
}

template <typename T>
__global__ void k_pcg_vec(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p, const T* __restrict__ Ap,
                          const T* __restrict__ dinv, T* __restrict__ z, double alpha, int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  double rr[2];
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    x[2 * n + c] += (T)(alpha * (double)p[2 * n + c]);
    rr[c] = (double)r[2 * n + c] - alpha * (double)Ap[2 * n + c];
    r[2 * n + c] = (T)rr[c];
  }
  double z0, z1;
  bj_apply<T>(dinv, n, rr[0], rr[1], z0, z1);
  z[2 * n] = (T)z0;
  z[2 * n + 1] = (T)z1;
}
template <typename T>
__global__ void k_xpby(const T* __restrict__ z, T* __restrict__ p, double beta, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = z[i] + (T)(beta * (double)p[i]);
}

// lambda_max(D^-1 A) from 10 steps of Jacobi-PCG (Lanczos coefficients).
template <typename T>
static double estimate_lmax(Ctx& c, MGLevel& L) {
  const int64_t n = 2 * L.g.nnod;
  T* x = (T*)L.x; T* r = (T*)L.r; T* p = (T*)L.d; T* z = (T*)L.b; T* Ap = (T*)L.t;
  const T* dinv = level_dinv<T>(L);
  DP_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, c.stream));
  klaunch(k_fill_pattern<T>, tpb(n), 256, 0, c.stream, r, n, (int)L.g.A(), L.g.pin);
  klaunch(k_bj<T>, tpb(L.g.nnod), 256, 0, c.stream, dinv, r, z, L.g.nnod);
  DP_CUDA(cudaMemcpyAsync(p, z, sizeof(T) * n, cudaMemcpyDeviceToDevice, c.stream));
  dot_level<T>(c, r, z, n, 20);
  DP_CUDA(cudaMemcpyAsync(c.h_scal + 20, c.scal + 20, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  DP_CUDA(cudaStreamSynchronize(c.stream));
  double rz = c.h_scal[20];
  std::vector<double> alphas, betas;
  const int kSteps = 10;
  for (int k = 0; k < kSteps && rz > 0.0; ++k) {
    apply_level<T>(c, L, p, Ap);
    dot_level<T>(c, p, Ap, n, 21);
    DP_CUDA(cudaMemcpyAsync(c.h_scal + 21, c.scal + 21, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    const double pAp = c.h_scal[21];
    if (!(pAp > 0.0)) break;
    const double alpha = rz / pAp;
    klaunch(k_pcg_vec<T>, tpb(L.g.nnod), 256, 0, c.stream, x, r, p, Ap, dinv, z, alpha, L.g.nnod);
    dot_level<T>(c, r, z, n, 20);
    DP_CUDA(cudaMemcpyAsync(c.h_scal + 20, c.scal + 20, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    const double rz_new = c.h_scal[20];
    const double beta = rz_new / rz;
    alphas.push_back(alpha);
    betas.push_back(beta);
    rz = rz_new;
    if (!(rz > 0.0)) break;
    klaunch(k_xpby<T>, tpb(n), 256, 0, c.stream, z, p, beta, n);
  }
  DP_LAUNCH_CHECK();
  const int m = (int)alphas.size();
  if (m == 0) return 2.0;
  std::vector<double> a(m), b(std::max(m - 1, 0));
  for (int j = 0; j < m; ++j) {
    a[j] = 1.0 / alphas[j] + (j > 0 ? betas[j - 1] / alphas[j - 1] : 0.0);
    if (j < m - 1) b[j] = std::sqrt(betas[j]) / alphas[j];
  }
  return tridiag_lmax(a, b);
}

template <typename T>
static void setup_level_vectors(MGLevel& L) {
  const size_t bytes = sizeof(T) * 2 * L.g.nnod;
  DP_CUDA(cudaMalloc(&L.x, bytes));
  DP_CUDA(cudaMalloc(&L.b, bytes));
  DP_CUDA(cudaMalloc(&L.r, bytes));
  DP_CUDA(cudaMalloc(&L.d, bytes));
  DP_CUDA(cudaMalloc(&L.t, bytes));
}

template <typename T>
static void mg_setup_t(Ctx& c, const MGOptions& o) {
  const int prec = std::is_same<T, float>::value ? 1 : 0;
  // level geometry (reuse if unchanged)
  if (c.mg.empty() || c.mg_prec != prec || c.mg_coarse_max != o.coarse_max) {
    mg_free(c);
    MGLevel L0;
    L0.g = c.fine;
    c.mg.push_back(L0);
    while (true) {
      const Level& g = c.mg.back().g;
      if (g.ncr % 2 || g.nct % 2 || g.nct / 2 < 4) break;
      if ((int)c.mg.size() >= o.max_levels) break;
      Level h;
      h.ncr = g.ncr / 2;
      h.nct = g.nct / 2;
      h.nel = 2 * (int64_t)h.ncr * h.nct;
      h.nnod = h.A() * h.B();
      h.pin = g.pin;
      if (2 * g.nnod <= o.coarse_max) break;
      MGLevel Lh;
      Lh.g = h;
      c.mg.push_back(Lh);
    }
    for (size_t l = 0; l < c.mg.size(); ++l) {
      MGLevel& L = c.mg[l];
      if (l > 0) {
        DP_CUDA(cudaMalloc(prec ? (void**)&L.K32 : (void**)&L.K64, sizeof(T) * kstore<T>(L.g.nel)));
      }
      DP_CUDA(cudaMalloc(prec ? (void**)&L.dinv32 : (void**)&L.dinv64, sizeof(T) * 3 * L.g.nnod));
      DP_CUDA(cudaMalloc(&L.cheb, sizeof(double) * 2 * (kMaxCheb + 1)));
      setup_level_vectors<T>(L);
    }
    c.coarse_n = 2 * c.mg.back().g.nnod;
    if (c.coarse_n <= o.coarse_max) {
      DP_CUDA(cudaMalloc(&c.coarse_inv, sizeof(double) * c.coarse_n * c.coarse_n * 2));
    } else {
      c.coarse_n = 0;
    }
    c.mg_prec = prec;
    c.mg_coarse_max = o.coarse_max;
  }
  // fine operator pointer, apply tiles
  if (prec) c.mg[0].K32 = c.K32; else c.mg[0].K64 = c.K64;
  for (MGLevel& L : c.mg) {
    L.g.warps = o.apply_warps;
    L.g.warps_t = o.apply_warps_t;
    L.g.det = c.fine.det;   // one scratch (sized for the fine level) serves every level in turn
    L.g.mfD64 = L.g.mfT64 = nullptr;
    L.g.mfD32 = L.g.mfT32 = nullptr;
  }
  // the fine level applies matrix-free when the fine context level does
  c.mg[0].g.mfD64 = c.fine.mfD64;
  c.mg[0].g.mfT64 = c.fine.mfT64;
  c.mg[0].g.mfD32 = c.fine.mfD32;
  c.mg[0].g.mfT32 = c.fine.mfT32;
  // Galerkin coarse operators
  for (size_t l = 1; l < c.mg.size(); ++l) {
    MGLevel& Lf = c.mg[l - 1];
    MGLevel& Lc = c.mg[l];
    const int64_t nthreads = Lc.g.nel * kKe;
    klaunch(k_galerkin<T>, (int)div_up(nthreads, 128), 128, 0, c.stream, level_K<T>(Lf), level_K<T>(Lc), (int)Lc.g.nel,
                                                                      Lc.g.ncr, Lc.g.nct, (int)Lf.g.nel, Lf.g.ncr,
                                                                      Lc.g.pin);
    DP_LAUNCH_CHECK();
  }
  // nodal diagonal blocks, eigenvalue estimates and Chebyshev coefficients
  double* diag = nullptr;
  DP_CUDA(cudaMalloc(&diag, sizeof(double) * 3 * c.mg[0].g.nnod));
  const int deg = std::max(1, std::min(o.cheb_degree, kMaxCheb));
  const int deg_coarse = o.cheb_degree_coarse > 0 ? std::max(1, std::min(o.cheb_degree_coarse, kMaxCheb)) : deg;
  for (size_t l = 0; l < c.mg.size(); ++l) {
    MGLevel& L = c.mg[l];
    L.degree = l == 0 ? deg : deg_coarse;
    if (L.g.det) {
      double* E = static_cast<double*>(L.g.det);
      klaunch(k_diag_blocks_elem<T>, (int)div_up(L.g.nel, 128), 128, 0, c.stream, level_K<T>(L), E, (int)L.g.nel);
      DP_LAUNCH_CHECK();
      launch_node_gather<double>(L.g, E, diag, 3, 2, c.stream);
    } else {
      DP_CUDA(cudaMemsetAsync(diag, 0, sizeof(double) * 3 * L.g.nnod, c.stream));
      klaunch(k_diag_blocks<T>, (int)div_up(L.g.nel, 128), 128, 0, c.stream, level_K<T>(L), diag, (int)L.g.nel,
              L.g.ncr, (int)L.g.A(), (int)L.g.B());
    }
    klaunch(k_block_invert<T>, tpb(L.g.nnod), 256, 0, c.stream, diag, level_dinv<T>(L), L.g.nnod, (int)L.g.A(), L.g.pin,
                                                            o.block_jacobi);
    DP_LAUNCH_CHECK();
    const bool is_coarsest_direct = (l + 1 == c.mg.size()) && c.coarse_n > 0;
    L.lmax = is_coarsest_direct ? 0.0 : estimate_lmax<T>(c, L);
    // Chebyshev recurrence coefficients on [lo, hi] * lmax (three-term form)
    double coef[2 * (kMaxCheb + 1)] = {0.0};
    if (L.lmax > 0.0) {
      const double lmx = o.cheb_hi * L.lmax, lmn = o.cheb_lo * L.lmax;
      const double theta = 0.5 * (lmx + lmn), delta = 0.5 * (lmx - lmn), sigma = theta / delta;
      double rho_prev = 1.0 / sigma;
      coef[0] = 1.0 / theta;
      for (int k = 1; k < L.degree; ++k) {
        const double rho = 1.0 / (2.0 * sigma - rho_prev);
        coef[2 * k] = rho * rho_prev;
        coef[2 * k + 1] = 2.0 * rho / delta;
        rho_prev = rho;
      }
    }
    DP_CUDA(cudaMemcpyAsync(L.cheb, coef, sizeof(coef), cudaMemcpyHostToDevice, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
  }
  c.mg_degree = deg + 16 * deg_coarse;  // both degrees shape the captured graph
  DP_CUDA(cudaFree(diag));
  // coarse dense inverse
  if (c.coarse_n > 0) {
    MGLevel& L = c.mg.back();
    const int n = (int)c.coarse_n;
    double* D = c.coarse_inv;
    double* Inv = D + (size_t)n * n;
    DP_CUDA(cudaMemsetAsync(D, 0, sizeof(double) * n * n, c.stream));
    if (L.g.det)
      klaunch(k_dense_assemble_seq<T>, 1, 128, 0, c.stream, level_K<T>(L), D, (int)L.g.nel, L.g.ncr, (int)L.g.A(),
              (int)L.g.B(), n);
    else
      klaunch(k_dense_assemble<T>, (int)div_up(L.g.nel, 128), 128, 0, c.stream, level_K<T>(L), D, (int)L.g.nel,
              L.g.ncr, (int)L.g.A(), (int)L.g.B(), n);
    klaunch(k_dense_fix_diag, (int)div_up(n, 256), 256, 0, c.stream, D, n);
    double* buf[2] = {D, Inv};
    double* W = nullptr;   // panel inverse (kGJPanel^2) and T (n x kGJPanel)
    DP_CUDA(cudaMalloc(&W, sizeof(double) * (kGJPanel * kGJPanel + (size_t)n * kGJPanel)));
    double* Tc = W + kGJPanel * kGJPanel;
    const int npanel = (int)div_up(n, kGJPanel);
    for (int p = 0; p < npanel; ++p) {
      const int k0 = p * kGJPanel, b = std::min(kGJPanel, n - k0);
      const double* Aold = buf[p & 1];
      klaunch(k_gj_panel_inverse, 1, dim3(kGJPanel, kGJPanel), 0, c.stream, Aold, W, n, k0, b);
      klaunch(k_gj_panel_cols, (int)div_up((int64_t)n * kGJPanel, 256), 256, 0, c.stream, Aold, (const double*)W, Tc,
              n, k0, b);
      klaunch(k_gj_panel_update, (int)div_up((int64_t)n * n, 256), 256, 0, c.stream, Aold, buf[(p + 1) & 1],
              (const double*)W, (const double*)Tc, n, k0, b);
    }
    // panel p writes buf[(p + 1) & 1]: for an even panel count the inverse ends in D
    if (!(npanel & 1)) DP_CUDA(cudaMemcpyAsync(Inv, D, sizeof(double) * n * n, cudaMemcpyDeviceToDevice, c.stream));
    klaunch(k_symmetrize, (int)div_up((int64_t)n * n, 256), 256, 0, c.stream, Inv, n);
    DP_LAUNCH_CHECK();
    DP_CUDA(cudaStreamSynchronize(c.stream));
    DP_CUDA(cudaFree(W));
  }
}

void mg_setup(Ctx& c, int precision, const MGOptions& o) {
  if (precision == 1) mg_setup_t<float>(c, o);
  else mg_setup_t<double>(c, o);
}

// Chebyshev smoothing of A x = b on level L.  mode 0: start from x = 0;
// mode 1: start from x = 0 with the first step already taken (fused into the
// restriction that produced b); mode 2: start from the given x, with L.r
// holding b on entry (the prolongation copies it there).  The recurrence
// coefficients live in L.cheb on the device, so this sequence is the same for
// every assembly and is captured once into the solve graph.
// On exit r = b - A (x - d_last), i.e. the true residual is r - A d_last.
template <typename T>
static void chebyshev(Ctx& c, MGLevel& L, const T* b, T* x, int mode) {
  const int64_t nn = L.g.nnod;
  T* r = (T*)L.r; T* d = (T*)L.d;
  const T* dinv = level_dinv<T>(L);
  if (mode == 0) {
    klaunch(k_cheb_first<T>, tpb(nn), 256, 0, c.stream, b, dinv, x, r, d, L.cheb, nn);
  } else if (mode == 2) {
    launch_apply_K_sub<T, T>(L.g, level_K<T>(L), x, r, c.stream);
    klaunch(k_cheb_first_x<T>, tpb(nn), 256, 0, c.stream, (const T*)r, dinv, x, d, L.cheb, nn);
  }
  for (int k = 1; k < L.degree; ++k) {
    launch_apply_K_sub<T, T>(L.g, level_K<T>(L), d, r, c.stream);
    klaunch(k_cheb_step<T>, tpb(nn), 256, 0, c.stream, (const T*)r, dinv, x, d, L.cheb + 2 * k, nn);
  }
  DP_LAUNCH_CHECK();
}

// first_done: the level's first pre-smoothing step was fused into the restriction.
template <typename T>
static void vcycle(Ctx& c, size_t l, const T* b, T* x, const MGOptions& o, bool first_done) {
  if (l == tail_start(c, o)) {
    launch_vcycle_tail<T>(c, l, b, x, first_done, o);
    return;
  }
  MGLevel& L = c.mg[l];
  const bool dense_coarsest = c.coarse_n > 0;
  if (l + 1 == c.mg.size()) {
    if (dense_coarsest) {
      // dense inverse: identity rows on constrained DOFs keep them at zero
      const int nn = (int)c.coarse_n;
      const double* Inv = c.coarse_inv + (size_t)nn * nn;
      klaunch(k_dense_apply<T>, nn, 128, 0, c.stream, Inv, b, x, nn);
      DP_LAUNCH_CHECK();
    } else {
      chebyshev<T>(c, L, b, x, first_done ? 1 : 0);
      for (int s = 1; s < o.coarse_sweeps; ++s) {
        DP_CUDA(cudaMemcpyAsync(L.r, b, sizeof(T) * 2 * L.g.nnod, cudaMemcpyDeviceToDevice, c.stream));
        chebyshev<T>(c, L, b, x, 2);
      }
    }
    return;
  }
  MGLevel& C = c.mg[l + 1];
  T* r = (T*)L.r;
  T* bc = (T*)C.b;
  T* xc = (T*)C.x;
  // pre-smoothing, r -= A d_last (the true residual), then restrict it (and take
  // the coarse level's first smoothing step in the same pass unless it is
  // solved densely)
  chebyshev<T>(c, L, b, x, first_done ? 1 : 0);
  launch_apply_K_sub<T, T>(L.g, level_K<T>(L), (const T*)L.d, r, c.stream);
  const bool fuse = !(l + 2 == c.mg.size() && dense_coarsest);
  // the cluster tail's smoother accumulates A d into t, which starts at zero
  T* tc = (l + 1 == tail_start(c, o)) ? (T*)C.t : nullptr;
  const int nA0 = (int)((C.g.A() + 1) >> 1);  // coarse nodes per parity class (upper bound)
  // the tiled form needs whole tiles along theta (its patch then wraps at most once)
  const bool small = C.g.nnod < 32768 || C.g.B() % kRTile != 0;
  if (small) {
    dim3 grid((unsigned)div_up(4 * (int64_t)nA0 * (C.g.B() >> 1), 256), 4);
    klaunch(k_restrict_g<T, 4>, grid, 256, 0, c.stream, (const T*)r, (const T*)nullptr, bc, (int)L.g.A(),
            (int)L.g.B(), (int)C.g.A(), (int)C.g.B(), C.g.pin, fuse ? 1 : 0, (const T*)level_dinv<T>(C), xc, (T*)C.r,
            (T*)C.d, tc, (const double*)C.cheb);
  } else {
    dim3 grid((unsigned)div_up(C.g.A(), kRTile), (unsigned)div_up(C.g.B(), kRTile));
    klaunch(k_restrict_tile<T>, grid, 256, 0, c.stream, (const T*)r, (const T*)nullptr, bc, (int)L.g.A(),
            (int)L.g.B(), (int)C.g.A(), (int)C.g.B(), C.g.pin, fuse ? 1 : 0, (const T*)level_dinv<T>(C), xc,
            (T*)C.r, (T*)C.d, tc, (const double*)C.cheb);
  }
  DP_LAUNCH_CHECK();
  vcycle<T>(c, l + 1, bc, xc, o, fuse);
  klaunch(k_prolong_add<T>, tpb(L.g.nnod), 256, 0, c.stream, (const T*)xc, x, b, r, (int)L.g.A(), (int)L.g.B(),
          C.g.ncr, (int)C.g.A(), (int)C.g.B(), L.g.pin);
  DP_LAUNCH_CHECK();
  chebyshev<T>(c, L, b, x, 2);
}

void mg_apply(Ctx& c, const double* b, double* x, const MGOptions& o) { vcycle<double>(c, 0, b, x, o, false); }
void mg_apply_f(Ctx& c, const float* b, float* x, const MGOptions& o) { vcycle<float>(c, 0, b, x, o, false); }

}  // namespace dp
