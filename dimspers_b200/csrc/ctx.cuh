// Context, device buffers and shared helpers of the B200 Stokes path.
//
// Device data layout (everything lives in HBM for the lifetime of a ctx):
//   lattice nodes     n = a + A*b, a = 0..2*ncr (radial), b = 0..2*nct-1 (angular,
//                     periodic); A = 2*ncr+1, B = 2*nct
//   velocity vectors  interleaved [u_theta, u_r] per lattice node (2*nnod)
//   pressure          continuous: vertex index (ref numbering = lattice vertex
//                     (a/2) + (ncr+1)*(b/2)); discontinuous: 3*e + k
//   element arrays    structure-of-arrays, entry-major: X[k*nel + e]
//                     (coalesced across consecutive elements)
//   elements          reference order e = 2*q + t, q = ir + ncr*it,
//                     connectivity derived from (ir, it, t) -- no index arrays
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "mesh.hpp"

namespace dp {

// Kernels launched by this thread (every launch site increments it); used to
// report the launches of a solve and, while capturing, the kernels per graph body.
inline thread_local int64_t g_klaunch = 0;

constexpr int kNip = 6;
constexpr int kKe = 78;   // packed lower 12x12
constexpr int kGe = 36;   // 12x3 column-major
constexpr int kMe = 6;    // packed lower 3x3
constexpr int kFe = 12;
constexpr int kDetPerElem = 18;  // deterministic scratch per element: 6 nodes x up to 3 values
constexpr int kMfTab = 84;  // per ring of the matrix-free apply: 6 IPs x (6 dN/dx, 6 dN/dz), 6 x (cos, sin)

enum MatKind { MAT_NONE = 0, MAT_ISO = 1, MAT_FULL = 2, MAT_TI = 3 };

// Geometry of one level of the structured hierarchy.
struct Level {
  int ncr = 0, nct = 0;
  int pin = 0;               // u_theta of lattice node (2*ncr, 0) is fixed
  int64_t nel = 0, nnod = 0;
  // Tile of the element-by-element applies: a CTA of `warps` warps, `warps_t` of
  // them stacked along theta (each warp = 16 radial cells x 2 triangles); the
  // stacked form needs ncr % 16 == 0 and falls back to the linear element order.
  int warps = 4, warps_t = 1;
  // Matrix-free element apply (fine level only): om * Q^T D Q per element and
  // IP (36 per element, ring-major) and the per-ring reference tables.  Null:
  // the applies read the packed element matrices.
  const double* mfD64 = nullptr;
  const double* mfT64 = nullptr;
  const float* mfD32 = nullptr;
  const float* mfT32 = nullptr;
  // Deterministic mode: scratch for per-element results (kDetPerElem values per
  // element, level precision), summed per node in a fixed order by
  // k_node_gather instead of scatter-added with atomics.  Null: atomics.
  void* det = nullptr;
  int64_t A() const { return 2 * (int64_t)ncr + 1; }
  int64_t B() const { return 2 * (int64_t)nct; }
};

template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
};

struct MGLevel {
  Level g;
  double* K64 = nullptr;     // 78*nel packed polar, masked
  float* K32 = nullptr;
  double* dinv64 = nullptr;  // 3*nnod inverse of the 2x2 nodal diagonal blocks (i00, i01, i11)
  float* dinv32 = nullptr;
  double lmax = 0.0;         // estimate of lambda_max(D^-1 A)
  int degree = 3;            // Chebyshev steps on this level
  double* cheb = nullptr;    // device: [1/theta, -, (c1, c2) per further step]
  // work vectors (precision of the hierarchy)
  void* x = nullptr;
  void* b = nullptr;
  void* r = nullptr;
  void* d = nullptr;
  void* t = nullptr;
};

struct Ctx {
  Mesh mesh;
  Level fine;
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;

  // geometry
  double* theta_lat = nullptr;  // nnod
  double* r_lat = nullptr;      // nnod
  int64_t* ref2lat = nullptr;   // nnod

  // material
  int mat_kind = MAT_NONE;
  double g = 0.0;
  double* eta = nullptr;        // 6*nel (ip-major)
  double* C = nullptr;          // FULL: 36*nel (field*6+ip); TI: 3*nel (delta, dx, dy)
  double* rho_lat = nullptr;    // nnod
  double* rho_ref = nullptr;    // nnod (reference numbering, for uploads)

  // assembled (polar, masked)
  int assembled = -1;           // precision of the last assembly, -1 = none
  double* K64 = nullptr;        // 78*nel
  float* K32 = nullptr;         // 78*nel (refined path)
  double* mfD64 = nullptr;      // 36*nel: matrix-free apply data (written by every assembly)
  double* mfT64 = nullptr;      // kMfTab*2*ncr
  float* mfD32 = nullptr;       // FP32 copies for the FP32 levels
  float* mfT32 = nullptr;
  bool mf32_stale = true;       // the FP32 copies predate the last assembly
  double* det_buf = nullptr;    // kDetPerElem*nel: deterministic mode's element results (dp_set_deterministic)
  double* Gp = nullptr;         // 36*nel
  double* F = nullptr;          // 2*nnod
  double* pc = nullptr;         // npres (1/rowsum M)
  double* Minv = nullptr;       // 6*nel inverse element mass blocks (discontinuous pressure)
  double* Fscale = nullptr;
  void* flush = nullptr;        // L2 flush buffer for cold kernel timings
  double* stress_buf = nullptr; // post-processor staging: eta 7, tensor 42, outputs 56 per element
  bool stress_tensor = false;   // the staged inputs carry a tensor
  double* rheo_buf = nullptr;   // viscosity update staging: 4 x 7 per element, 4 per node
  double* fabric_buf = nullptr; // FSE / DEM tensor staging (fabric_cap doubles)
  int64_t fabric_cap = 0;
  int64_t fabric_dem[3] = {0, 0, 0};  // the last staged DEM table: nrows, n_a1a2, sblk (0: none)
  double fabric_w = 0.0;
  double* th_buf = nullptr;     // thermal step: 21 x nel element blocks + 10 nnod vectors
  void* th_exec = nullptr;      // cudaGraphExec_t of the thermal CG loop
  int th_heated = -1;           // wall configuration the loop graph was captured for
  double rheo_law[8] = {};      // the last viscosity update's law (eta0, R, Ea, Va, T0, sin, cos, phi)

  // multigrid hierarchy (level 0 = fine)
  std::vector<MGLevel> mg;
  int mg_prec = -1;             // 0 = fp64, 1 = fp32
  int mg_degree = 3;            // Chebyshev steps in use
  int64_t mg_coarse_max = -1;   // coarse_max the hierarchy was built for
  int64_t alloc_gen = 0;        // bumped whenever buffers a captured graph may hold are freed
  double* coarse_inv = nullptr; // coarsest level: work matrix, then its dense inverse (2 n^2)
  int64_t coarse_n = 0;
  int64_t* coarse_map = nullptr;// coarsest DOF -> dense index (-1 fixed)

  // scratch
  double* scal = nullptr;       // device scalars
  double* h_scal = nullptr;     // pinned host mirror
  double* partial = nullptr;    // reduction partials
  unsigned int* counter = nullptr;
  std::vector<void*> work;      // solver vectors

  // graph-captured solve (graph.cu)
  void* ctl = nullptr;          // device control block (DevCtl)
  void* h_ctl = nullptr;        // pinned host mirror
  cudaStream_t aux[4] = {nullptr, nullptr, nullptr, nullptr};  // capture streams of nested loop bodies
  void* graph = nullptr;        // cudaGraph_t
  void* gexec = nullptr;        // cudaGraphExec_t
  int64_t gkey = -1;
  int64_t ggen = -1;            // alloc_gen the cached graph was captured with
  const void* gU = nullptr;
  const void* gP = nullptr;
  int64_t gk_main = 0;          // kernel nodes outside loop bodies
  int64_t cap_nested = 0;       // kernels captured inside nested bodies (capture bookkeeping)
  int64_t gk_body[5] = {0, 0, 0, 0, 0};  // kernel nodes per body execution (outer, pcg64, pcg32, refinement, restart)

  ~Ctx();
};

// ---- error handling --------------------------------------------------------
struct CudaError {
  cudaError_t e;
  const char* what;
  int line;
};

#define DP_CUDA(call)                                             \
  do {                                                            \
    cudaError_t e__ = (call);                                     \
    if (e__ != cudaSuccess) throw ::dp::CudaError{e__, #call, __LINE__}; \
  } while (0)

#define DP_LAUNCH_CHECK() DP_CUDA(cudaGetLastError())

// ---- programmatic dependent launch -------------------------------------------
// The solver is a long chain of short kernels, many of them (coarse multigrid
// levels, reductions, control) shorter than their own launch latency.  With
// g_pdl set, klaunch gives each launch the programmatic-stream-serialization
// attribute: the kernel may be scheduled while its predecessor is still
// running, and waits in grid_dep_wait() (griddepcontrol.wait, which returns
// once the predecessor grid has completed and its memory is visible) before it
// touches memory.  Every kernel of the solve path calls grid_dep_wait() first,
// so a launch with or without the attribute computes the same thing; without
// the attribute the wait returns at once.
__device__ __forceinline__ void grid_dep_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

inline thread_local int g_pdl = 0;
// Scheduling priority given to kernels while a batch is captured (per-node
// priorities of the batch graph); kNoPriority = the stream's own.
constexpr int kNoPriority = 1 << 30;
inline thread_local int g_prio = kNoPriority;

template <typename... P, typename... A>
inline void klaunch(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args) {
  ++g_klaunch;
  cudaLaunchAttribute attr[2];
  unsigned n = 0;
  if (g_pdl) {
    attr[n].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[n].val.programmaticStreamSerializationAllowed = 1;
    ++n;
  }
  if (g_prio != kNoPriority) {
    attr[n].id = cudaLaunchAttributePriority;
    attr[n].val.priority = g_prio;
    ++n;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = n;
  DP_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<P>(args)...));
}

// ---- lattice helpers (host + device) ---------------------------------------
// Constrained DOFs: u_r on both walls (free slip, boundary_conditions.jl:27-37)
// and, when pinned, u_theta of the outer-wall node at theta = 0 (the one-node
// tangential constraint of free_slip(nr, ids), boundary_conditions.jl:180-194).
__host__ __device__ inline bool dof_fixed(int a, int b, int comp, int amax, int pin) {
  if (comp == 1) return a == 0 || a == amax;
  return pin && a == amax && b == 0;
}

__host__ __device__ inline int64_t wrapb(int64_t b, int64_t B) { return b >= B ? b - B : (b < 0 ? b + B : b); }

// Lattice (a, b) of the 6 local nodes of element e on a level with ncr radial cells.
__host__ __device__ inline void element_nodes(int64_t e, int ncr, int64_t A, int64_t B, int64_t n[6]) {
  const int64_t q = e >> 1;
  const int t = (int)(e & 1);
  const int64_t ir = q % ncr, it = q / ncr;
  const int64_t a0 = 2 * ir, b0 = 2 * it;
  int64_t a[6], b[6];
  if (t == 0) {  // [v1, v2, v4]
    a[0] = a0;     b[0] = b0;
    a[1] = a0;     b[1] = b0 + 2;
    a[2] = a0 + 2; b[2] = b0;
    a[3] = a0;     b[3] = b0 + 1;
    a[4] = a0 + 1; b[4] = b0 + 1;
    a[5] = a0 + 1; b[5] = b0;
  } else {       // [v2, v3, v4]
    a[0] = a0;     b[0] = b0 + 2;
    a[1] = a0 + 2; b[1] = b0 + 2;
    a[2] = a0 + 2; b[2] = b0;
    a[3] = a0 + 1; b[3] = b0 + 2;
    a[4] = a0 + 2; b[4] = b0 + 1;
    a[5] = a0 + 1; b[5] = b0 + 1;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) n[k] = a[k] + A * wrapb(b[k], B);
}

__host__ __device__ inline void element_pdofs_cont(int64_t e, int ncr, int nct, int64_t p[3]) {
  const int64_t q = e >> 1;
  const int t = (int)(e & 1);
  const int64_t ir = q % ncr, it = q / ncr;
  const int64_t nr = ncr + 1;
  const int64_t it1 = (it + 1 == nct) ? 0 : it + 1;
  const int64_t v1 = ir + nr * it, v2 = ir + nr * it1, v3 = ir + 1 + nr * it1, v4 = ir + 1 + nr * it;
  if (t == 0) { p[0] = v1; p[1] = v2; p[2] = v4; }
  else        { p[0] = v2; p[1] = v3; p[2] = v4; }
}

// Pressure DOFs of element e: continuous = vertex numbering (EL2NOD[1:3,:],
// mesher.jl:213); discontinuous = 3e+k (reshape(1:3nel,3,nel), mesher.jl:212).
__host__ __device__ inline void element_pdofs(int64_t e, int ncr, int nct, int pressure, int64_t p[3]) {
  if (pressure == 1) {
    p[0] = 3 * e; p[1] = 3 * e + 1; p[2] = 3 * e + 2;
  } else {
    element_pdofs_cont(e, ncr, nct, p);
  }
}

// Packed lower-column-major index of the 12x12 element matrix entry (R >= C);
// the reference's loops emit Ke in this order (StokesSolver.jl:696-741).
__host__ __device__ constexpr int packed_index12(int R, int C) {
  // R >= C; column-major lower packing of a 12x12 matrix
  return C * 12 - (C * (C - 1)) / 2 + (R - C);
}

inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Packed element matrices are stored array-of-structures-of-arrays: elements in
// warp blocks of 32; inside a block the 78 entries of consecutive elements are
// interleaved in 16-byte groups (2 doubles / 4 floats), so a warp loading group j
// of its 32 elements reads 512 contiguous bytes and each thread issues 39
// (FP64) or 20 (FP32, 78 entries padded to 80) 16-byte loads.
__host__ __device__ inline int64_t kpad(int64_t nel) { return (nel + 31) & ~(int64_t)31; }
__host__ __device__ inline int64_t kidx64(int p, int64_t e) {
  return (e >> 5) * (32 * 78) + (int64_t)(p >> 1) * 64 + (e & 31) * 2 + (p & 1);
}
__host__ __device__ inline int64_t kidx32(int p, int64_t e) {
  return (e >> 5) * (32 * 80) + (int64_t)(p >> 2) * 128 + (e & 31) * 4 + (p & 3);
}
template <typename T>
__host__ __device__ inline int64_t kidx(int p, int64_t e);
template <>
__host__ __device__ inline int64_t kidx<double>(int p, int64_t e) { return kidx64(p, e); }
template <>
__host__ __device__ inline int64_t kidx<float>(int p, int64_t e) { return kidx32(p, e); }
// number of T in the packed store of nel elements
template <typename T>
inline int64_t kstore(int64_t nel) { return kpad(nel) * (sizeof(T) == 8 ? 78 : 80); }

}  // namespace dp
