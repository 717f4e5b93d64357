// Multigrid hierarchy interface and lattice helpers shared by its kernels.
#pragma once
#include "ctx.cuh"

namespace dp {

constexpr int kMaxCheb = 8;

struct MGOptions {
  int cheb_degree = 3;      // Chebyshev steps per smoothing (each one A-apply)
  int cheb_degree_coarse = 0;  // on the levels below the finest (0: cheb_degree)
  double cheb_lo = 0.15;    // smoothing interval [lo, hi] * lambda_max(D^-1 A)
  double cheb_hi = 1.1;
  int block_jacobi = 1;     // 1: 2x2 nodal blocks (u_theta, u_r); 0: point Jacobi
  int max_levels = 16;
  int64_t coarse_max = 1536;// largest dense coarsest system
  int coarse_sweeps = 4;    // smoothing sweeps when the coarsest is not dense
  int64_t tail_max_el = 0;  // levels up to this many elements run as one cluster kernel (0: off)
  int apply_warps = 4;      // tile of the element-by-element applies (Level::warps)
  int apply_warps_t = 1;    // (Level::warps_t)
};

// Local node offsets (radial, angular) inside the cell for triangle type t.
__host__ __device__ inline int kLocA_dev(int t, int k) {
  const int A0[6] = {0, 0, 2, 0, 1, 1}, A1[6] = {0, 2, 2, 1, 2, 1};
  return t == 0 ? A0[k] : A1[k];
}
__host__ __device__ inline int kLocB_dev(int t, int k) {
  const int B0[6] = {0, 2, 0, 1, 1, 0}, B1[6] = {2, 2, 0, 2, 1, 1};
  return t == 0 ? B0[k] : B1[k];
}
__host__ __device__ inline void element_nodes_mg(int e, int ncr, int A, int B, int nd[6]) {
  const int q = e >> 1, t = e & 1;
  const int ir = q % ncr, it = q / ncr;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    int b = 2 * it + kLocB_dev(t, k);
    if (b >= B) b -= B;
    nd[k] = 2 * ir + kLocA_dev(t, k) + A * b;
  }
}

void upload_mg_constants();
void mg_setup(Ctx& c, int precision, const MGOptions& o);
void mg_free(Ctx& c);
void mg_apply(Ctx& c, const double* b, double* x, const MGOptions& o);
void mg_apply_f(Ctx& c, const float* b, float* x, const MGOptions& o);

// The small levels as one thread-block-cluster kernel (mgtail.cu): first level
// it covers, and its launcher (V-cycle of levels l0.. with b, x of level l0).
size_t tail_start(const Ctx& c, const MGOptions& o);
template <typename T>
void launch_vcycle_tail(Ctx& c, size_t l0, const T* b, T* x, bool first_done, const MGOptions& o);

}  // namespace dp
