// Launchers of the device kernels (one declaration per kernel family).
#pragma once
#include "ctx.cuh"

namespace dp {

// ---- quadrature constants (uploaded once per device) -----------------------
void upload_quadrature_constants();

// ---- assembly (assemble.cu) -----------------------------------------------
struct CartOut {   // optional reference-layout Cartesian element blocks (78/36/6/12 x nel)
  double* Ke = nullptr;
  double* Ge = nullptr;
  double* Me = nullptr;
  double* Fb = nullptr;
};
void launch_assemble(Ctx& c, int precision, const CartOut* cart);
void launch_ti_tensor_fill(Ctx& c, const double* delta, const double* dx, const double* dy);
void launch_fse_director(Ctx& c, const double* F, double* dx, double* dy, int64_t nel);

// ---- operator applies (ops.cu) --------------------------------------------
template <typename Tm, typename Tv>
void launch_apply_K(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s);       // zeroes y
template <typename Tm, typename Tv>
void launch_apply_K_acc(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s);   // y += K x
template <typename Tm, typename Tv>
void launch_apply_K_sub(const Level& L, const Tm* K, const Tv* x, Tv* y, cudaStream_t s);   // y -= K x
// Deterministic mode: per node, y (mode 0: +=, 1: -=, 2: =) the sum over its
// elements, in a fixed order, of E[(nc k + c) nel + e] (nc = 2; nc = 3 with mode 2)
template <typename T>
void launch_node_gather(const Level& L, const T* E, T* y, int nc, int mode, cudaStream_t s);
void launch_apply_G(Ctx& c, const double* p, double* y);     // y = G p   (zeroes y)
void launch_apply_GT(Ctx& c, const double* x, double* p);    // p = G^T x (zeroes p)

// ---- vector kernels & reductions (ops.cu) ---------------------------------
// out[slot] = sum_i a_i * b_i, deterministic (fixed grid, fixed order)
void launch_dot(Ctx& c, const double* a, const double* b, int64_t n, int slot);
void launch_dot_f(Ctx& c, const float* a, const float* b, int64_t n, int slot);
void launch_sum(Ctx& c, const double* a, int64_t n, int slot);
// compensated (double-double) dot and sum: the Schur-complement reductions
void launch_dot_c(Ctx& c, const double* a, const double* b, int64_t n, int slot);
void launch_sum_c(Ctx& c, const double* a, int64_t n, int slot);
void launch_gather_ref2lat(Ctx& c, const double* ref, double* lat, int comps);
void launch_scatter_lat2ref(Ctx& c, const double* lat, double* ref, int comps);
void launch_pc_invert(Ctx& c, double* pc, int64_t n);

}  // namespace dp
