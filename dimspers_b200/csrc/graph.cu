// The whole Stokes solve as one CUDA graph with device-side control flow.
//
// StokesPcCG (IterativeSolvers.jl:94-168) is a loop of outer Schur iterations,
// each with an inner K-solve that is itself a loop (PCG, and for the
// FP32-refined path a refinement loop around an FP32 PCG).  Every loop here
// is a WHILE conditional graph node whose condition is set on the device
// (cudaGraphSetConditional) at the end of its body, by a one-thread check
// kernel or, for the inner PCG, by the last block of the update kernel, so a
// solve is one graph launch and one final synchronisation: no host
// round-trip per iteration.  Stopping tests are the reference's:
//   outer: ||r|| < rtol * ||r0|| and it >= itmin, or it == itmax,
//          or breakdown (q.Sq <= 0 / non-finite) -> status
//   inner: ||y - K z|| <= inner_rtol ||y|| or inner_itmax.
// In the true-residual mode the outer loop sits in one more WHILE loop that
// re-solves U = K^-1 (F + G P) and restarts until the TRUE residual passes.
// The captured sequence depends only on the hierarchy shape and the options
// baked into it (precision, preconditioner, guess, rotation removal), so the
// instantiated graph is cached in the context and reused across assemblies;
// tolerances and iteration caps are read from device memory at run time.
#include <algorithm>
#include <cstring>
#include <stdexcept>

#include "kernels.cuh"
#include "mg.cuh"
#include "reduce.cuh"
#include "solver.cuh"

namespace dp {

struct DevCtl {
  // parameters (written by the host before each launch)
  double rtol, inner_rtol, inner_rtol32, relax_cap, relax_base;
  int itmax, itmin, inner_itmax, max_refine;
  // state
  int outer_it, in_it, in32_it, ref_it, status, guess_used, restarts, max_restarts;
  long long in_total, in32_total, ref_total;
  double r0, tol, in_tol2, in32_tol2, ref_tol2, r0ref, r0guess;
};

enum GSlot { G_RZ = 16, G_RZN = 17, G_PAP = 18, G_IRR = 19, G_YY = 20,
             F_RZ = 21, F_RZN = 22, F_PAP = 23, F_IRR = 24, F_YY = 25,
             R_YY = 26, R_RES2 = 27, G_TMP3 = 28, G_RZREF = 29 };

// ---- control kernels (one thread) ---------------------------------------------
// Inner tolerance: fixed, or (relax) loosened in proportion to the outer
// residual, rtol_k = min(cap, max(inner_rtol, base * ||r0|| / ||r_k||)): an
// inexact-Krylov relaxation that keeps the product of step size and inner
// error bounded (base: the outer target's scale; inner_rtol when unset).
__device__ inline double inner_rtol_now(const DevCtl* ctl, const double* scal, int relax) {
  double rt = ctl->inner_rtol;
  if (relax && ctl->relax_cap > 0.0 && ctl->r0 > 0.0) {
    const double rk = sqrt(scal[S_RR]);
    const double base = ctl->relax_base > 0.0 ? ctl->relax_base : ctl->inner_rtol;
    if (rk > 0.0) rt = fmin(ctl->relax_cap, fmax(rt, base * ctl->r0 / rk));
  }
  return rt;
}

__global__ void k_in_init(cudaGraphConditionalHandle h, DevCtl* ctl, const double* scal, int yy_slot, int irr_slot,
                          double* scal_w, int fp32, int relax) {
  grid_dep_wait();
  const double yy = scal[yy_slot];
  const double rt = fp32 ? ctl->inner_rtol32 : inner_rtol_now(ctl, scal, relax);
  const double tol2 = rt * rt * yy;
  if (fp32) { ctl->in32_it = 0; ctl->in32_tol2 = tol2; }
  else { ctl->in_it = 0; ctl->in_tol2 = tol2; }
  scal_w[irr_slot] = yy;
  cudaGraphSetConditional(h, (yy > 0.0 && yy > tol2) ? 1u : 0u);
}

__global__ void k_ref_init(cudaGraphConditionalHandle h, DevCtl* ctl, double* scal, int relax) {
  grid_dep_wait();
  const double yy = scal[R_YY];
  const double rt = inner_rtol_now(ctl, scal, relax);
  ctl->ref_it = 0;
  ctl->ref_tol2 = rt * rt * yy;
  scal[R_RES2] = yy;
  cudaGraphSetConditional(h, yy > 0.0 ? 1u : 0u);
}

__global__ void k_ref_check(cudaGraphConditionalHandle h, DevCtl* ctl, const double* scal) {
  grid_dep_wait();
  const int it = ++ctl->ref_it;
  ctl->ref_total += 1;
  const double rr = scal[R_RES2];
  cudaGraphSetConditional(h, (isfinite(rr) && rr > ctl->ref_tol2 && it < ctl->max_refine) ? 1u : 0u);
}

// use_ref: the stopping tolerance is relative to the zero-guess residual
// ||r(P = 0)|| (learned-guess mode), so a guess shortens the solve only by
// starting closer to the same absolute target.
// A non-finite initial residual (a failed initial inner solve) is a breakdown,
// not a zero right-hand side.
__global__ void k_outer_init(cudaGraphConditionalHandle h, DevCtl* ctl, const double* scal, int use_ref) {
  grid_dep_wait();
  const double r0 = use_ref ? ctl->r0ref : sqrt(scal[S_RR]);
  ctl->r0 = r0;
  ctl->tol = r0 * ctl->rtol;
  ctl->outer_it = 0;
  ctl->status = !isfinite(r0) || !isfinite(scal[S_RR]) ? 2 : (r0 > 0.0 ? 1 : 0);
  cudaGraphSetConditional(h, (ctl->status == 1 && ctl->itmax >= 1) ? 1u : 0u);
}

__global__ void k_outer_check(cudaGraphConditionalHandle h, DevCtl* ctl, const double* scal) {
  grid_dep_wait();
  const int it = ++ctl->outer_it;
  const double qsq = scal[S_QSQ], rd = scal[S_RD], rn = sqrt(scal[S_RR]);
  unsigned go = 1u;
  if (!(qsq > 0.0) || !isfinite(qsq) || !isfinite(rd) || !isfinite(rn)) {
    ctl->status = 2;
    go = 0u;
  } else if (rn < ctl->tol && it >= ctl->itmin) {
    ctl->status = 0;
    go = 0u;
  } else if (it >= ctl->itmax) {
    go = 0u;
  }
  cudaGraphSetConditional(h, go);
}

// ---- true-residual restarts ------------------------------------------------------
// With relaxed (inexact) inner solves the outer residual r, updated by
// recurrence, drifts from the true Schur residual -G^T K^-1 (F + G P), and U
// (accumulated from inexact solves) from K^-1 (F + G P).  In the restart mode
// the outer loop runs inside a second WHILE loop: when it stops, U is solved
// afresh to the tight inner tolerance, the true residual is formed, and the
// loop restarts from the current P (same r0, same iteration count) unless the
// true residual meets the tolerance.
__global__ void k_outer_start(DevCtl* ctl, const double* scal, int use_ref) {
  grid_dep_wait();
  const double r0 = use_ref ? ctl->r0ref : sqrt(scal[S_RR]);
  ctl->r0 = r0;
  ctl->tol = r0 * ctl->rtol;
  ctl->outer_it = 0;
  ctl->restarts = 0;
  ctl->status = !isfinite(r0) || !isfinite(scal[S_RR]) ? 2 : (r0 > 0.0 ? 1 : 0);
}
__global__ void k_restart_init(cudaGraphConditionalHandle h, const DevCtl* ctl) {
  grid_dep_wait();
  cudaGraphSetConditional(h, (ctl->status == 1 && ctl->itmax >= 1) ? 1u : 0u);
}
// outer loop (re)entry: continue while the current (true) residual misses the tolerance
__global__ void k_outer_resume(cudaGraphConditionalHandle h, DevCtl* ctl, const double* scal) {
  grid_dep_wait();
  const double rn = sqrt(scal[S_RR]);
  const bool done = (rn < ctl->tol && ctl->outer_it >= ctl->itmin) || ctl->outer_it >= ctl->itmax;
  ctl->status = done ? (rn < ctl->tol ? 0 : 1) : 1;
  cudaGraphSetConditional(h, done ? 0u : 1u);
}
__global__ void k_restart_check(cudaGraphConditionalHandle h, DevCtl* ctl, const double* scal) {
  grid_dep_wait();
  ctl->restarts += 1;
  const double rn = sqrt(scal[S_RR]);
  unsigned go = 0u;
  if (ctl->status == 2) {
    go = 0u;                                   // breakdown
  } else if (rn < ctl->tol && ctl->outer_it >= ctl->itmin) {
    ctl->status = 0;
  } else {
    ctl->status = 1;
    go = (ctl->outer_it < ctl->itmax && ctl->restarts <= ctl->max_restarts) ? 1u : 0u;
  }
  cudaGraphSetConditional(h, go);
}

// Learned-guess selection: keep the guess only if its initial Schur residual
// is below the zero guess's (otherwise fall back to P = 0).
__global__ void k_guess_select(DevCtl* ctl, double* scal) {
  grid_dep_wait();
  const double rg = scal[S_RR], rz = scal[G_RZREF];
  const int use = rg < rz ? 1 : 0;
  ctl->guess_used = use;
  ctl->r0ref = sqrt(rz);
  ctl->r0guess = sqrt(rg);
  if (!use) {
    scal[S_RR] = rz;
  }
}
__global__ void k_guess_apply(const DevCtl* ctl, double* __restrict__ U, const double* __restrict__ Uz,
                              double* __restrict__ r, const double* __restrict__ rz, double* __restrict__ P,
                              int64_t nU, int64_t nP) {
  grid_dep_wait();
  if (ctl->guess_used) return;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < nU) U[i] = Uz[i];
  if (i < nP) {
    r[i] = rz[i];
    P[i] = 0.0;
  }
}

// ---- PCG vector kernels reading their scalars from the table --------------------
// p = z + beta p with beta = rzn/rz, except p = z on the first iteration
template <typename T>
__global__ void k_pcg_dir_g(T* __restrict__ p, const T* __restrict__ z, T* __restrict__ Ap, int64_t n,
                            const double* scal, int rzn, int rz, const int* it) {
  grid_dep_wait();
  const double beta = (*it == 0 || scal[rz] == 0.0) ? 0.0 : scal[rzn] / scal[rz];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) {
    p[i] = (T)((double)z[i] + beta * (double)p[i]);
    Ap[i] = (T)0;  // the next apply accumulates into Ap
  }
}

// p = s z32 + beta p (s = ||b||, the FP32 V-cycle ran on r / ||b||), Ap = 0:
// the mixed-precision form reads the FP32 preconditioned residual directly
__global__ void k_pcg_dir_f32z(double* __restrict__ p, const float* __restrict__ z32, double* __restrict__ Ap,
                               int64_t n, const double* scal, int yy, int rzn, int rz, const int* it) {
  grid_dep_wait();
  const double beta = (*it == 0 || scal[rz] == 0.0) ? 0.0 : scal[rzn] / scal[rz];
  const double s = sqrt(scal[yy]);
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) {
    p[i] = s * (double)z32[i] + beta * p[i];
    Ap[i] = 0.0;  // the next apply accumulates into Ap
  }
}

// FP64 residual -> FP32 hierarchy input, scaled by 1/sqrt(scal[irr]) (keeps FP32 in range)
__global__ void k_r_to_f32(const double* __restrict__ r, float* __restrict__ r32, const double* scal, int irr, int64_t n) {
  grid_dep_wait();
  const double s = 1.0 / sqrt(scal[irr]);
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) r32[i] = (float)(s * r[i]);
}
// nodal block Jacobi with an inverse of another precision
template <typename Td, typename Tv>
__global__ void k_bj_mixed(const Td* __restrict__ dinv, const Tv* __restrict__ r, Tv* __restrict__ z, int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  double z0, z1;
  bj_apply<Td>(dinv, n, (double)r[2 * n], (double)r[2 * n + 1], z0, z1);
  z[2 * n] = (Tv)z0;
  z[2 * n + 1] = (Tv)z1;
}

// x += alpha p; r -= alpha Ap; alpha = rzn/pAp; ||r||^2 -> irr

// rz = r . z with z = ||b|| z32 (the V-cycle ran on r / ||b||); z itself is
// never stored: k_pcg_dir_f32z reads z32 again
__global__ void __launch_bounds__(kRedThreads) k_rz_f32(const float* __restrict__ z32, const double* __restrict__ r,
                                                        double* scal, int yy, int rzn, int64_t n, double* partial,
                                                        unsigned int* counter) {
  grid_dep_wait();
  const double sc = sqrt(scal[yy]);
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads)
    s += r[i] * (sc * (double)z32[i]);
  double v[1] = {s};
  double* o[1] = {scal + rzn};
  grid_finish<1>(v, partial, counter, o);
}

// x += alpha p; r -= alpha Ap; ||r||^2 (alpha = rz / pAp from the table); the
// last block also takes the loop's stopping decision: continue while
// ||r||^2 > tol^2 ||b||^2 and it < inner_itmax.  r32 != null (FP64 Krylov on
// the FP32 hierarchy): also writes the next V-cycle's input r / ||b||.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_pcg_upd_check(T* __restrict__ x, T* __restrict__ r,
                                                                const T* __restrict__ p, const T* __restrict__ Ap,
                                                                int64_t n, double* scal, int rz, int rzn, int pap,
                                                                int irr, double* partial, unsigned int* counter,
                                                                cudaGraphConditionalHandle h, DevCtl* ctl, int fp32,
                                                                float* __restrict__ r32, int yy) {
  grid_dep_wait();
  const double inv_s = r32 ? 1.0 / sqrt(scal[yy]) : 0.0;
  // a non-positive or non-finite p.Ap (breakdown, e.g. an FP32 operator that
  // rounding made indefinite) leaves x and r unchanged and ends the loop
  const double pap_v = scal[pap];
  const bool ok = pap_v > 0.0 && isfinite(pap_v) && isfinite(scal[rzn]);
  const double alpha = ok ? scal[rzn] / pap_v : 0.0;
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    x[i] += (T)(alpha * (double)p[i]);
    const double ri = (double)r[i] - alpha * (double)Ap[i];
    r[i] = (T)ri;
    if (r32) r32[i] = (float)(inv_s * ri);
    s += ri * ri;
  }
  double v[1] = {s};
  double* o[1] = {scal + irr};
  if (grid_finish<1>(v, partial, counter, o) && threadIdx.x == 0 && ctl != nullptr) {
    int it;
    double tol2;
    if (fp32) { it = ++ctl->in32_it; tol2 = ctl->in32_tol2; ctl->in32_total += 1; }
    else { it = ++ctl->in_it; tol2 = ctl->in_tol2; ctl->in_total += 1; }
    scal[rz] = scal[rzn];
    const double rr = scal[irr];
    const bool go = ok && isfinite(rr) && rr > tol2 && it < ctl->inner_itmax;
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

__global__ void k_to_f32_scaled(const double* __restrict__ a, float* __restrict__ b, const double* scal, int64_t n) {
  grid_dep_wait();
  const double s = 1.0 / sqrt(scal[R_RES2]);
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)(s * a[i]);
}
__global__ void k_add_f32_scaled(double* __restrict__ z, const float* __restrict__ e, const double* scal, int64_t n) {
  grid_dep_wait();
  const double s = sqrt(scal[R_RES2]);
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) z[i] += s * (double)e[i];
}

// ---- capture helpers ---------------------------------------------------------------
struct StreamSwap {
  Ctx& c;
  cudaStream_t saved;
  StreamSwap(Ctx& cc, cudaStream_t s) : c(cc), saved(cc.stream) { c.stream = s; }
  ~StreamSwap() { c.stream = saved; }
};

static cudaGraphConditionalHandle new_handle(cudaStream_t s) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  DP_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  if (st != cudaStreamCaptureStatusActive) throw std::runtime_error("stream is not capturing");
  cudaGraphConditionalHandle h;
  DP_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  return h;
}

// Appends a WHILE node on handle h at the current capture position of s and
// returns its body graph.
static cudaGraph_t add_while(cudaStream_t s, cudaGraphConditionalHandle h) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  DP_CUDA(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  DP_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
  DP_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return np.conditional.phGraph_out[0];
}

// Loop bodies by role, for the launch count: kernels per execution of each body.
enum BodyRole { B_OUTER = 0, B_PCG64 = 1, B_PCG32 = 2, B_REF = 3, B_RESTART = 4 };

// Captures emit() into body on the auxiliary stream of the given depth.
template <typename F>
static void capture_body(Ctx& c, cudaGraph_t body, int depth, int role, F&& emit) {
  cudaStream_t aux = c.aux[depth];
  DP_CUDA(cudaStreamBeginCaptureToGraph(aux, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  const int64_t start = g_klaunch;
  const int64_t saved = c.cap_nested;
  c.cap_nested = 0;
  {
    StreamSwap sw(c, aux);
    emit();
  }
  cudaGraph_t out = nullptr;
  DP_CUDA(cudaStreamEndCapture(aux, &out));
  const int64_t all = g_klaunch - start;
  c.gk_body[role] = all - c.cap_nested;   // kernels directly in this body
  c.cap_nested = saved + all;             // the whole subtree is nested for the parent
}

static int g_nb(int64_t n) { return (int)div_up(n, 256); }

// ---- emitted segments ----------------------------------------------------------------
// PCG on K (precision T) for b -> x with preconditioner pc_kind; slots per precision.
template <typename T>
static void emit_pcg(Ctx& c, const SolveCfg& cfg, const T* Kmat, const T* b, T* x, T* r, T* z, T* p, T* Ap, int depth,
                     int relax) {
  const Level& L = c.fine;
  const int64_t n = 2 * L.nnod;
  const bool f32 = std::is_same<T, float>::value;
  const int RZ = f32 ? F_RZ : G_RZ, RZN = f32 ? F_RZN : G_RZN, PAP = f32 ? F_PAP : G_PAP, IRR = f32 ? F_IRR : G_IRR,
            YY = f32 ? F_YY : G_YY;
  DevCtl* ctl = (DevCtl*)c.ctl;
  DP_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, c.stream));
  DP_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, c.stream));
  if (f32) launch_dot_f(c, (const float*)b, (const float*)b, n, YY);
  else launch_dot(c, (const double*)b, (const double*)b, n, YY);
  // FP64 Krylov on the FP32 hierarchy: the V-cycle runs on r / ||b|| in FP32
  // (r32, written by the update kernel of the previous iteration) and its
  // output z32 is read directly by the dot and the direction update
  const bool mixed = cfg.inner_pc == 0 && !f32 && c.mg_prec == 1;
  float* r32 = (float*)c.work[W_F_R];
  float* z32 = (float*)c.work[W_F_Z];
  if (mixed) klaunch(k_r_to_f32, g_nb(n), 256, 0, c.stream, (const double*)b, r32, c.scal, YY, n);
  cudaGraphConditionalHandle h = new_handle(c.stream);
  klaunch(k_in_init, 1, 1, 0, c.stream, h, ctl, c.scal, YY, IRR, c.scal, f32 ? 1 : 0, relax);
  DP_LAUNCH_CHECK();
  cudaGraph_t body = add_while(c.stream, h);
  const int* itp = f32 ? &ctl->in32_it : &ctl->in_it;
  capture_body(c, body, depth, f32 ? B_PCG32 : B_PCG64, [&] {
    if (cfg.inner_pc == 0) {
      if (f32) {
        mg_apply_f(c, (const float*)r, (float*)z, cfg.mg);
      } else if (mixed) {
        mg_apply_f(c, r32, z32, cfg.mg);
      } else {
        mg_apply(c, (const double*)r, (double*)z, cfg.mg);
      }
    } else {
      if (c.mg_prec == 1) klaunch(k_bj_mixed<float, T>, g_nb(L.nnod), 256, 0, c.stream, c.mg[0].dinv32, r, z, L.nnod);
      else klaunch(k_bj_mixed<double, T>, g_nb(L.nnod), 256, 0, c.stream, c.mg[0].dinv64, r, z, L.nnod);
    }
    if (mixed)
      klaunch(k_rz_f32, red_grid(n), kRedThreads, 0, c.stream, (const float*)z32, (const double*)r, c.scal, YY, RZN, n,
              c.partial, c.counter);
    else if (f32) launch_dot_f(c, (const float*)r, (const float*)z, n, RZN);
    else launch_dot(c, (const double*)r, (const double*)z, n, RZN);
    if (mixed)
      klaunch(k_pcg_dir_f32z, g_nb(n), 256, 0, c.stream, (double*)p, (const float*)z32, (double*)Ap, n,
              (const double*)c.scal, YY, RZN, RZ, itp);
    else
      klaunch(k_pcg_dir_g<T>, g_nb(n), 256, 0, c.stream, p, z, Ap, n, c.scal, RZN, RZ, itp);
    launch_apply_K_acc<T, T>(L, Kmat, p, Ap, c.stream);
    if (f32) launch_dot_f(c, (const float*)p, (const float*)Ap, n, PAP);
    else launch_dot(c, (const double*)p, (const double*)Ap, n, PAP);
    klaunch(k_pcg_upd_check<T>, red_grid(n), kRedThreads, 0, c.stream, x, r, p, Ap, n, c.scal, RZ, RZN, PAP, IRR,
            c.partial, c.counter, h, ctl, f32 ? 1 : 0, mixed ? r32 : (float*)nullptr, YY);
    DP_LAUNCH_CHECK();
  });
}

// Inner solve K x = b (FP64 in/out) at capture depth `depth`.
static void emit_inner(Ctx& c, const SolveCfg& cfg, const double* b, double* x, int depth, int relax) {
  const int64_t n = 2 * c.fine.nnod;
  if (cfg.precision <= 1) {
    emit_pcg<double>(c, cfg, c.K64, b, x, (double*)c.work[W_IN_R], (double*)c.work[W_IN_Z], (double*)c.work[W_IN_P],
                     (double*)c.work[W_IN_AP], depth, relax);
    return;
  }
  DevCtl* ctl = (DevCtl*)c.ctl;
  double* res = (double*)c.work[W_RES];
  float* fb = (float*)c.work[W_F_B];
  float* fx = (float*)c.work[W_F_X];
  DP_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, c.stream));
  DP_CUDA(cudaMemcpyAsync(res, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  launch_dot(c, b, b, n, R_YY);
  cudaGraphConditionalHandle h = new_handle(c.stream);
  klaunch(k_ref_init, 1, 1, 0, c.stream, h, ctl, c.scal, relax);
  DP_LAUNCH_CHECK();
  cudaGraph_t body = add_while(c.stream, h);
  capture_body(c, body, depth, B_REF, [&] {
    klaunch(k_to_f32_scaled, g_nb(n), 256, 0, c.stream, res, fb, c.scal, n);
    emit_pcg<float>(c, cfg, c.K32, fb, fx, (float*)c.work[W_F_R], (float*)c.work[W_F_Z], (float*)c.work[W_F_P],
                    (float*)c.work[W_F_AP], depth + 1, 0);
    klaunch(k_add_f32_scaled, g_nb(n), 256, 0, c.stream, x, fx, c.scal, n);
    launch_apply_K<double, double>(c.fine, c.K64, x, res, c.stream);
    klaunch(k_residual, g_nb(n), 256, 0, c.stream, b, res, n);
    launch_dot(c, res, res, n, R_RES2);
    klaunch(k_ref_check, 1, 1, 0, c.stream, h, ctl, c.scal);
    DP_LAUNCH_CHECK();
  });
}

static void emit_solve(Ctx& c, const SolveCfg& cfg, double* U, double* P) {
  const Level& L = c.fine;
  const int64_t nU = 2 * L.nnod, nP = c.mesh.npres;
  double* r = (double*)c.work[W_R];
  double* rlast = (double*)c.work[W_RLAST];
  double* d = (double*)c.work[W_D];
  double* q = (double*)c.work[W_Q];
  double* y = (double*)c.work[W_Y];
  double* z = (double*)c.work[W_Z];
  double* Sq = (double*)c.work[W_SQ];
  double* rhs = (double*)c.work[W_RHS];
  DevCtl* ctl = (DevCtl*)c.ctl;
  DP_CUDA(cudaMemsetAsync(&ctl->in_total, 0, 3 * sizeof(long long), c.stream));
  if (cfg.use_guess == 2) {
    // zero-guess reference: Uz = K^-1 F, rz = -G^T Uz (mean removed), ||rz||
    double* Uz = (double*)c.work[W_UC];
    double* rz = (double*)c.work[W_RLAST];
    emit_inner(c, cfg, c.F, Uz, 0, 0);
    launch_apply_GT(c, Uz, rz);
    klaunch(k_neg, g_nb(nP), 256, 0, c.stream, rz, nP);
    launch_sum_c(c, rz, nP, S_SUMR);
    klaunch(k_sub_mean, g_nb(nP), 256, 0, c.stream, rz, nP, c.scal + S_SUMR);
    launch_dot_c(c, rz, rz, nP, G_RZREF);
  }
  // Rhs = F + G P ; U = K^-1 Rhs (tight inner tolerance) ; r = -G^T U ;
  // rm0space!(r) ; ||r||^2 -> S_RR.  The initial residual, and in the restart
  // mode the true residual after each pass of the outer loop.
  auto true_residual = [&](int depth) {
    launch_apply_G(c, P, y);
    klaunch(k_add, g_nb(nU), 256, 0, c.stream, c.F, y, rhs, nU);
    emit_inner(c, cfg, rhs, U, depth, 0);
    launch_apply_GT(c, U, r);
    klaunch(k_neg, g_nb(nP), 256, 0, c.stream, r, nP);
    launch_sum_c(c, r, nP, S_SUMR);
    klaunch(k_sub_mean, g_nb(nP), 256, 0, c.stream, r, nP, c.scal + S_SUMR);
    launch_dot_c(c, r, r, nP, S_RR);
  };
  // d = r .* pc (or M^-1 r) ; q = d
  auto pc_start = [&] {
    if (cfg.schur_pc == 1) {
      klaunch(k_mass_blk, g_nb(L.nel), 256, 0, c.stream, r, c.Minv, d, (int)L.nel);
    } else {
      klaunch(k_mul_into, g_nb(nP), 256, 0, c.stream, r, c.pc, d, nP);
    }
    DP_CUDA(cudaMemcpyAsync(q, d, sizeof(double) * nP, cudaMemcpyDeviceToDevice, c.stream));
    launch_sum_c(c, q, nP, S_SUMQ);
  };
  // the StokesPcCG iteration (IterativeSolvers.jl:130-166) as a WHILE body
  auto outer_body = [&](cudaGraphConditionalHandle h, int depth) {
    klaunch(k_q_center_rd, red_grid(nP), kRedThreads, 0, c.stream, q, r, d, nP, c.scal, c.partial, c.counter);
    launch_apply_G(c, q, y);
    emit_inner(c, cfg, y, z, depth + 1, cfg.inner_relax > 0.0 ? 1 : 0);
    launch_apply_GT(c, z, Sq);
    launch_dot_c(c, q, Sq, nP, S_QSQ);
    klaunch(k_schur_update_p, red_grid(nP), kRedThreads, 0, c.stream, P, r, rlast, q, Sq, nP, c.scal, c.partial,
            c.counter);
    klaunch(k_axpy_slot, g_nb(nU), 256, 0, c.stream, U, z, nU, c.scal);
    if (cfg.schur_pc == 1)
      klaunch(k_schur_center_blk, red_grid(L.nel), kRedThreads, 0, c.stream, r, rlast, c.Minv, d, (int)L.nel, c.scal,
              c.partial, c.counter);
    else
      klaunch(k_schur_center, red_grid(nP), kRedThreads, 0, c.stream, r, rlast, c.pc, d, nP, c.scal, c.partial,
              c.counter);
    klaunch(k_q_update, red_grid(nP), kRedThreads, 0, c.stream, q, d, nP, c.scal, c.partial, c.counter);
    klaunch(k_outer_check, 1, 1, 0, c.stream, h, ctl, c.scal);
    DP_LAUNCH_CHECK();
  };

  // Pressure gauge: constant pressure is in the null space of G under free slip,
  // so P is defined up to a constant.  StokesPcCG starts from P = 0 and adds
  // only mean-free directions (IterativeSolvers.jl:101, rm0space! of q), so its
  // P has zero mean; a given initial P (a guess) has its mean removed first so
  // that the answer carries the same gauge.  It changes nothing else (G 1 = 0).
  if (!cfg.use_guess) {
    DP_CUDA(cudaMemsetAsync(P, 0, sizeof(double) * nP, c.stream));
  } else {
    launch_sum_c(c, P, nP, S_TMP2);
    klaunch(k_sub_mean, g_nb(nP), 256, 0, c.stream, P, nP, (const double*)(c.scal + S_TMP2));
  }
  true_residual(0);
  if (cfg.use_guess == 2) {
    klaunch(k_guess_select, 1, 1, 0, c.stream, ctl, c.scal);
    klaunch(k_guess_apply, g_nb(std::max(nU, nP)), 256, 0, c.stream, ctl, U, (const double*)c.work[W_UC], r,
            (const double*)c.work[W_RLAST], P, nU, nP);
  }
  if (!cfg.true_residual) {
    pc_start();
    cudaGraphConditionalHandle h = new_handle(c.stream);
    klaunch(k_outer_init, 1, 1, 0, c.stream, h, ctl, c.scal, cfg.use_guess == 2 ? 1 : 0);
    DP_LAUNCH_CHECK();
    cudaGraph_t body = add_while(c.stream, h);
    capture_body(c, body, 0, B_OUTER, [&] { outer_body(h, 0); });
  } else {
    klaunch(k_outer_start, 1, 1, 0, c.stream, ctl, c.scal, cfg.use_guess == 2 ? 1 : 0);
    cudaGraphConditionalHandle hr = new_handle(c.stream);
    klaunch(k_restart_init, 1, 1, 0, c.stream, hr, ctl);
    DP_LAUNCH_CHECK();
    cudaGraph_t rbody = add_while(c.stream, hr);
    capture_body(c, rbody, 0, B_RESTART, [&] {
      pc_start();
      cudaGraphConditionalHandle h = new_handle(c.stream);
      klaunch(k_outer_resume, 1, 1, 0, c.stream, h, ctl, c.scal);
      DP_LAUNCH_CHECK();
      cudaGraph_t body = add_while(c.stream, h);
      capture_body(c, body, 1, B_OUTER, [&] { outer_body(h, 1); });
      true_residual(1);
      klaunch(k_restart_check, 1, 1, 0, c.stream, hr, ctl, c.scal);
      DP_LAUNCH_CHECK();
    });
  }
  // diagnostics on the raw solution
  launch_apply_K<double, double>(L, c.K64, U, rhs, c.stream);
  launch_apply_G(c, P, y);
  klaunch(k_add, g_nb(nU), 256, 0, c.stream, c.F, y, y, nU);
  klaunch(k_residual, g_nb(nU), 256, 0, c.stream, y, rhs, nU);
  launch_dot(c, rhs, rhs, nU, S_TMP);
  launch_dot(c, c.F, c.F, nU, S_TMP2);
  launch_apply_GT(c, U, Sq);
  launch_sum_c(c, Sq, nP, S_SUMR);
  klaunch(k_sub_mean, g_nb(nP), 256, 0, c.stream, Sq, nP, c.scal + S_SUMR);
  launch_dot_c(c, Sq, Sq, nP, G_TMP3);
  if (cfg.remove_rotation) {
    klaunch(k_rot_integrals, red_grid(L.nel), kRedThreads, 0, c.stream, U, c.rho_lat, c.theta_lat, c.r_lat, (int)L.nel, L.ncr,
                                                                   (int)L.A(), (int)L.B(), c.scal, c.partial, c.counter);
    klaunch(k_rot_remove, g_nb(L.nnod), 256, 0, c.stream, U, c.r_lat, L.nnod, c.scal);
  }
  DP_LAUNCH_CHECK();
}

static int64_t graph_key(const SolveCfg& cfg, const Ctx& c) {
  return (int64_t)cfg.precision | ((int64_t)cfg.inner_pc << 2) | ((int64_t)cfg.use_guess << 3) |
         ((int64_t)cfg.remove_rotation << 5) | ((int64_t)c.mg_degree << 40) | ((int64_t)c.mg.size() << 10) |
         ((int64_t)(cfg.inner_relax > 0.0) << 15) | ((int64_t)c.mg_prec << 16) | ((int64_t)cfg.schur_pc << 18) |
         ((int64_t)cfg.mg.block_jacobi << 20) | ((int64_t)(c.coarse_n > 0) << 21) |
         ((int64_t)cfg.mg.apply_warps << 24) | ((int64_t)cfg.mg.apply_warps_t << 28) |
         ((int64_t)cfg.launch_overlap << 32) | ((int64_t)tail_start(c, cfg.mg) << 33) |
         ((int64_t)cfg.matrix_free << 37) |
         ((int64_t)cfg.true_residual << 38) | ((int64_t)(c.fine.det != nullptr) << 39);
}

void graph_free(Ctx& c) {
  if (c.gexec) cudaGraphExecDestroy((cudaGraphExec_t)c.gexec);
  if (c.graph) cudaGraphDestroy((cudaGraph_t)c.graph);
  c.gexec = nullptr;
  c.graph = nullptr;
  c.gkey = -1;
}

static void ensure_ctl(Ctx& c) {
  if (!c.ctl) {
    DP_CUDA(cudaMalloc(&c.ctl, sizeof(DevCtl)));
    DP_CUDA(cudaMallocHost(&c.h_ctl, sizeof(DevCtl)));
    for (int i = 0; i < 4; ++i) DP_CUDA(cudaStreamCreateWithFlags(&c.aux[i], cudaStreamNonBlocking));
  }
}

// The graph-only vector kernels of one inner iteration (FP64 Krylov, FP32
// multigrid) launched once each outside a graph, without loop control: the
// scaled FP32 residual (before the loop), r.z from z32, the direction update
// from z32 and the fused x/r update with ||r||^2 and the next FP32 residual.
// Profilers cannot look inside conditional graph nodes; this is what they time
// instead.  Vector contents are zeroed and the scalars set to 1, so every value
// stays finite.
void profile_inner_vector_kernels(Ctx& c) {
  ensure_ctl(c);
  const int64_t n = 2 * c.fine.nnod;
  double* x = (double*)c.work[W_Z];
  double* r = (double*)c.work[W_IN_R];
  double* z = (double*)c.work[W_IN_Z];
  double* p = (double*)c.work[W_IN_P];
  double* Ap = (double*)c.work[W_IN_AP];
  float* r32 = (float*)c.work[W_F_R];
  float* z32 = (float*)c.work[W_F_Z];
  DevCtl* ctl = (DevCtl*)c.ctl;
  for (double* v : {x, r, z, p, Ap}) DP_CUDA(cudaMemsetAsync(v, 0, sizeof(double) * n, c.stream));
  DP_CUDA(cudaMemsetAsync(r32, 0, sizeof(float) * n, c.stream));
  DP_CUDA(cudaMemsetAsync(z32, 0, sizeof(float) * n, c.stream));
  DP_CUDA(cudaMemsetAsync(&ctl->in_it, 0, sizeof(int), c.stream));
  for (int k = 0; k < 4; ++k) c.h_scal[48 + k] = 1.0;
  DP_CUDA(cudaMemcpyAsync(c.scal + G_RZ, c.h_scal + 48, 4 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  DP_CUDA(cudaStreamSynchronize(c.stream));
  klaunch(k_r_to_f32, g_nb(n), 256, 0, c.stream, (const double*)r, r32, c.scal, (int)G_IRR, n);
  klaunch(k_rz_f32, red_grid(n), kRedThreads, 0, c.stream, (const float*)z32, (const double*)r, c.scal, (int)G_IRR,
          (int)G_RZN, n, c.partial, c.counter);
  klaunch(k_pcg_dir_f32z, g_nb(n), 256, 0, c.stream, p, (const float*)z32, Ap, n, (const double*)c.scal, (int)G_IRR,
          (int)G_RZN, (int)G_RZ, (const int*)&ctl->in_it);
  klaunch(k_pcg_upd_check<double>, red_grid(n), kRedThreads, 0, c.stream, x, r, (const double*)p,
          (const double*)Ap, n, c.scal, (int)G_RZ, (int)G_RZN, (int)G_PAP, (int)G_IRR, c.partial, c.counter,
          (cudaGraphConditionalHandle)0, (DevCtl*)nullptr, 0, r32, (int)G_IRR);
  DP_LAUNCH_CHECK();
}

// Captures the solve of c (on c.stream, which may be part of an enclosing
// capture) and records its kernel-count bookkeeping.
static void capture_solve(Ctx& c, const SolveCfg& cfg, double* U, double* P) {
  PdlScope pdl(cfg.launch_overlap);
  const int64_t start = g_klaunch;
  c.cap_nested = 0;
  emit_solve(c, cfg, U, P);
  c.gk_main = (g_klaunch - start) - c.cap_nested;
}

static void upload_params(Ctx& c, const SolveCfg& cfg, cudaStream_t s) {
  DevCtl h{};
  h.rtol = cfg.rtol;
  h.inner_rtol = cfg.inner_rtol;
  h.inner_rtol32 = cfg.inner_rtol32;
  h.relax_cap = cfg.inner_relax;
  h.relax_base = cfg.relax_base;
  h.itmax = cfg.itmax;
  h.itmin = cfg.itmin;
  h.inner_itmax = cfg.inner_itmax;
  h.max_refine = cfg.max_refine;
  h.max_restarts = cfg.max_restarts;
  *(DevCtl*)c.h_ctl = h;
  DP_CUDA(cudaMemcpyAsync(c.ctl, c.h_ctl, sizeof(DevCtl), cudaMemcpyHostToDevice, s));
}

// Reads the device control block and scalars of a finished solve (synchronises s).
static void collect_result(Ctx& c, const SolveCfg& cfg, cudaStream_t s, SolveResult& res) {
  DP_CUDA(cudaMemcpyAsync(c.h_ctl, c.ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, s));
  DP_CUDA(cudaMemcpyAsync(c.h_scal, c.scal, sizeof(double) * 32, cudaMemcpyDeviceToHost, s));
  DP_CUDA(cudaStreamSynchronize(s));
  const DevCtl& o = *(const DevCtl*)c.h_ctl;
  res.status = o.status;
  res.iterations = o.outer_it;
  res.r0 = o.r0;
  res.relres = o.r0 > 0 ? std::sqrt(c.h_scal[S_RR]) / o.r0 : 0.0;
  res.mom_residual = std::sqrt(c.h_scal[S_TMP] / std::max(c.h_scal[S_TMP2], 1e-300));
  res.div_residual = o.r0 > 0 ? std::sqrt(c.h_scal[G_TMP3]) / o.r0 : 0.0;
  res.omega = cfg.remove_rotation ? c.h_scal[S_AM] / c.h_scal[S_MOM] : 0.0;
  res.inner_its = cfg.precision == 2 ? o.in32_total : o.in_total;
  res.launches = c.gk_main + c.gk_body[B_OUTER] * o.outer_it + c.gk_body[B_PCG64] * o.in_total +
                 c.gk_body[B_PCG32] * o.in32_total + c.gk_body[B_REF] * o.ref_total +
                 (cfg.true_residual ? c.gk_body[B_RESTART] * o.restarts : 0);
  res.restarts = cfg.true_residual ? o.restarts : 1;
  res.refinements = o.ref_total;
  res.fallback = (cfg.use_guess == 2) ? (o.guess_used ? 0 : 1) : 0;
  res.r0_guess = o.r0guess;
}

int schur_pcg_graph(Ctx& c, const SolveCfg& cfg, double* U, double* P, SolveResult& res) {
  ensure_ctl(c);
  const int64_t key = graph_key(cfg, c);
  if (!c.gexec || c.gkey != key || c.gU != U || c.gP != P || c.ggen != c.alloc_gen) {
    graph_free(c);
    DP_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
    try {
      capture_solve(c, cfg, U, P);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c.stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    cudaGraph_t g = nullptr;
    DP_CUDA(cudaStreamEndCapture(c.stream, &g));
    cudaGraphExec_t ex = nullptr;
    DP_CUDA(cudaGraphInstantiate(&ex, g, 0));
    c.graph = g;
    c.gexec = ex;
    c.gkey = key;
    c.gU = U;
    c.gP = P;
    c.ggen = c.alloc_gen;
  }
  upload_params(c, cfg, c.stream);
  DP_CUDA(cudaGraphLaunch((cudaGraphExec_t)c.gexec, c.stream));
  collect_result(c, cfg, c.stream, res);
  return res.status;
}

// ---- batches: independent solves of several contexts in ONE graph launch ------------
// The graph is captured with a fork/join over the contexts' streams: one branch per
// context holds that context's whole solve (its own WHILE nodes and device control
// block).  An external event-record node at the end of each branch timestamps its
// completion; a second (capture-internal) event joins the branch back.
struct Batch {
  std::vector<Ctx*> ctx;
  std::vector<SolveCfg> cfg;
  std::vector<int64_t> gen;   // each context's allocation generation at capture
  int priorities = 1;          // kernel priorities by problem size
  cudaStream_t s = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t fork = nullptr, start = nullptr;
  std::vector<cudaEvent_t> done, join;
  std::string err;
  void free_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  ~Batch() {
    free_graph();
    for (cudaEvent_t e : done) cudaEventDestroy(e);
    for (cudaEvent_t e : join) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (start) cudaEventDestroy(start);
    if (s) cudaStreamDestroy(s);
  }
};

void batch_build(Batch& b) {
  if (!b.s) {
    DP_CUDA(cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking));
    DP_CUDA(cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming));
    DP_CUDA(cudaEventCreate(&b.start));
    b.done.resize(b.ctx.size());
    b.join.resize(b.ctx.size());
    for (auto& e : b.done) DP_CUDA(cudaEventCreate(&e));
    for (auto& e : b.join) DP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  b.free_graph();
  b.gen.clear();
  for (Ctx* c : b.ctx) {
    ensure_ctl(*c);
    b.gen.push_back(c->alloc_gen);
  }
  // kernel priorities: the smaller a problem, the higher its priority, so the
  // small solves finish early and the large ones fill the remaining SMs
  int least = 0, greatest = 0;
  DP_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  std::vector<int64_t> sizes;
  for (Ctx* c : b.ctx) sizes.push_back(c->fine.nel);
  std::vector<int64_t> distinct = sizes;
  std::sort(distinct.begin(), distinct.end());
  distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
  const int levels = least - greatest;  // number of priority steps (greatest is numerically lowest)
  DP_CUDA(cudaStreamBeginCapture(b.s, cudaStreamCaptureModeRelaxed));
  try {
    DP_CUDA(cudaEventRecord(b.fork, b.s));
    for (size_t i = 0; i < b.ctx.size(); ++i) {
      Ctx& c = *b.ctx[i];
      DP_CUDA(cudaStreamWaitEvent(c.stream, b.fork, 0));
      const int rank = (int)(std::lower_bound(distinct.begin(), distinct.end(), sizes[i]) - distinct.begin());
      const int steps = (int)distinct.size() > 1 ? (int)distinct.size() - 1 : 1;
      g_prio = b.priorities ? greatest + (levels * rank) / steps : kNoPriority;
      capture_solve(c, b.cfg[i], (double*)c.work[W_U], (double*)c.work[W_P]);
      g_prio = kNoPriority;
      DP_CUDA(cudaEventRecordWithFlags(b.done[i], c.stream, cudaEventRecordExternal));
      DP_CUDA(cudaEventRecord(b.join[i], c.stream));
      DP_CUDA(cudaStreamWaitEvent(b.s, b.join[i], 0));
    }
  } catch (...) {
    g_prio = kNoPriority;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(b.s, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  DP_CUDA(cudaStreamEndCapture(b.s, &b.graph));
  DP_CUDA(cudaGraphInstantiate(&b.exec, b.graph, b.priorities ? cudaGraphInstantiateFlagUseNodePriority : 0));
  DP_CUDA(cudaGraphUpload(b.exec, b.s));
}

// Launches the batch once; per-context results and completion times (ms from launch).
// The graph holds the contexts' buffer addresses: a context whose multigrid or FP32
// operator storage was reallocated since the capture (another precision or coarse
// size solved on it meanwhile) makes the batch capture again first.
void batch_run(Batch& b, std::vector<SolveResult>& res, std::vector<double>& done_ms) {
  for (size_t i = 0; i < b.ctx.size(); ++i)
    if (b.ctx[i]->alloc_gen != b.gen[i]) {
      batch_build(b);
      break;
    }
  for (size_t i = 0; i < b.ctx.size(); ++i) upload_params(*b.ctx[i], b.cfg[i], b.s);
  DP_CUDA(cudaEventRecord(b.start, b.s));
  DP_CUDA(cudaGraphLaunch(b.exec, b.s));
  DP_CUDA(cudaStreamSynchronize(b.s));
  res.resize(b.ctx.size());
  done_ms.resize(b.ctx.size());
  for (size_t i = 0; i < b.ctx.size(); ++i) {
    collect_result(*b.ctx[i], b.cfg[i], b.s, res[i]);
    float ms = 0.f;
    DP_CUDA(cudaEventElapsedTime(&ms, b.start, b.done[i]));
    done_ms[i] = ms;
  }
}

}  // namespace dp
