// Solver configuration and work-vector layout.
#pragma once
#include "ctx.cuh"
#include "mg.cuh"

namespace dp {

struct SolveCfg {
  double rtol = 1e-8;       // outer (IterativeSolvers.jl:95)
  int itmax = 200;          // outer (:96)
  int itmin = 10;           // outer (:97)
  int precision = 0;        // 0 FP64; 1 FP64 Krylov + FP32 hierarchy; 2 FP32 PCG in FP64 refinement
  int inner_pc = 0;         // 0 multigrid, 1 Jacobi
  double inner_rtol = 1e-10;
  double inner_rtol32 = 1e-5;
  int inner_itmax = 500;
  int max_refine = 6;
  int remove_rotation = 1;
  int use_guess = 0;        // 0 zero guess; 1 warm start from P; 2 learned guess with fallback
  int verbose = 0;
  int host_loop = 0;        // 1: host-driven loops (debug); 0: one CUDA graph per solve
  double inner_relax = 0.0; // > 0: relaxed inner tolerance with this cap
  double relax_base = 0.0;  // base of the relaxation (0: inner_rtol)
  int schur_pc = 0;         // 0 lumped mass (StokesPcCG), 1 element-block mass inverse
  int launch_overlap = 1;   // 1: programmatic dependent launch between solver kernels
  int matrix_free = 0;      // 1: fine-level applies from the rotated tensors (no element matrices)
  int true_residual = 1;    // 1: outer loop restarted until the true Schur residual meets rtol
  int max_restarts = 4;
  MGOptions mg;
};

// Sets g_pdl for the kernels launched in its scope (solve capture or host loop).
struct PdlScope {
  int saved;
  explicit PdlScope(int on) : saved(g_pdl) { g_pdl = on; }
  ~PdlScope() { g_pdl = saved; }
};

struct InnerStats {
  int64_t its = 0;
  double last_relres = 0.0;
};

struct SolveResult {
  int status = 0;
  int iterations = 0;
  int64_t inner_its = 0;
  int64_t launches = 0;       // kernels launched by the solve
  int64_t refinements = 0;    // FP64 refinement steps (FP32-refined path)
  int fallback = 0;           // learned guess rejected
  double r0_guess = 0.0;      // ||r(P0)|| of the guess
  int restarts = 0;           // passes of the outer loop in the true-residual mode
  double relres = 0.0, r0 = 0.0, omega = 0.0, div_residual = 0.0, mom_residual = 0.0;
};

// indices into Ctx::work
enum Work {
  W_R = 0, W_RLAST, W_D, W_Q, W_SQ,                 // pressure-sized (FP64)
  W_Y, W_Z, W_RHS, W_IN_R, W_IN_Z, W_IN_P, W_IN_AP, W_RES,   // velocity-sized (FP64)
  W_F_B, W_F_X, W_F_R, W_F_Z, W_F_P, W_F_AP,        // velocity-sized (FP32)
  W_U, W_P, W_UC,                                   // solution staging (FP64)
  W_COUNT
};

int inner_solve(Ctx& c, const double* y, double* z, const SolveCfg& cfg, InnerStats& st);
int schur_pcg(Ctx& c, const SolveCfg& cfg, double* U, double* P, SolveResult& res);
void to_cartesian(Ctx& c, const double* U, double* Uc);
int schur_pcg_graph(Ctx& c, const SolveCfg& cfg, double* U, double* P, SolveResult& res);
void graph_free(Ctx& c);
void profile_inner_vector_kernels(Ctx& c);

}  // namespace dp
