/*
 * dimspers_b200 -- C ABI of the B200 Stokes hot path (P2-P1 annulus assembly
 * and Schur-complement PCG) of DimsPers / Persephone.
 *
 * Every entry point returns a status code (dp_status) and never exits or
 * aborts.  Host arrays are borrowed for the duration of a call.  Device
 * buffers are owned by the context.  Index arrays crossing the ABI are
 * 1-based and column-major as Julia stores them.  One context per host
 * thread; calls are synchronous to the caller (stream-ordered inside).
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   solveStokes                src/Stokes/StokesSolver.jl:7-54
 *   assembly_stokes_cylindric  src/Stokes/StokesSolver.jl:247-404
 *   _prepare_matrices          src/Stokes/StokesSolver.jl:192-201
 *   _apply_bcs                 src/Stokes/StokesSolver.jl:186-190
 *   StokesPcCG                 src/IterativeSolvers.jl:94-168
 *   updatevelocity2            src/Stokes/StokesSolver.jl:170-184
 *   Grid_split1 / color_mesh   src/Grid/mesher.jl:152-233, src/Grid/coloring.jl:5-64
 */
#ifndef DIMSPERS_B200_H
#define DIMSPERS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DP_OK = 0,
  DP_NOT_CONVERGED = 1,  /* outer itmax reached (the reference returns silently) */
  DP_BREAKDOWN = 2,      /* q.Sq <= 0 or a non-finite scalar in the PCG        */
  DP_BAD_ARG = 3,
  DP_CUDA_ERROR = 4,
  DP_DEVICE_TIMEOUT = 5
} dp_status;

typedef enum { DP_PRESSURE_CONTINUOUS = 0, DP_PRESSURE_DISCONTINUOUS = 1 } dp_pressure_space;
/* FP64: all in FP64.  FP32_REFINED: FP32 element matrices and FP32 multigrid
 * (the bulk of the applies) preconditioning an FP64 Krylov solve whose
 * residual, updates and dot products stay FP64.  FP32_IR: classic iterative
 * refinement, an FP32 PCG inside an FP64 residual / correction loop. */
typedef enum { DP_PREC_FP64 = 0, DP_PREC_FP32_REFINED = 1, DP_PREC_FP32_IR = 2 } dp_precision;
typedef enum { DP_MEM_HOST = 0, DP_MEM_DEVICE = 1 } dp_memory;
typedef enum { DP_INNER_MG = 0, DP_INNER_JACOBI = 1 } dp_inner_pc;

/* Mesh description.  Cells, not nodes: the reference's init_grid/Grid_split1
 * take node counts (nr = cells + 1, ntheta = cells). */
typedef struct {
  int32_t nr_cells;        /* radial cells (>= 1)                              */
  int32_t ntheta_cells;    /* angular cells (>= 3)                             */
  double r_in, r_out;      /* radii (1.22, 2.22 in the reference)              */
  int32_t pressure_space;  /* dp_pressure_space                               */
  int32_t device;          /* CUDA device ordinal                             */
  int32_t pin_rotation;    /* 1: also fix u_theta of the outer-wall node at
                              theta = 0 (free_slip(nr, ids),
                              boundary_conditions.jl:180-194), which removes the
                              rigid-rotation near-null mode of K; 0: the plain
                              free_slip(ids) of MAIN.jl                         */
} dp_mesh_desc;

typedef struct {
  double rtol;             /* outer relative tolerance (reference: 1e-8)      */
  int32_t itmax;           /* outer iteration cap (reference: 200)            */
  int32_t itmin;           /* outer minimum iterations (reference: 10)        */
  int32_t precision;       /* dp_precision                                    */
  int32_t inner_pc;        /* dp_inner_pc                                     */
  double inner_rtol;       /* inner K-solve relative tolerance                */
  int32_t inner_itmax;     /* inner iteration cap                             */
  int32_t remove_rotation; /* apply updatevelocity2's rigid-rotation removal  */
  int32_t use_guess;       /* 0: P = 0 (StokesPcCG); 1: warm start from the P
                              passed in, tolerance relative to its own r0 (as
                              StokesPcCG_pardiso keeps U, P); 2: learned guess:
                              start from the P passed in only if its Schur
                              residual is below the zero guess's, and stop at
                              rtol relative to the zero-guess residual.  A
                              given P has its mean removed first: pressure is
                              defined up to a constant here, and StokesPcCG's
                              answer (from P = 0) has zero mean             */
  int32_t verbose;
  int32_t cheb_degree;     /* Chebyshev smoothing steps per level             */
  double inner_rtol32;     /* FP32 inner tolerance per refinement step        */
  int32_t max_refine;      /* FP32-refined: refinement steps per inner solve  */
  int32_t host_loop;       /* 1: drive the loops from the host (debugging);
                              0: the whole solve is one CUDA graph with
                              device-side loop control                        */
  int32_t block_jacobi;    /* smoother: 1 = 2x2 nodal blocks, 0 = point Jacobi */
  double cheb_lo, cheb_hi; /* Chebyshev interval as fractions of lambda_max  */
  double inner_relax;      /* > 0: relax the inner tolerance as the outer
                              residual falls, inner_rtol * ||r0|| / ||r_k||,
                              capped at this value; 0: fixed inner_rtol       */
  int32_t coarse_max;      /* largest coarsest-level system solved densely    */
  int32_t schur_pc;        /* Schur preconditioner: 0 = 1/rowsum(M), the lumped
                              mass of StokesPcCG (IterativeSolvers.jl:120,238);
                              1 = M^-1 from the element mass blocks, what the
                              incomplete LDL^T of StokesPcCG_pardiso (:32,242)
                              gives for block-diagonal (discontinuous) M      */
  int32_t apply_warps;     /* CTA of the element-by-element K applies, in warps
                              (1, 2, 4, 8; 0 = default 4)                     */
  int32_t apply_warps_t;   /* of those, warps stacked along theta (1 = linear
                              element order; 0 = default 1)                   */
  int32_t launch_overlap;  /* 1 = each solver kernel may launch while its
                              predecessor runs (programmatic dependent launch;
                              default), 0 = plain stream order               */
  int32_t mg_tail;         /* > 0: multigrid levels of at most this many
                              elements run as one thread-block-cluster kernel
                              (0 = off, the default: on B200 a cluster phase
                              costs about as much as a kernel launch)        */
  int32_t matrix_free;     /* 1 = fine-level K applies computed from the
                              element's rotated viscous tensor at the IPs and
                              per-ring reference shape derivatives (144 B per
                              element read instead of 312; slower on B200, where
                              the packed apply runs near HBM peak), 0 = packed
                              element matrices (default)                      */
  int32_t cheb_degree_coarse; /* Chebyshev degree on the levels below the
                              finest (0 = cheb_degree)                        */
  int32_t true_residual;   /* 1 (default): when the outer loop stops, U is
                              solved afresh, U = K^-1 (F + G P), and the loop
                              restarts from P until the TRUE residual
                              ||G^T U|| meets rtol (needed with inner_relax,
                              where the recursive residual drifts); 0: stop on
                              the recursive residual as StokesPcCG does      */
  double relax_base;       /* with inner_relax > 0: inner tolerance of outer
                              iteration k = min(inner_relax, max(inner_rtol,
                              relax_base * ||r0|| / ||r_k||)); 0 = inner_rtol.
                              The initial and true-residual solves keep
                              inner_rtol.                                     */
} dp_solve_opts;

typedef struct {
  int32_t status;
  int32_t iterations;          /* outer (Schur) iterations                    */
  int64_t inner_iterations;    /* total inner K-solve iterations              */
  double relres;               /* final outer ||r|| / ||r0|| (reference measure) */
  double r0;                   /* ||r0||                                       */
  double omega;                /* removed rigid angular velocity              */
  double div_residual;         /* ||G^T U|| / ||G^T U0||                       */
  double mom_residual;         /* ||K U - F - G P|| / ||F|| on free DOFs       */
  double t_assemble_ms, t_setup_ms, t_solve_ms;
  int32_t fallback_used;       /* learned guess rejected -> zero guess        */
  int32_t mg_levels;
  int64_t kernel_launches;     /* kernels this library launched for the solve */
  int64_t refinements;         /* FP64 refinement steps (FP32-refined path)   */
  double r0_guess;             /* use_guess = 2: ||r(P0)|| of the guess; r0 is then
                                  the zero-guess residual                     */
  int32_t restarts;            /* passes of the outer loop (true_residual = 1)  */
} dp_solve_report;

typedef struct dp_ctx dp_ctx;

/* ---- host-only queries (no GPU needed) --------------------------------- */

/* Sizes of the split-1 P2 mesh (mesher.jl:152-233). */
int dp_mesh_sizes(const dp_mesh_desc* desc, int64_t* nel, int64_t* nnod,
                  int64_t* npres, int64_t* nfixed);

/* Build the mesh on the host in the reference's numbering:
 *   e2n     6 x nel, column-major, 1-based  (gr.e2n, mesher.jl:202-204)
 *   theta,r nnod                            (gr.theta, gr.r incl. midpoints)
 *   colors  nel, 1-based greedy colours     (color_mesh, coloring.jl:5-64)
 *   ncolors number of colours
 * Any output pointer may be NULL. */
int dp_mesh_build(const dp_mesh_desc* desc, int64_t* e2n, double* theta, double* r,
                  int32_t* colors, int32_t* ncolors);

/* Free-slip constraint set (boundary_conditions.jl:15-37): Omega (1-based
 * DOFs 2*node of wall nodes, top then bottom) and its count. */
int dp_mesh_free_slip(const dp_mesh_desc* desc, int64_t* omega, int64_t* nomega);

const char* dp_status_string(int status);

/* ---- context ------------------------------------------------------------ */

int dp_ctx_create(const dp_mesh_desc* desc, dp_ctx** out);
void dp_ctx_destroy(dp_ctx* ctx);
const char* dp_last_error(const dp_ctx* ctx);
/* cudaStream_t the context launches on (as void*). */
void* dp_ctx_stream(dp_ctx* ctx);
int dp_get_connectivity(dp_ctx* ctx, int64_t* e2n, int32_t* colors);

/* Material inputs in the reference layouts:
 *   eta_ip   nel x ld columns, element-fastest (eta.ip; IPs 1..6 read)
 *   C6       NULL (isotropic) or 6 pointers in StiffnessTensor order
 *            (C11, C33, C55, C13, C15, C35), each nel x ld_C element-fastest
 *   rho_node nnod nodal density (vertices enter the body force)
 *   g        gravity factor (body force g*rho*r_hat)
 * mem = dp_memory of every pointer. */
int dp_set_material(dp_ctx* ctx, const double* eta_ip, int64_t ld_eta,
                    const double* const* C6, int64_t ld_C, const double* rho_node,
                    double g, int32_t mem);

/* Transversely isotropic material: per-element delta (weak-plane shear
 * viscosity eta/delta) and director (dir_x, dir_y); the tensor is the frame
 * tensor a = c = 4/3, h = -2/3, e = 1/delta rotated on the device as in
 * directRotation2D (anisotropy.jl:503-536). */
int dp_set_material_ti(dp_ctx* ctx, const double* eta_ip, int64_t ld_eta,
                       const double* delta, const double* dir_x, const double* dir_y,
                       const double* rho_node, double g, int32_t mem);

/* Director = major eigenvector of F F^T per element (FSE.jl:143-161).
 * F is 4 x nel column-major (F11, F21, F12, F22 as a Julia 2x2 per element). */
int dp_fse_director(dp_ctx* ctx, const double* F, double* dir_x, double* dir_y, int32_t mem);

/* Element assembly + rotation + BC mask on the device (precision: dp_precision). */
int dp_assemble(dp_ctx* ctx, int32_t precision);

/* Deterministic mode (on = 1): every scatter of the solve path (the K and G
 * applies in FP32 and FP64, the right-hand side, the multigrid diagonal blocks
 * and the dense coarsest matrix) runs without atomics, as element results
 * summed per node in a fixed order, so repeated solves of the same inputs give
 * the same U, P and iteration counts bit for bit.  Costs 144 bytes of device
 * scratch per element and two passes per apply.  Needs discontinuous
 * pressure and matrix_free = 0.  Switching it on discards the current assembly
 * (call dp_assemble again); on = 0 returns to the atomic scatter.  A dp_batch
 * created from this context before a switch keeps the launches it captured:
 * create the batch again after switching.  (The
 * reference's threaded assembly gets race freedom from element colouring,
 * coloring.jl:1-64; the atomic device scatter has none of its ordering.) */
int dp_set_deterministic(dp_ctx* ctx, int32_t on);

/* Copy the un-rotated Cartesian element blocks in the reference layouts
 * (K_all 78 x nel, G_all 36 x nel, M_all 6 x nel, Fb_all 12 x nel, column-major).
 * Any pointer may be NULL. */
int dp_get_element_matrices(dp_ctx* ctx, double* Ke, double* Ge, double* Me, double* Fb);

/* Full solve: StokesPcCG + optional rigid-rotation removal.  U (2*nnod,
 * interleaved [u_theta, u_r] per node, reference numbering) and P (npres)
 * are overwritten; Ucart (2*nnod, may be NULL) receives TT*U. */
int dp_solve(dp_ctx* ctx, double* U, double* P, double* Ucart, const dp_solve_opts* opts,
             dp_solve_report* report, int32_t mem);

/* Operator applies for testing, on polar (rotated) DOFs in reference numbering:
 * y = K x (free DOFs, fixed rows zero), yG = G p, pG = G^T x. */
int dp_apply_K(dp_ctx* ctx, const double* x, double* y, int32_t mem);
int dp_apply_G(dp_ctx* ctx, const double* p, double* y, int32_t mem);
int dp_apply_GT(dp_ctx* ctx, const double* x, double* p, int32_t mem);
/* The deterministic reductions of the solver, on caller vectors of length n
 * (host or device per mem): op 0 = sum a_i b_i, 1 = the same compensated
 * (double-double accumulation, the Schur-complement loop's dots), 2 = sum a_i,
 * 3 = the same compensated (the loop's means).  Replaces mydot/mynorm and the
 * sums of vmean (src/Algebra/Algebra.jl:104-113, src/IterativeSolvers.jl:
 * 172-186), which the reference computes in plain FP64. */
int dp_reduce(dp_ctx* ctx, const double* a, const double* b, int64_t n, int32_t op, double* out, int32_t mem);
/* Assembled right-hand side (polar, reference numbering) and lumped pressure
 * preconditioner 1/rowsum(M). */
int dp_get_rhs(dp_ctx* ctx, double* F, double* pc);

void dp_default_opts(dp_solve_opts* opts);

/* y = K x like dp_apply_K, for callers that cannot allocate device memory:
 * hosts whose device memory is owned by their own pool or allocator, which the
 * library must not bypass, and real-time loops that forbid allocation after
 * start-up (cudaMalloc/cudaFree can synchronise the device and take unbounded
 * time).  No counterpart in the reference.  x and y are DEVICE pointers
 * (2*nnod, reference numbering); the two staging vectors live in one static
 * 32 MiB device array of the library, so nnod <= 1,048,576 (larger meshes:
 * DP_BAD_ARG).  No cudaMalloc/cudaFree is called.  The call runs on the
 * context's stream and returns when that stream has finished it, so the
 * caller must have finished writing x (and any reading of y) beforehand, e.g.
 * by synchronising its own stream.  All calls on a device share that array:
 * calls that overlap on the GPU race.  The first call on a device looks up the
 * array's address; make it before any stream capture begins. */
int dp_apply_K_noalloc(dp_ctx* ctx, const double* x, double* y);

/* ---- strain-rate / stress post-processor --------------------------------
 * stress! (src/Stress/StressCalculation.jl:23-249; MAIN.jl:241-243): per
 * element and 7-point IP (Quadrature.jl:109-138), the strain rate of the
 * Cartesian velocity Ucart (interleaved [ux, uz], reference numbering), its
 * second invariant, the deviatoric stress (isotropic eta, or the tensor fields
 * C6 in StiffnessTensor order with the reference's anisotropic formula) and
 * its second invariant.  eta_ip and the C6 fields: nel x ld element-fastest
 * (columns 1..7 read).  out: 8 matrices nel x 7 (element fastest), in the
 * order eps.xx, eps.zz, eps.xz, epsII, tau.xx, tau.zz, tau.xz, tauII. */
int dp_stress(dp_ctx* ctx, const double* Ucart, const double* eta_ip, int64_t ld_eta,
              const double* const* C6, int64_t ld_C, double* out, int32_t mem);

/* ---- per-IP viscosity update (Arrhenius law, Drucker-Prager plasticity) --
 * getviscosity!(::Arrhenius, ...) (src/Rheology/Rheology.jl:348-403; law
 * :60-97, :171-173): at the 7-point IPs, eta = clamp(lambda(z) eta0 exp((Ea +
 * P Va)/(R T) - Ea/(R T0)), 1e18, 1e25) with T and z = r by P2 interpolation
 * and P by linear interpolation of the vertex pressure plus |min P|; where
 * cohesion, phi and epsII are non-zero, eta = clamp(tau_y / (2 epsII), 1e18,
 * 1e25) if tau_y = cosd(phi) C + sind(phi) P < tauII, else unchanged.
 * T_node, r_node: nnod (reference numbering); P_vertex: the nvert vertex
 * values; epsII, tauII, cohesion, eta_ip (in/out): nel x 7 element-fastest. */
typedef struct {
  double eta0, R, Ea, Va, T0, phi_deg;
} dp_arrhenius;
int dp_viscosity_arrhenius(dp_ctx* ctx, const dp_arrhenius* law, const double* T_node, const double* P_vertex,
                           int64_t nvert, const double* r_node, const double* epsII, const double* tauII,
                           const double* cohesion, double* eta_ip, int32_t mem);

/* ---- per-IP finite-strain ellipsoid and DEM viscous tensor ---------------
 * dp_fse: getFSE / _FSE (src/Stress/FSE.jl:131-161) at every IP: from the
 * deformation gradient F (nel x 6 Julia SMatrix{2,2} per IP: F11, F21, F12,
 * F22 at ((ip * nel) + e) * 4) to fse = {vx1, vx2, vy1, vy2, a1, a2}, each
 * nel x ld_out element-fastest (columns 1..6 written): the major and minor
 * eigenvectors of F F^T and the square roots of its eigenvalues.  The signs
 * of the eigenvectors are not significant (the tensor depends on products of
 * pairs of components only).
 *
 * dp_anisotropic_tensor: anisotropic_tensor (src/Rheology/anisotropy.jl:
 * 140-285): per IP 1..6 the nearest row of the DEM table (argminsorted over
 * a1a2_blk for the fabric shape r1 and over the sorted a2a3_blk for r2, row
 * sblk (i1 - 1) + permutation_blk[i2]), its C11, C33, max(C55, w), C13 rotated
 * by the FSE axis (vx1, vy1) with directRotation2D, eta55 floored at w; IP 7 =
 * the mean of IPs 1..6.  vx1, vy1, r1, r2: nel x ld_in (columns 1..6 read);
 * r1 = log10(a1/a2), r2 = log10(a2/a3) of the inclusion shape, as Fabrics.jl's
 * fabric_shape(a1, 1, parameterization) returns it.  The table is in host
 * memory: C is nrows x 9 column-major ([C11 C22 C33 C44 C55 C66 C12 C13 C23]),
 * permutation_blk is 1-based, n_a1a2 * sblk <= nrows.  Out: the six
 * StiffnessTensor fields (C11, C33, C55, C13, C15, C35), nel x ld_out. */
typedef struct {
  const double* C;
  int64_t nrows;
  const double* a1a2_blk;
  int64_t n_a1a2;
  const double* a2a3_blk;
  const int64_t* permutation_blk;
  int64_t sblk;
  double w;
} dp_dem;
/* ---- thermal diffusion step ---------------------------------------------
 * solveDiffusion_threaded (src/ThermalDiffusion/AssemblerThermal.jl:1-57):
 * backward Euler (M + dt K) T_new = M T_old with M the rho Cp mass and K the
 * conduction matrix of the P2 elements (7-point rule), T fixed to Ttop on the
 * outer wall and, if heated, Tbot on the inner one (heated_bottom /
 * insulated_bottom, boundary_conditions.jl:77-105).  Stopping test ||r|| <=
 * atol + rtol ||b|| (Krylov.jl's defaults: sqrt(eps) both).  rho_node: nodal
 * density (vertices read); T: nnod, reference numbering, T_old in, T_new out.
 * Returns DP_NOT_CONVERGED when itmax iterations did not meet the test.
 * itmax = 0: the number of nodes. */
typedef struct {
  double K, Cp, dt, Ttop, Tbot, rtol, atol;
  int32_t heated, itmax;
} dp_thermal_opts;
void dp_default_thermal_opts(dp_thermal_opts* opts);
int dp_thermal_step(dp_ctx* ctx, const dp_thermal_opts* opts, const double* rho_node, double* T,
                    int32_t* iterations, double* relres, int32_t mem);

int dp_fse(dp_ctx* ctx, const double* F, double* const* fse, int64_t ld_out, int32_t mem);
int dp_anisotropic_tensor(dp_ctx* ctx, const dp_dem* dem, const double* vx1, const double* vy1, const double* r1,
                          const double* r2, int64_t ld_in, double* const* C6_out, int64_t ld_out, int32_t mem);

/* ---- batches of independent solves ---------------------------------------
 * Independent problems (contexts of any resolution, all on one device) solved
 * by ONE graph launch: the batch graph holds one branch per context with that
 * context's whole solve, so small problems run side by side.  dp_batch_create
 * prepares and captures (opts: one dp_solve_opts per context, NULL = defaults;
 * no host loops); dp_batch_run recomputes each context's multigrid values for
 * its current assembly, uploads the guesses (use_guess != 0), launches once
 * and returns per-problem reports and completion times (ms from the launch).
 * U, P, P_guess: arrays of n pointers (entries or whole arrays may be NULL for
 * U and P). */
typedef struct dp_batch dp_batch;
int dp_batch_create(dp_ctx* const* ctxs, int32_t n, const dp_solve_opts* opts, dp_batch** out);
int dp_batch_run(dp_batch* batch, double* const* P_guess, double* const* U, double* const* P, int32_t mem,
                 dp_solve_report* reports, double* done_ms);
void dp_batch_destroy(dp_batch* batch);

/* ---- learned initial guess ----------------------------------------------
 * A small convolutional network on the polar grid of the half-resolution
 * mesh's vertices (nrg = ncr/2 + 1 radial x ntg = nct/2 angular, periodic in
 * theta) predicts P/g; dp_guess_from_grid prolongates it to the pressure DOFs
 * for dp_solve with use_guess = 2.  Forward, backward and Adam run in this
 * library's own kernels.  Activations: [batch][channel][r][theta], FP32,
 * device pointers.  (No counterpart in the reference, whose StokesPcCG starts
 * from P = 0.) */
typedef struct dp_cnn dp_cnn;
int dp_cnn_create(int32_t nrg, int32_t ntg, int32_t channels, int32_t layers, const int32_t* dilations,
                  int32_t max_batch, int32_t device, dp_cnn** out);
void dp_cnn_destroy(dp_cnn* net);
int64_t dp_cnn_num_params(const dp_cnn* net);
/* Arithmetic of the convolutions: bf16 = 1 (default) runs the forward pass and
 * the data gradient as implicit GEMMs on the tensor cores (BF16 operands,
 * FP32 accumulation; grids whose theta size is a multiple of 16), 0 runs all
 * of them in FP32 on CUDA cores (the path checked against an FP64 reference).
 * Weight gradients and Adam are FP32 either way (FP32 master weights). */
int dp_cnn_set_math(dp_cnn* net, int32_t bf16);
int dp_cnn_set_params(dp_cnn* net, const float* params, int64_t n);          /* host; resets Adam */
int dp_cnn_get_params(dp_cnn* net, float* params, float* grads, int64_t n);   /* host; either may be NULL */
int dp_cnn_forward(dp_cnn* net, const float* x, float* y, int32_t batch);
int dp_cnn_gradients(dp_cnn* net, const float* x, const float* target, int32_t batch, double* loss);
int dp_cnn_train_step(dp_cnn* net, const float* x, const float* target, int32_t batch, float lr, double* loss);
/* Network inputs (rho, log10 eta, cos 2phi, sin 2phi) of the context's material on its grid. */
int dp_cnn_inputs(dp_ctx* ctx, float* x, int32_t nrg, int32_t ntg);
/* P = scale * (grid field, bilinear at the element vertices) -> pressure DOFs. */
int dp_guess_from_grid(dp_ctx* ctx, const float* p_grid, int32_t nrg, int32_t ntg, double scale, double* P,
                       int32_t mem);

/* Average device time (ms) of one launch of a hot kernel on the context's
 * stream, from CUDA events, after an assembly: which = 0 fine-level A-apply
 * FP32, 1 fine-level A-apply FP64, 2 one multigrid V-cycle (precision of the
 * last solve), 3 the stress post-processor on the inputs of the last
 * dp_stress call, 4 the viscosity update on the inputs of the last
 * dp_viscosity_arrhenius call, 5 the DEM tensor lookup on the inputs of the
 * last dp_anisotropic_tensor call, 6 the thermal element-by-element apply
 * (A p of the last dp_thermal_step's blocks), 7 the vector kernels of one
 * inner iteration of the graph solve launched outside the graph (for
 * profilers; the event time includes their zeroing).  flush_l2 = 0: `reps` back-to-back launches (warm L2);
 * 1: a 256 MB buffer is read before each launch and each launch is timed
 * alone (cold L2, DRAM-bound figure). */
int dp_profile_kernel(dp_ctx* ctx, int32_t which, int32_t reps, int32_t flush_l2, double* ms_per_launch);

#ifdef __cplusplus
}
#endif
#endif
