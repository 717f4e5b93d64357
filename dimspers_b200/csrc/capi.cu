// C ABI entry points (include/dimspers_b200.h).  Every entry point catches
// CUDA and host errors and turns them into a status code plus a message that
// dp_last_error() returns; nothing here exits or aborts.
#include <chrono>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>

#include "../../include/dimspers_b200.h"
#include "kernels.cuh"
#include "mg.cuh"
#include "solver.cuh"

struct dp_ctx {
  dp::Ctx c;
};

namespace dp {

static thread_local std::string g_err;

Ctx::~Ctx() {
  graph_free(*this);
  cudaFree(ctl);
  cudaFreeHost(h_ctl);
  for (cudaStream_t s : aux)
    if (s) cudaStreamDestroy(s);
  mg_free(*this);
  cudaFree(theta_lat); cudaFree(r_lat); cudaFree(ref2lat);
  cudaFree(eta); cudaFree(C); cudaFree(rho_lat); cudaFree(rho_ref);
  cudaFree(mfD64); cudaFree(mfT64); cudaFree(mfD32); cudaFree(mfT32); cudaFree(det_buf);
  cudaFree(K64); cudaFree(K32); cudaFree(Gp); cudaFree(F); cudaFree(pc); cudaFree(Minv); cudaFree(Fscale);
  cudaFree(flush);
  cudaFree(stress_buf);
  cudaFree(rheo_buf);
  cudaFree(fabric_buf);
  if (th_exec) cudaGraphExecDestroy((cudaGraphExec_t)th_exec);
  cudaFree(th_buf);
  cudaFree(scal); cudaFreeHost(h_scal); cudaFree(partial); cudaFree(counter);
  for (void* p : work) cudaFree(p);
  if (stream) cudaStreamDestroy(stream);
}

struct BadArg : std::runtime_error {
  using std::runtime_error::runtime_error;
};

template <typename F>
static int guarded(Ctx* c, F&& f) {
  try {
    return f();
  } catch (const CudaError& e) {
    std::string m = std::string("CUDA error ") + cudaGetErrorName(e.e) + " (" + cudaGetErrorString(e.e) + ") in " +
                    e.what + " line " + std::to_string(e.line);
    if (c) c->err = m; else g_err = m;
    return DP_CUDA_ERROR;
  } catch (const BadArg& e) {
    if (c) c->err = e.what(); else g_err = e.what();
    return DP_BAD_ARG;
  } catch (const std::exception& e) {
    if (c) c->err = e.what(); else g_err = e.what();
    return DP_BAD_ARG;
  }
}

static void check(const dp_mesh_desc* d) {
  if (!d) throw BadArg("null mesh description");
  const std::string m = check_desc(d->nr_cells, d->ntheta_cells, d->r_in, d->r_out, d->pressure_space);
  if (!m.empty()) throw BadArg(m);
}

static cudaMemcpyKind kind_in(int mem) { return mem == DP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; }
static cudaMemcpyKind kind_out(int mem) { return mem == DP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost; }

template <typename T>
static void dalloc(T** p, size_t n) {
  DP_CUDA(cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)));
}

static void upload_eta(Ctx& c, const double* eta_ip, int64_t ld, int mem) {
  const int64_t nel = c.fine.nel;
  if (!eta_ip) throw BadArg("eta_ip is null");
  if (ld < nel) throw BadArg("ld_eta < nel");
  for (int ip = 0; ip < kNip; ++ip)
    DP_CUDA(cudaMemcpyAsync(c.eta + ip * nel, eta_ip + ip * ld, sizeof(double) * nel, kind_in(mem), c.stream));
}

static void upload_rho(Ctx& c, const double* rho, double g, int mem) {
  if (!rho) throw BadArg("rho_node is null");
  DP_CUDA(cudaMemcpyAsync(c.rho_ref, rho, sizeof(double) * c.fine.nnod, kind_in(mem), c.stream));
  launch_gather_ref2lat(c, c.rho_ref, c.rho_lat, 1);
  c.g = g;
}

static void ensure_C(Ctx& c, int64_t n) {
  static_cast<void>(n);
  if (!c.C) dalloc(&c.C, 36 * c.fine.nel);
}

static SolveCfg make_cfg(const dp_solve_opts* o) {
  SolveCfg cfg;
  dp_solve_opts d;
  dp_default_opts(&d);
  if (!o) o = &d;
  cfg.rtol = o->rtol;
  cfg.itmax = o->itmax;
  cfg.itmin = o->itmin;
  cfg.precision = o->precision;
  cfg.inner_pc = o->inner_pc;
  cfg.inner_rtol = o->inner_rtol;
  cfg.inner_itmax = o->inner_itmax;
  cfg.remove_rotation = o->remove_rotation;
  cfg.use_guess = o->use_guess;
  cfg.verbose = o->verbose;
  if (o->cheb_degree > 0) cfg.mg.cheb_degree = o->cheb_degree;
  if (o->cheb_degree_coarse < 0) throw BadArg("cheb_degree_coarse must be >= 0");
  cfg.mg.cheb_degree_coarse = o->cheb_degree_coarse;
  if (o->inner_rtol32 > 0) cfg.inner_rtol32 = o->inner_rtol32;
  if (o->max_refine > 0) cfg.max_refine = o->max_refine;
  cfg.host_loop = o->host_loop;
  cfg.mg.block_jacobi = o->block_jacobi;
  if (o->cheb_lo > 0) cfg.mg.cheb_lo = o->cheb_lo;
  if (o->cheb_hi > 0) cfg.mg.cheb_hi = o->cheb_hi;
  if (!(cfg.mg.cheb_lo < cfg.mg.cheb_hi)) throw BadArg("cheb_lo must be below cheb_hi");
  if (!(cfg.rtol > 0) || cfg.itmax < 1 || cfg.itmin < 0 || !(cfg.inner_rtol > 0) || cfg.inner_itmax < 1)
    throw BadArg("invalid solve options");
  if (cfg.precision < 0 || cfg.precision > 2) throw BadArg("precision must be 0, 1 or 2");
  cfg.inner_relax = o->inner_relax;
  if (o->coarse_max > 0) cfg.mg.coarse_max = o->coarse_max;
  cfg.schur_pc = o->schur_pc;
  if (cfg.schur_pc != 0 && cfg.schur_pc != 1) throw BadArg("schur_pc must be 0 (lumped) or 1 (mass)");
  if (o->launch_overlap != 0 && o->launch_overlap != 1) throw BadArg("launch_overlap must be 0 or 1");
  cfg.launch_overlap = o->launch_overlap;
  if (o->matrix_free != 0 && o->matrix_free != 1) throw BadArg("matrix_free must be 0 or 1");
  cfg.matrix_free = o->matrix_free;
  if (o->true_residual != 0 && o->true_residual != 1) throw BadArg("true_residual must be 0 or 1");
  cfg.true_residual = o->true_residual;
  if (!(o->relax_base >= 0.0) || o->relax_base >= 1.0) throw BadArg("relax_base must be in [0, 1)");
  cfg.relax_base = o->relax_base;
  if (o->mg_tail < 0) throw BadArg("mg_tail must be 0 (off) or a positive element count");
  cfg.mg.tail_max_el = o->mg_tail;
  if (o->apply_warps > 0) cfg.mg.apply_warps = o->apply_warps;
  if (o->apply_warps_t > 0) cfg.mg.apply_warps_t = o->apply_warps_t;
  {
    const int w = cfg.mg.apply_warps, wt = cfg.mg.apply_warps_t;
    if (w != 1 && w != 2 && w != 4 && w != 8) throw BadArg("apply_warps must be 1, 2, 4 or 8");
    if ((wt & (wt - 1)) != 0 || wt > w) throw BadArg("apply_warps_t must be a power of two <= apply_warps");
  }
  if (cfg.inner_pc != 0 && cfg.inner_pc != 1) throw BadArg("inner_pc must be 0 or 1");
  return cfg;
}

// FP32 copy of the packed FP64 element matrices (the layouts differ)
__global__ void k_f64_to_f32(const double* a, float* b, int64_t nel) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nel * kKe) return;
  const int64_t e = i % nel;
  const int p = (int)(i / nel);
  b[kidx32(p, e)] = (float)a[kidx64(p, e)];
}

// FP32 copy of the operator when a mode needs it, then the multigrid values
// (Galerkin operators, smoother bounds, coarse inverse) for the current assembly.
static void check_solve_cfg(const Ctx& c, const SolveCfg& cfg) {
  if (c.assembled < 0) throw BadArg("dp_assemble must run before solving");
  if (cfg.schur_pc == 1 && c.mesh.pressure != 1)
    throw BadArg("schur_pc = 1 (element-block mass inverse) needs discontinuous pressure");
  if (cfg.use_guess < 0 || cfg.use_guess > 2) throw BadArg("use_guess must be 0, 1 or 2");
  if (cfg.use_guess == 2 && cfg.host_loop) throw BadArg("the learned-guess mode runs in the graph path only");
  if (c.fine.det && cfg.matrix_free) throw BadArg("matrix_free applies scatter with atomics: not in deterministic mode");
}

// FP32 copy of the assembled operator (once per assembly) for the FP32 modes.
static void ensure_k32(Ctx& c, const SolveCfg& cfg) {
  if (cfg.precision >= 1 && c.assembled == 0) {
    if (!c.K32) {
      dalloc(&c.K32, kstore<float>(c.fine.nel));
      DP_CUDA(cudaMemsetAsync(c.K32, 0, sizeof(float) * kstore<float>(c.fine.nel), c.stream));
    }
    const int64_t n = kKe * c.fine.nel;
    ++g_klaunch;
    k_f64_to_f32<<<(int)div_up(n, 256), 256, 0, c.stream>>>(c.K64, c.K32, c.fine.nel);
    DP_LAUNCH_CHECK();
    c.assembled = 1;
  }
}

__global__ void k_f64_to_f32_plain(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

// Tile and matrix-free form of the fine-level applies.  The matrix-free data
// are written by every assembly in FP64; the FP32 levels get a rounded copy.
static void set_fine_apply(Ctx& c, const SolveCfg& cfg) {
  c.fine.warps = cfg.mg.apply_warps;
  c.fine.warps_t = cfg.mg.apply_warps_t;
  c.fine.mfD64 = c.fine.mfT64 = nullptr;
  c.fine.mfD32 = c.fine.mfT32 = nullptr;
  if (!cfg.matrix_free) return;
  if (!c.mfD64) {
    // first matrix-free solve on this context: allocate the data and assemble
    // again to fill it (every later assembly keeps it current)
    dalloc(&c.mfD64, 36 * c.fine.nel);
    dalloc(&c.mfT64, (int64_t)kMfTab * 2 * c.fine.ncr);
    const int keep = c.assembled;
    launch_assemble(c, c.assembled >= 1 ? 1 : 0, nullptr);
    c.assembled = keep;
    c.mf32_stale = true;
  }
  c.fine.mfD64 = c.mfD64;
  c.fine.mfT64 = c.mfT64;
  if (cfg.precision >= 1) {
    const int64_t nd = 36 * c.fine.nel, nt = (int64_t)kMfTab * 2 * c.fine.ncr;
    if (!c.mfD32) {
      dalloc(&c.mfD32, nd);
      dalloc(&c.mfT32, nt);
      c.mf32_stale = true;
    }
    if (c.mf32_stale) {
      ++g_klaunch;
      k_f64_to_f32_plain<<<(int)div_up(nd, 256), 256, 0, c.stream>>>(c.mfD64, c.mfD32, nd);
      ++g_klaunch;
      k_f64_to_f32_plain<<<(int)div_up(nt, 256), 256, 0, c.stream>>>(c.mfT64, c.mfT32, nt);
      DP_LAUNCH_CHECK();
      c.mf32_stale = false;
    }
    c.fine.mfD32 = c.mfD32;
    c.fine.mfT32 = c.mfT32;
  }
}

// Checks, the FP32 operator when needed, then the multigrid values (Galerkin
// operators, smoother bounds, coarse inverse) of the current assembly.
static void prepare_solve(Ctx& c, const SolveCfg& cfg) {
  check_solve_cfg(c, cfg);
  ensure_k32(c, cfg);
  set_fine_apply(c, cfg);
  mg_setup(c, cfg.precision >= 1 ? 1 : 0, cfg.mg);
}

// Solution (lattice, work vectors) -> caller's arrays in the reference numbering.
static void deliver_solution(Ctx& c, double* U, double* P, double* Ucart, int mem) {
  const int64_t nn = c.fine.nnod, np = c.mesh.npres;
  double* dU = (double*)c.work[W_U];
  double* dP = (double*)c.work[W_P];
  double* stage = (double*)c.work[W_UC];
  if (U) {
    launch_scatter_lat2ref(c, dU, stage, 2);
    DP_CUDA(cudaMemcpyAsync(U, stage, sizeof(double) * 2 * nn, kind_out(mem), c.stream));
  }
  if (P) DP_CUDA(cudaMemcpyAsync(P, dP, sizeof(double) * np, kind_out(mem), c.stream));
  if (Ucart) {
    double* uc = (double*)c.work[W_RES];
    to_cartesian(c, dU, uc);
    launch_scatter_lat2ref(c, uc, stage, 2);
    DP_CUDA(cudaMemcpyAsync(Ucart, stage, sizeof(double) * 2 * nn, kind_out(mem), c.stream));
  }
}

static void fill_report(const Ctx& c, const SolveResult& res, dp_solve_report* rep) {
  if (!rep) return;
  std::memset(rep, 0, sizeof(*rep));
  rep->status = res.status;
  rep->iterations = res.iterations;
  rep->inner_iterations = res.inner_its;
  rep->relres = res.relres;
  rep->r0 = res.r0;
  rep->omega = res.omega;
  rep->div_residual = res.div_residual;
  rep->mom_residual = res.mom_residual;
  rep->mg_levels = (int)c.mg.size();
  rep->kernel_launches = res.launches;
  rep->refinements = res.refinements;
  rep->fallback_used = res.fallback;
  rep->r0_guess = res.r0_guess;
  rep->restarts = res.restarts;
}

}  // namespace dp

struct dp_batch {
  dp::Batch b;
};

using namespace dp;

extern "C" {

int dp_batch_create(dp_ctx* const* ctxs, int32_t n, const dp_solve_opts* opts, dp_batch** out) {
  if (!ctxs || n < 1 || !out) return DP_BAD_ARG;
  *out = nullptr;
  dp_batch* h = nullptr;
  int st = guarded(nullptr, [&] {
    h = new dp_batch();
    const int dev = ctxs[0] ? ctxs[0]->c.device : 0;
    DP_CUDA(cudaSetDevice(dev));
    for (int i = 0; i < n; ++i) {
      if (!ctxs[i]) throw BadArg("null context in batch");
      Ctx& c = ctxs[i]->c;
      if (c.device != dev) throw BadArg("all contexts of a batch must be on one device");
      for (int j = 0; j < i; ++j)
        if (ctxs[j] == ctxs[i]) throw BadArg("a context appears twice in the batch");
      SolveCfg cfg = make_cfg(opts ? &opts[i] : nullptr);
      if (cfg.host_loop) throw BadArg("batches run in the graph path only");
      prepare_solve(c, cfg);
      DP_CUDA(cudaStreamSynchronize(c.stream));
      h->b.ctx.push_back(&c);
      h->b.cfg.push_back(cfg);
    }
    batch_build(h->b);
    return (int)DP_OK;
  });
  if (st != DP_OK) {
    delete h;
    return st;
  }
  *out = h;
  return DP_OK;
}

int dp_batch_run(dp_batch* h, double* const* P_guess, double* const* U, double* const* P, int32_t mem,
                 dp_solve_report* reports, double* done_ms) {
  if (!h) return DP_BAD_ARG;
  Batch& b = h->b;
  int st = guarded(nullptr, [&] {
    const int n = (int)b.ctx.size();
    DP_CUDA(cudaSetDevice(b.ctx[0]->device));
    for (int i = 0; i < n; ++i) {
      Ctx& c = *b.ctx[i];
      prepare_solve(c, b.cfg[i]);   // multigrid values of the current assembly
      if (b.cfg[i].use_guess) {
        if (!P_guess || !P_guess[i]) throw BadArg("use_guess needs a guess for every problem");
        DP_CUDA(cudaMemcpyAsync(c.work[W_P], P_guess[i], sizeof(double) * c.mesh.npres, kind_in(mem), c.stream));
      }
      DP_CUDA(cudaStreamSynchronize(c.stream));
    }
    std::vector<SolveResult> res;
    std::vector<double> ms;
    batch_run(b, res, ms);
    for (int i = 0; i < n; ++i) {
      Ctx& c = *b.ctx[i];
      deliver_solution(c, U ? U[i] : nullptr, P ? P[i] : nullptr, nullptr, mem);
      DP_CUDA(cudaStreamSynchronize(c.stream));
      fill_report(c, res[i], reports ? &reports[i] : nullptr);
      if (done_ms) done_ms[i] = ms[i];
    }
    return (int)DP_OK;
  });
  if (st != DP_OK) b.err = g_err;
  return st;
}

void dp_batch_destroy(dp_batch* h) {
  if (!h) return;
  if (h->b.s) cudaStreamSynchronize(h->b.s);
  delete h;
}

void dp_default_opts(dp_solve_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->rtol = 1e-8;
  o->itmax = 200;
  o->itmin = 10;
  o->precision = DP_PREC_FP64;
  o->inner_pc = DP_INNER_MG;
  o->inner_rtol = 1e-10;
  o->inner_itmax = 500;
  o->remove_rotation = 1;
  o->use_guess = 0;
  o->verbose = 0;
  o->cheb_degree = 3;
  o->inner_rtol32 = 1e-5;
  o->max_refine = 6;
  o->host_loop = 0;
  o->block_jacobi = 1;
  o->cheb_lo = 0.1;
  o->cheb_hi = 1.1;
  o->inner_relax = 0.0;
  o->coarse_max = 1536;
  o->apply_warps = 4;
  o->apply_warps_t = 1;
  o->launch_overlap = 1;
  o->mg_tail = 0;
  o->matrix_free = 0;
  o->true_residual = 1;
  o->relax_base = 0.0;
}

const char* dp_status_string(int s) {
  switch (s) {
    case DP_OK: return "OK";
    case DP_NOT_CONVERGED: return "NOT_CONVERGED";
    case DP_BREAKDOWN: return "BREAKDOWN";
    case DP_BAD_ARG: return "BAD_ARG";
    case DP_CUDA_ERROR: return "CUDA_ERROR";
    case DP_DEVICE_TIMEOUT: return "DEVICE_TIMEOUT";
    default: return "UNKNOWN";
  }
}

int dp_mesh_sizes(const dp_mesh_desc* d, int64_t* nel, int64_t* nnod, int64_t* npres, int64_t* nfixed) {
  return guarded(nullptr, [&] {
    check(d);
    mesh_sizes(d->nr_cells, d->ntheta_cells, d->pressure_space, nel, nnod, npres, nfixed);
    if (nfixed && d->pin_rotation) *nfixed += 1;
    return (int)DP_OK;
  });
}

int dp_mesh_build(const dp_mesh_desc* d, int64_t* e2n, double* theta, double* r, int32_t* colors, int32_t* ncolors) {
  return guarded(nullptr, [&] {
    check(d);
    Mesh m;
    build_mesh(m, d->nr_cells, d->ntheta_cells, d->r_in, d->r_out, d->pressure_space, colors || ncolors);
    if (e2n)
      for (int64_t i = 0; i < 6 * m.nel; ++i) e2n[i] = m.e2n[i] + 1;
    if (theta) std::memcpy(theta, m.theta.data(), sizeof(double) * m.nnod);
    if (r) std::memcpy(r, m.r.data(), sizeof(double) * m.nnod);
    if (colors) std::memcpy(colors, m.colors.data(), sizeof(int32_t) * m.nel);
    if (ncolors) *ncolors = m.ncolors;
    return (int)DP_OK;
  });
}

int dp_mesh_free_slip(const dp_mesh_desc* d, int64_t* omega, int64_t* nomega) {
  return guarded(nullptr, [&] {
    check(d);
    Mesh m;
    build_mesh(m, d->nr_cells, d->ntheta_cells, d->r_in, d->r_out, d->pressure_space, false);
    std::vector<int64_t> om = m.omega;
    if (d->pin_rotation) om.push_back(2 * (int64_t)d->nr_cells);  // u_theta of node nr (0-based 2*(nr-1))
    if (nomega) *nomega = (int64_t)om.size();
    if (omega)
      for (size_t i = 0; i < om.size(); ++i) omega[i] = om[i] + 1;
    return (int)DP_OK;
  });
}

int dp_ctx_create(const dp_mesh_desc* d, dp_ctx** out) {
  if (!out) return DP_BAD_ARG;
  *out = nullptr;
  dp_ctx* h = nullptr;
  int st = guarded(nullptr, [&] {
    check(d);
    int ndev = 0;
    DP_CUDA(cudaGetDeviceCount(&ndev));
    if (d->device < 0 || d->device >= ndev) throw BadArg("device ordinal out of range");
    const int64_t nel = 2 * (int64_t)d->nr_cells * d->ntheta_cells;
    if (nel * kKe >= ((int64_t)1 << 31)) throw BadArg("mesh too large for 32-bit element indexing");
    h = new dp_ctx();
    Ctx& c = h->c;
    c.device = d->device;
    DP_CUDA(cudaSetDevice(c.device));
    build_mesh(c.mesh, d->nr_cells, d->ntheta_cells, d->r_in, d->r_out, d->pressure_space, true);
    c.fine.ncr = d->nr_cells;
    c.fine.nct = d->ntheta_cells;
    c.fine.pin = d->pin_rotation ? 1 : 0;
    c.fine.nel = c.mesh.nel;
    c.fine.nnod = c.mesh.nnod;
    DP_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    upload_quadrature_constants();
    upload_mg_constants();
    const int64_t nn = c.mesh.nnod, np = c.mesh.npres;
    std::vector<double> tl(nn), rl(nn);
    for (int64_t i = 0; i < nn; ++i) {
      tl[c.mesh.ref2lat[i]] = c.mesh.theta[i];
      rl[c.mesh.ref2lat[i]] = c.mesh.r[i];
    }
    dalloc(&c.theta_lat, nn);
    dalloc(&c.r_lat, nn);
    dalloc(&c.ref2lat, nn);
    DP_CUDA(cudaMemcpy(c.theta_lat, tl.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
    DP_CUDA(cudaMemcpy(c.r_lat, rl.data(), sizeof(double) * nn, cudaMemcpyHostToDevice));
    DP_CUDA(cudaMemcpy(c.ref2lat, c.mesh.ref2lat.data(), sizeof(int64_t) * nn, cudaMemcpyHostToDevice));
    dalloc(&c.eta, kNip * nel);
    dalloc(&c.rho_lat, nn);
    dalloc(&c.rho_ref, nn);
    dalloc(&c.K64, kstore<double>(nel));
    DP_CUDA(cudaMemset(c.K64, 0, sizeof(double) * kstore<double>(nel)));
    dalloc(&c.Gp, kGe * nel);
    dalloc(&c.F, 2 * nn);
    dalloc(&c.pc, np);
    dalloc(&c.Minv, 6 * nel);
    dalloc(&c.scal, 64);
    DP_CUDA(cudaMemset(c.scal, 0, sizeof(double) * 64));
    DP_CUDA(cudaMallocHost((void**)&c.h_scal, sizeof(double) * 64));
    dalloc(&c.partial, kPartialDoubles);
    dalloc(&c.counter, 1);
    DP_CUDA(cudaMemset(c.counter, 0, sizeof(unsigned int)));
    c.work.assign(W_COUNT, nullptr);
    for (int w = 0; w < W_COUNT; ++w) {
      size_t bytes;
      if (w <= W_SQ) bytes = sizeof(double) * np;
      else if (w <= W_RES) bytes = sizeof(double) * 2 * nn;
      else if (w <= W_F_AP) bytes = sizeof(float) * 2 * nn;
      else if (w == W_P) bytes = sizeof(double) * np;
      else bytes = sizeof(double) * 2 * nn;
      DP_CUDA(cudaMalloc(&c.work[w], bytes ? bytes : 8));
    }
    return (int)DP_OK;
  });
  if (st != DP_OK) {
    delete h;
    return st;
  }
  *out = h;
  return DP_OK;
}

void dp_ctx_destroy(dp_ctx* h) {
  if (!h) return;
  cudaSetDevice(h->c.device);
  if (h->c.stream) cudaStreamSynchronize(h->c.stream);
  delete h;
}

const char* dp_last_error(const dp_ctx* h) { return h ? h->c.err.c_str() : g_err.c_str(); }

void* dp_ctx_stream(dp_ctx* h) { return h ? (void*)h->c.stream : nullptr; }

int dp_get_connectivity(dp_ctx* h, int64_t* e2n, int32_t* colors) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    if (e2n)
      for (int64_t i = 0; i < 6 * c.mesh.nel; ++i) e2n[i] = c.mesh.e2n[i] + 1;
    if (colors) std::memcpy(colors, c.mesh.colors.data(), sizeof(int32_t) * c.mesh.nel);
    return (int)DP_OK;
  });
}

int dp_set_material(dp_ctx* h, const double* eta_ip, int64_t ld_eta, const double* const* C6, int64_t ld_C,
                    const double* rho_node, double g, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    upload_eta(c, eta_ip, ld_eta, mem);
    if (C6) {
      const int64_t nel = c.fine.nel;
      if (ld_C < nel) throw BadArg("ld_C < nel");
      ensure_C(c, 36 * nel);
      for (int f = 0; f < 6; ++f) {
        if (!C6[f]) throw BadArg("null tensor field");
        for (int ip = 0; ip < kNip; ++ip)
          DP_CUDA(cudaMemcpyAsync(c.C + ((size_t)f * 6 + ip) * nel, C6[f] + ip * ld_C, sizeof(double) * nel,
                                  kind_in(mem), c.stream));
      }
      c.mat_kind = MAT_FULL;
    } else {
      c.mat_kind = MAT_ISO;
    }
    upload_rho(c, rho_node, g, mem);
    c.assembled = -1;
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

int dp_set_material_ti(dp_ctx* h, const double* eta_ip, int64_t ld_eta, const double* delta, const double* dir_x,
                       const double* dir_y, const double* rho_node, double g, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!delta || !dir_x || !dir_y) throw BadArg("null delta / director");
    upload_eta(c, eta_ip, ld_eta, mem);
    const int64_t nel = c.fine.nel;
    ensure_C(c, 3 * nel);
    DP_CUDA(cudaMemcpyAsync(c.C, delta, sizeof(double) * nel, kind_in(mem), c.stream));
    DP_CUDA(cudaMemcpyAsync(c.C + nel, dir_x, sizeof(double) * nel, kind_in(mem), c.stream));
    DP_CUDA(cudaMemcpyAsync(c.C + 2 * nel, dir_y, sizeof(double) * nel, kind_in(mem), c.stream));
    c.mat_kind = MAT_TI;
    upload_rho(c, rho_node, g, mem);
    c.assembled = -1;
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

int dp_fse_director(dp_ctx* h, const double* F, double* dir_x, double* dir_y, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!F || !dir_x || !dir_y) throw BadArg("null argument");
    const int64_t nel = c.fine.nel;
    double *dF = nullptr, *dx = nullptr, *dy = nullptr;
    const bool host = mem != DP_MEM_DEVICE;
    if (host) {
      dalloc(&dF, 4 * nel);
      dalloc(&dx, nel);
      dalloc(&dy, nel);
      DP_CUDA(cudaMemcpyAsync(dF, F, sizeof(double) * 4 * nel, cudaMemcpyHostToDevice, c.stream));
    }
    launch_fse_director(c, host ? dF : F, host ? dx : dir_x, host ? dy : dir_y, nel);
    if (host) {
      DP_CUDA(cudaMemcpyAsync(dir_x, dx, sizeof(double) * nel, cudaMemcpyDeviceToHost, c.stream));
      DP_CUDA(cudaMemcpyAsync(dir_y, dy, sizeof(double) * nel, cudaMemcpyDeviceToHost, c.stream));
    }
    DP_CUDA(cudaStreamSynchronize(c.stream));
    cudaFree(dF); cudaFree(dx); cudaFree(dy);
    return (int)DP_OK;
  });
}

int dp_assemble(dp_ctx* h, int32_t precision) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (c.mat_kind == MAT_NONE) throw BadArg("material not set");
    if (precision < 0 || precision > 2) throw BadArg("precision must be 0, 1 or 2");
    if (precision >= 1 && !c.K32) {
      dalloc(&c.K32, kstore<float>(c.fine.nel));
      DP_CUDA(cudaMemset(c.K32, 0, sizeof(float) * kstore<float>(c.fine.nel)));
    }
    launch_assemble(c, precision, nullptr);  // also refreshes the matrix-free data once enabled
    c.mf32_stale = true;
    c.assembled = precision;
    c.mg_prec = c.mg.empty() ? -1 : c.mg_prec;  // hierarchy values are rebuilt on the next solve
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

int dp_set_deterministic(dp_ctx* h, int32_t on) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (on != 0 && on != 1) throw BadArg("on must be 0 or 1");
    if (on && c.mesh.pressure != 1)
      throw BadArg("deterministic mode needs discontinuous pressure (the continuous space's G^T and lumped "
                   "mass still scatter with atomics)");
    DP_CUDA(cudaStreamSynchronize(c.stream));
    if (on && !c.det_buf) dalloc(&c.det_buf, (size_t)kDetPerElem * c.fine.nel);
    c.fine.det = on ? c.det_buf : nullptr;
    graph_free(c);                          // the captured launches differ between the modes
    if (on) c.assembled = -1;               // the right-hand side must be assembled again without atomics
    return (int)DP_OK;
  });
}

int dp_get_element_matrices(dp_ctx* h, double* Ke, double* Ge, double* Me, double* Fb) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (c.mat_kind == MAT_NONE) throw BadArg("material not set");
    const int64_t nel = c.fine.nel;
    CartOut co;
    dalloc(&co.Ke, kKe * nel);
    dalloc(&co.Ge, kGe * nel);
    dalloc(&co.Me, kMe * nel);
    dalloc(&co.Fb, kFe * nel);
    launch_assemble(c, c.assembled == 1 ? 1 : 0, &co);
    if (Ke) DP_CUDA(cudaMemcpyAsync(Ke, co.Ke, sizeof(double) * kKe * nel, cudaMemcpyDeviceToHost, c.stream));
    if (Ge) DP_CUDA(cudaMemcpyAsync(Ge, co.Ge, sizeof(double) * kGe * nel, cudaMemcpyDeviceToHost, c.stream));
    if (Me) DP_CUDA(cudaMemcpyAsync(Me, co.Me, sizeof(double) * kMe * nel, cudaMemcpyDeviceToHost, c.stream));
    if (Fb) DP_CUDA(cudaMemcpyAsync(Fb, co.Fb, sizeof(double) * kFe * nel, cudaMemcpyDeviceToHost, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    cudaFree(co.Ke); cudaFree(co.Ge); cudaFree(co.Me); cudaFree(co.Fb);
    if (c.assembled < 0) c.assembled = 0;
    return (int)DP_OK;
  });
}

int dp_solve(dp_ctx* h, double* U, double* P, double* Ucart, const dp_solve_opts* opts, dp_solve_report* rep,
             int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!U || !P) throw BadArg("null U or P");
    SolveCfg cfg = make_cfg(opts);
    check_solve_cfg(c, cfg);
    const int64_t nn = c.fine.nnod, np = c.mesh.npres;
    ensure_k32(c, cfg);
    set_fine_apply(c, cfg);
    cudaEvent_t e0, e1, e2;
    DP_CUDA(cudaEventCreate(&e0));
    DP_CUDA(cudaEventCreate(&e1));
    DP_CUDA(cudaEventCreate(&e2));
    DP_CUDA(cudaEventRecord(e0, c.stream));
    mg_setup(c, cfg.precision >= 1 ? 1 : 0, cfg.mg);
    DP_CUDA(cudaEventRecord(e1, c.stream));
    double* dU = (double*)c.work[W_U];
    double* dP = (double*)c.work[W_P];
    if (cfg.use_guess) {
      DP_CUDA(cudaMemcpyAsync(dP, P, sizeof(double) * np, kind_in(mem), c.stream));
    }
    DP_CUDA(cudaMemsetAsync(dU, 0, sizeof(double) * 2 * nn, c.stream));
    SolveResult res;
    if (cfg.host_loop) {
      const int64_t k0 = g_klaunch;
      PdlScope pdl(cfg.launch_overlap);
      schur_pcg(c, cfg, dU, dP, res);
      res.launches = g_klaunch - k0;
    } else {
      schur_pcg_graph(c, cfg, dU, dP, res);
    }
    // lattice -> reference numbering
    deliver_solution(c, U, P, Ucart, mem);
    DP_CUDA(cudaEventRecord(e2, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    float ms_setup = 0, ms_solve = 0;
    cudaEventElapsedTime(&ms_setup, e0, e1);
    cudaEventElapsedTime(&ms_solve, e1, e2);
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2);
    fill_report(c, res, rep);
    if (rep) {
      rep->t_setup_ms = ms_setup;
      rep->t_solve_ms = ms_solve;
    }
    if (res.status == 1) c.err = "outer iteration cap reached";
    if (res.status == 2) c.err = "breakdown: q.Sq <= 0 or non-finite scalar";
    return res.status;
  });
}

static int apply_common(dp_ctx* h, const double* in, double* out, int32_t mem, int which) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (c.assembled < 0) throw BadArg("dp_assemble must run first");
    if (!in || !out) throw BadArg("null argument");
    const int64_t nn = c.fine.nnod, np = c.mesh.npres;
    double* a = (double*)c.work[W_Y];
    double* b = (double*)c.work[W_Z];
    double* stage = (double*)c.work[W_UC];
    double* pbuf = (double*)c.work[W_P];
    if (which == 0) {  // K
      DP_CUDA(cudaMemcpyAsync(stage, in, sizeof(double) * 2 * nn, kind_in(mem), c.stream));
      launch_gather_ref2lat(c, stage, a, 2);
      launch_apply_K<double, double>(c.fine, c.K64, a, b, c.stream);
      launch_scatter_lat2ref(c, b, stage, 2);
      DP_CUDA(cudaMemcpyAsync(out, stage, sizeof(double) * 2 * nn, kind_out(mem), c.stream));
    } else if (which == 1) {  // G
      DP_CUDA(cudaMemcpyAsync(pbuf, in, sizeof(double) * np, kind_in(mem), c.stream));
      launch_apply_G(c, pbuf, b);
      launch_scatter_lat2ref(c, b, stage, 2);
      DP_CUDA(cudaMemcpyAsync(out, stage, sizeof(double) * 2 * nn, kind_out(mem), c.stream));
    } else {  // G^T
      DP_CUDA(cudaMemcpyAsync(stage, in, sizeof(double) * 2 * nn, kind_in(mem), c.stream));
      launch_gather_ref2lat(c, stage, a, 2);
      launch_apply_GT(c, a, pbuf);
      DP_CUDA(cudaMemcpyAsync(out, pbuf, sizeof(double) * np, kind_out(mem), c.stream));
    }
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

int dp_reduce(dp_ctx* h, const double* a, const double* b, int64_t n, int32_t op, double* out, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!a || !out || n < 0 || op < 0 || op > 3 || (op < 2 && !b)) throw BadArg("dp_reduce: bad argument");
    const double* da = a;
    const double* db = b;
    double* tmp = nullptr;
    if (mem == DP_MEM_HOST && n > 0) {
      DP_CUDA(cudaMalloc(&tmp, sizeof(double) * 2 * n));
      DP_CUDA(cudaMemcpyAsync(tmp, a, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
      if (op < 2) DP_CUDA(cudaMemcpyAsync(tmp + n, b, sizeof(double) * n, cudaMemcpyHostToDevice, c.stream));
      da = tmp;
      db = tmp + n;
    }
    const int slot = 40;
    if (op == 0) launch_dot(c, da, db, n, slot);
    else if (op == 1) launch_dot_c(c, da, db, n, slot);
    else if (op == 2) launch_sum(c, da, n, slot);
    else launch_sum_c(c, da, n, slot);
    DP_CUDA(cudaMemcpyAsync(c.h_scal + slot, c.scal + slot, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    if (tmp) DP_CUDA(cudaFree(tmp));
    *out = c.h_scal[slot];
    return (int)DP_OK;
  });
}

int dp_apply_K(dp_ctx* h, const double* x, double* y, int32_t mem) { return apply_common(h, x, y, mem, 0); }
int dp_apply_G(dp_ctx* h, const double* p, double* y, int32_t mem) { return apply_common(h, p, y, mem, 1); }
int dp_apply_GT(dp_ctx* h, const double* x, double* p, int32_t mem) { return apply_common(h, x, p, mem, 2); }

// Reads the flush buffer (so the L2 holds only clean lines of it afterwards;
// a write-based flush would leave dirty lines whose write-back overlaps the
// timed kernel).  The sink is written only if the sum hits an impossible value.
__global__ void k_flush_read(const uint4* __restrict__ buf, int64_t n, unsigned int* sink) {
  unsigned int acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint4 v = buf[i];
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9e3779b9u) sink[0] = acc;
}

namespace dp {
void launch_stress_staged(Ctx& c, bool tensor);
void launch_viscosity_staged(Ctx& c);
void launch_dem_staged(Ctx& c);
void launch_th_apply_staged(Ctx& c);
}

int dp_profile_kernel(dp_ctx* h, int32_t which, int32_t reps, int32_t flush_l2, double* ms) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (which < 3 && c.assembled < 0) throw BadArg("dp_assemble must run first");
    if (reps < 1 || !ms) throw BadArg("reps must be >= 1");
    if (which == 0 && !c.K32) throw BadArg("no FP32 element matrices (assemble with precision 1)");
    if (which == 2 && c.mg.empty()) throw BadArg("no multigrid hierarchy (run a solve first)");
    if (which == 3 && !c.stress_buf) throw BadArg("no staged post-processor inputs (call dp_stress first)");
    if (which == 4 && !c.rheo_buf) throw BadArg("no staged viscosity inputs (call dp_viscosity_arrhenius first)");
    if (which == 5 && c.fabric_dem[0] == 0)
      throw BadArg("no staged DEM tensor inputs (call dp_anisotropic_tensor first)");
    if (which == 6 && !c.th_buf) throw BadArg("no thermal element blocks (call dp_thermal_step first)");
    if (which < 0 || which > 7) throw BadArg("which must be 0..7");
    const int64_t n = 2 * c.fine.nnod;
    double* x64 = (double*)c.work[W_IN_P];
    double* y64 = (double*)c.work[W_IN_AP];
    float* x32 = (float*)c.work[W_F_P];
    float* y32 = (float*)c.work[W_F_AP];
    DP_CUDA(cudaMemsetAsync(x64, 0, sizeof(double) * n, c.stream));
    DP_CUDA(cudaMemsetAsync(x32, 0, sizeof(float) * n, c.stream));
    // the applies accumulate into y (x is zero, so y stays zero): the events
    // bracket the kernel alone, not the zeroing that launch_apply_K adds
    DP_CUDA(cudaMemsetAsync(y64, 0, sizeof(double) * n, c.stream));
    DP_CUDA(cudaMemsetAsync(y32, 0, sizeof(float) * n, c.stream));
    auto once = [&] {
      if (which == 0) launch_apply_K_acc<float, float>(c.fine, c.K32, x32, y32, c.stream);
      else if (which == 1) launch_apply_K_acc<double, double>(c.fine, c.K64, x64, y64, c.stream);
      else if (which == 3) launch_stress_staged(c, c.stress_tensor);
      else if (which == 4) launch_viscosity_staged(c);
      else if (which == 5) launch_dem_staged(c);
      else if (which == 6) launch_th_apply_staged(c);
      else if (which == 7) profile_inner_vector_kernels(c);
      else if (c.mg_prec == 1) mg_apply_f(c, x32, y32, MGOptions());
      else mg_apply(c, x64, y64, MGOptions());
    };
    once();
    cudaEvent_t e0, e1;
    DP_CUDA(cudaEventCreate(&e0));
    DP_CUDA(cudaEventCreate(&e1));
    double total = 0.0;
    if (flush_l2) {
      // cold L2: read a buffer of twice the L2 size before every launch
      // and time each launch on its own
      const size_t fb = 256ull << 20;
      if (!c.flush) {
        DP_CUDA(cudaMalloc(&c.flush, fb + 256));
        DP_CUDA(cudaMemsetAsync(c.flush, 0, fb + 256, c.stream));
      }
      for (int i = 0; i < reps; ++i) {
        ++g_klaunch;
        k_flush_read<<<1184, 256, 0, c.stream>>>((const uint4*)c.flush, (int64_t)(fb / sizeof(uint4)),
                                                 (unsigned int*)((char*)c.flush + fb));
        DP_LAUNCH_CHECK();
        DP_CUDA(cudaEventRecord(e0, c.stream));
        once();
        DP_CUDA(cudaEventRecord(e1, c.stream));
        DP_CUDA(cudaEventSynchronize(e1));
        float t = 0;
        DP_CUDA(cudaEventElapsedTime(&t, e0, e1));
        total += t;
      }
    } else {
      DP_CUDA(cudaEventRecord(e0, c.stream));
      for (int i = 0; i < reps; ++i) once();
      DP_CUDA(cudaEventRecord(e1, c.stream));
      DP_CUDA(cudaEventSynchronize(e1));
      float t = 0;
      DP_CUDA(cudaEventElapsedTime(&t, e0, e1));
      total = t;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = total / reps;
    return (int)DP_OK;
  });
}

int dp_get_rhs(dp_ctx* h, double* F, double* pc) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (c.assembled < 0) throw BadArg("dp_assemble must run first");
    double* stage = (double*)c.work[W_UC];
    if (F) {
      launch_scatter_lat2ref(c, c.F, stage, 2);
      DP_CUDA(cudaMemcpyAsync(F, stage, sizeof(double) * 2 * c.fine.nnod, cudaMemcpyDeviceToHost, c.stream));
    }
    if (pc) DP_CUDA(cudaMemcpyAsync(pc, c.pc, sizeof(double) * c.mesh.npres, cudaMemcpyDeviceToHost, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

}  // extern "C"
