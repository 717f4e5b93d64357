// Thermal diffusion step on the P2 annulus: solveDiffusion_threaded
// (src/ThermalDiffusion/AssemblerThermal.jl:1-57), backward Euler
//   (M + dt K) T_new = M T_old,  T = Ttop / Tbot on the walls,
// with M = rho Cp mass and K the conduction matrix of assemble_element!
// (:114-226; 7-point rule, the element's curved inverse Jacobian).  The
// reference's force vector never reaches the system (the function returns
// before update_force_vector!), so neither does one here.
//
// Layout: the element blocks A_e = M_e + dt K_e (symmetric 6x6, 21 packed
// upper entries) entry-major, 168 B per element, in lattice order; the free
// nodes are all but the two walls (lattice radial index 0 and 2 ncr), found
// from the node index, so no index list is stored.
//
// k_th_assemble (one thread per element, FP64): A_e, diag(A) and b = M T_old
// - A T_bc by atomics (T_bc: the wall values, zero inside).  The solve is
// Jacobi-preconditioned CG (the matrix is SPD; the reference runs
// unpreconditioned GMRES) with the reference's stopping test ||r|| <= atol +
// rtol ||b|| (Krylov.jl's defaults sqrt(eps)), captured once per context as a
// CUDA graph whose WHILE node is continued or ended by the last block of the
// update kernel: per iteration k_th_apply (q = A p), k_th_pq (alpha),
// k_th_update (x, r, z, beta and the stop test), k_th_dir (p, q = 0).
#include "kernels.cuh"
#include "reduce.cuh"

namespace dp {

// scalar-table slots of the thermal loop
enum ThSlot { TH_RZ = 48, TH_PQ = 49, TH_ALPHA = 50, TH_BETA = 51, TH_RR = 52, TH_TOL2 = 53, TH_IT = 54,
              TH_ITMAX = 55, TH_BB = 56, TH_RZN = 57 };

__constant__ double c_w7[7];  // 7-point weights x 0.5 (Quadrature.jl:109-138)

static void upload_thermal_constants() {
  const double w1 = (155.0 - std::sqrt(15.0)) / 1200.0, w2 = (155.0 + std::sqrt(15.0)) / 1200.0;
  const double w[7] = {0.5 * 0.225, 0.5 * w1, 0.5 * w1, 0.5 * w1, 0.5 * w2, 0.5 * w2, 0.5 * w2};
  DP_CUDA(cudaMemcpyToSymbol(c_w7, w, sizeof(w)));
}

constexpr int kThPack = 21;

__device__ __forceinline__ bool th_fixed(int64_t n, int64_t A, int amax, int heated) {
  const int a = (int)(n % A);
  return a == amax || (heated && a == 0);
}

struct ThAsmArgs {
  const double* theta_lat;
  const double* r_lat;
  const double* rho_lat;
  const double* Told;  // lattice
  const double* Tbc;   // lattice: wall values, 0 inside
  double* Ae;          // 21 x nel
  double* diag;        // nnod
  double* b;           // nnod
  double K, Cp, dt;
  int nel, ncr, A, B;
};

__global__ void __launch_bounds__(128) k_th_assemble(ThAsmArgs p) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= p.nel) return;
  int64_t nd[6];
  element_nodes(e, p.ncr, p.A, p.B, nd);
  double th[3], rr[3], rho[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    th[k] = p.theta_lat[nd[k]];
    rr[k] = p.r_lat[nd[k]];
    rho[k] = p.rho_lat[nd[k]];
  }
  {
    const double PI = 3.14159265358979323846;
    const double d1 = fabs(th[0] - th[1]), d2 = fabs(th[1] - th[2]), d3 = fabs(th[2] - th[0]);
    if ((d1 + d2 + d3) > PI) {
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (th[k] < PI) th[k] += 2.0 * PI;
    }
  }
  // J = dN3ds * [theta r]: rows (dN/dxi, dN/deta) = (-1, 1, 0), (-1, 0, 1)
  const double J1 = -th[0] + th[1], J2 = -th[0] + th[2], J3 = -rr[0] + rr[1], J4 = -rr[0] + rr[2];
  const double detJ = J1 * J4 - J2 * J3;
  const double R21 = rr[1] - rr[0], R31 = rr[2] - rr[0];
  const double T31 = th[2] - th[0], T21 = th[1] - th[0];
  double Ke[kThPack], Me[kThPack];
#pragma unroll
  for (int k = 0; k < kThPack; ++k) Ke[k] = Me[k] = 0.0;
  for (int ip = 0; ip < 7; ++ip) {
    const double th_ip = th[0] * c_N3s[ip][0] + th[1] * c_N3s[ip][1] + th[2] * c_N3s[ip][2];
    const double r_ip = rr[0] * c_N3s[ip][0] + rr[1] * c_N3s[ip][1] + rr[2] * c_N3s[ip][2];
    const double rho_ip = rho[0] * c_N3s[ip][0] + rho[1] * c_N3s[ip][1] + rho[2] * c_N3s[ip][2];
    double s, c;
    sincos(th_ip, &s, &c);
    const double cr = c / r_ip, sr = s / r_ip;
    const double a11 = R31 * cr - T31 * s, a12 = -R21 * cr + T21 * s;
    const double a21 = -R31 * sr - T31 * c, a22 = R21 * sr + T21 * c;
    double dx[6], dz[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      dx[k] = (a11 * c_dNs[ip][0][k] + a12 * c_dNs[ip][1][k]) / detJ;
      dz[k] = (a21 * c_dNs[ip][0][k] + a22 * c_dNs[ip][1][k]) / detJ;
    }
    const double om = r_ip * detJ * c_w7[ip];
    const double wk = p.K * om, wm = om * rho_ip * p.Cp;
    int k = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
      for (int j = i; j < 6; ++j, ++k) {
        Ke[k] += wk * (dx[i] * dx[j] + dz[i] * dz[j]);
        Me[k] += wm * c_N6s[ip][i] * c_N6s[ip][j];
      }
    }
  }
  double to[6], tb[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    to[i] = p.Told[nd[i]];
    tb[i] = p.Tbc[nd[i]];
  }
  double be[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const size_t st = (size_t)p.nel;
  int k = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j, ++k) {
      const double a = Me[k] + p.dt * Ke[k];
      p.Ae[(size_t)k * st + e] = a;
      if (i == j) {
        atomicAdd(&p.diag[nd[i]], a);
        be[i] += Me[k] * to[i] - a * tb[i];
      } else {
        be[i] += Me[k] * to[j] - a * tb[j];
        be[j] += Me[k] * to[i] - a * tb[i];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) atomicAdd(&p.b[nd[i]], be[i]);
}

// q += A p over elements (q zeroed by the caller)
__global__ void __launch_bounds__(128) k_th_apply(const double* __restrict__ Ae, const double* __restrict__ x,
                                                  double* __restrict__ y, int nel, int ncr, int64_t A, int64_t B) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  double a[kThPack];
  const size_t st = (size_t)nel;
#pragma unroll
  for (int k = 0; k < kThPack; ++k) a[k] = Ae[(size_t)k * st + e];
  int64_t nd[6];
  element_nodes(e, ncr, A, B, nd);
  double xv[6], yv[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    xv[i] = x[nd[i]];
    yv[i] = 0.0;
  }
  int k = 0;
#pragma unroll
  for (int i = 0; i < 6; ++i) {
#pragma unroll
    for (int j = i; j < 6; ++j, ++k) {
      yv[i] += a[k] * xv[j];
      if (j != i) yv[j] += a[k] * xv[i];
    }
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) atomicAdd(&y[nd[i]], yv[i]);
}

// r = b (free), 0 (walls); z = r / diag; p = z; x = 0; q = 0; sums r.z and b.b
__global__ void __launch_bounds__(kRedThreads) k_th_init(const double* __restrict__ b, const double* __restrict__ diag,
                                                         double* __restrict__ x, double* __restrict__ r,
                                                         double* __restrict__ z, double* __restrict__ pv,
                                                         double* __restrict__ q, int64_t n, int64_t A, int amax,
                                                         int heated, double* scal, double* partial,
                                                         unsigned int* counter, double rtol, double atol, int itmax) {
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool fx = th_fixed(i, A, amax, heated);
    const double ri = fx ? 0.0 : b[i];
    const double zi = fx ? 0.0 : ri / diag[i];
    x[i] = 0.0;
    r[i] = ri;
    z[i] = zi;
    pv[i] = zi;
    q[i] = 0.0;
    v[0] += ri * zi;
    v[1] += ri * ri;
  }
  double* outs[2] = {scal + TH_RZ, scal + TH_BB};
  if (grid_finish<2>(v, partial, counter, outs) && threadIdx.x == 0) {
    const double tol = atol + rtol * sqrt(scal[TH_BB]);
    scal[TH_TOL2] = tol * tol;
    scal[TH_RR] = scal[TH_BB];
    scal[TH_IT] = 0.0;
    scal[TH_ITMAX] = (double)itmax;
  }
}

// sets the loop's condition before its first pass
__global__ void k_th_start(cudaGraphConditionalHandle h, const double* scal) {
  grid_dep_wait();
  cudaGraphSetConditional(h, (scal[TH_RR] > scal[TH_TOL2] && scal[TH_ITMAX] >= 1.0) ? 1u : 0u);
}

__global__ void __launch_bounds__(kRedThreads) k_th_pq(const double* __restrict__ pv, const double* __restrict__ q,
                                                       int64_t n, double* scal, double* partial,
                                                       unsigned int* counter) {
  grid_dep_wait();
  double v[1] = {0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[0] += pv[i] * q[i];
  double* outs[1] = {scal + TH_PQ};
  if (grid_finish<1>(v, partial, counter, outs) && threadIdx.x == 0) scal[TH_ALPHA] = scal[TH_RZ] / scal[TH_PQ];
}

__global__ void __launch_bounds__(kRedThreads) k_th_update(double* __restrict__ x, double* __restrict__ r,
                                                           double* __restrict__ z, const double* __restrict__ pv,
                                                           const double* __restrict__ q,
                                                           const double* __restrict__ diag, int64_t n, int64_t A,
                                                           int amax, int heated, double* scal, double* partial,
                                                           unsigned int* counter, cudaGraphConditionalHandle h) {
  grid_dep_wait();
  const double alpha = scal[TH_ALPHA];
  double v[2] = {0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (th_fixed(i, A, amax, heated)) continue;
    x[i] += alpha * pv[i];
    const double ri = r[i] - alpha * q[i];
    const double zi = ri / diag[i];
    r[i] = ri;
    z[i] = zi;
    v[0] += ri * zi;
    v[1] += ri * ri;
  }
  double* outs[2] = {scal + TH_RZN, scal + TH_RR};
  if (grid_finish<2>(v, partial, counter, outs) && threadIdx.x == 0) {
    scal[TH_BETA] = scal[TH_RZN] / scal[TH_RZ];
    scal[TH_RZ] = scal[TH_RZN];
    const double it = scal[TH_IT] + 1.0;
    scal[TH_IT] = it;
    const double rr = scal[TH_RR];
    const bool go = isfinite(rr) && isfinite(scal[TH_ALPHA]) && rr > scal[TH_TOL2] && it < scal[TH_ITMAX];
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

__global__ void k_th_dir(double* __restrict__ pv, double* __restrict__ q, const double* __restrict__ z, int64_t n,
                         const double* scal) {
  grid_dep_wait();
  const double beta = scal[TH_BETA];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) {
    pv[i] = z[i] + beta * pv[i];
    q[i] = 0.0;
  }
}

// T = x + Tbc (free: x, walls: the prescribed value)
__global__ void k_th_finish(const double* __restrict__ x, const double* __restrict__ Tbc, double* __restrict__ T,
                            int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) T[i] = x[i] + Tbc[i];
}

// Tbc: lattice wall values
__global__ void k_th_bc(double* __restrict__ Tbc, int64_t n, int64_t A, int amax, int heated, double Ttop,
                        double Tbot) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int a = (int)(i % A);
  Tbc[i] = a == amax ? Ttop : ((heated && a == 0) ? Tbot : 0.0);
}

// thermal work vectors, nnod each, after the 21 x nel element blocks
enum ThVec { TV_TOLD = 0, TV_TBC, TV_DIAG, TV_B, TV_X, TV_R, TV_Z, TV_P, TV_Q, TV_STAGE, TV_COUNT };

static double* th_vec(Ctx& c, int k) { return c.th_buf + kThPack * c.fine.nel + (size_t)k * c.fine.nnod; }

static void th_emit_loop(Ctx& c, int heated) {
  const Level& L = c.fine;
  const int64_t n = L.nnod;
  const int amax = 2 * L.ncr;
  double *x = th_vec(c, TV_X), *r = th_vec(c, TV_R), *z = th_vec(c, TV_Z), *pv = th_vec(c, TV_P),
         *q = th_vec(c, TV_Q), *dg = th_vec(c, TV_DIAG);
  cudaGraphConditionalHandle h = new_handle(c.stream);
  klaunch(k_th_start, 1, 1, 0, c.stream, h, (const double*)c.scal);
  DP_LAUNCH_CHECK();
  cudaGraph_t body = add_while(c.stream, h);
  cudaStream_t aux = c.aux[0];
  DP_CUDA(cudaStreamBeginCaptureToGraph(aux, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  klaunch(k_th_apply, (int)div_up(L.nel, 128), 128, 0, aux, (const double*)c.th_buf, (const double*)pv, q, (int)L.nel,
          L.ncr, L.A(), L.B());
  klaunch(k_th_pq, red_grid(n), kRedThreads, 0, aux, (const double*)pv, (const double*)q, n, c.scal, c.partial,
          c.counter);
  klaunch(k_th_update, red_grid(n), kRedThreads, 0, aux, x, r, z, (const double*)pv, (const double*)q,
          (const double*)dg, n, L.A(), amax, heated, c.scal, c.partial, c.counter, h);
  klaunch(k_th_dir, (int)div_up(n, 256), 256, 0, aux, pv, q, (const double*)z, n, (const double*)c.scal);
  DP_LAUNCH_CHECK();
  cudaGraph_t out = nullptr;
  DP_CUDA(cudaStreamEndCapture(aux, &out));
}

void launch_th_apply_staged(Ctx& c) {
  const Level& L = c.fine;
  ++g_klaunch;
  k_th_apply<<<(int)div_up(L.nel, 128), 128, 0, c.stream>>>(c.th_buf, th_vec(c, TV_P), th_vec(c, TV_Q), (int)L.nel,
                                                             L.ncr, L.A(), L.B());
  DP_LAUNCH_CHECK();
}

}  // namespace dp

using namespace dp;

extern "C" void dp_default_thermal_opts(dp_thermal_opts* o) {
  if (!o) return;
  o->K = 3.3;
  o->Cp = 1.2e3;
  o->dt = 0.0;
  o->Ttop = 300.0;
  o->Tbot = 4000.0;
  o->rtol = 1.4901161193847656e-08;  // sqrt(eps), Krylov.jl's default
  o->atol = 1.4901161193847656e-08;
  o->heated = 1;
  o->itmax = 0;  // 0: the number of nodes (Krylov.jl's 2n cap for GMRES; CG needs far fewer)
}

extern "C" int dp_thermal_step(dp_ctx* h, const dp_thermal_opts* o, const double* rho_node, double* T,
                               int32_t* iterations, double* relres, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!o || !rho_node || !T) throw BadArg("null argument");
    if (!(o->dt >= 0.0) || !std::isfinite(o->dt)) throw BadArg("dt must be finite and >= 0");
    if (!(o->K >= 0.0) || !(o->Cp > 0.0)) throw BadArg("K must be >= 0 and Cp > 0");
    if (!(o->rtol >= 0.0) || !(o->atol >= 0.0)) throw BadArg("tolerances must be >= 0");
    if (o->itmax < 0) throw BadArg("itmax must be >= 0");
    const Level& L = c.fine;
    const int64_t nel = L.nel, nn = L.nnod;
    static bool uploaded[64] = {false};
    if (c.device < 0 || c.device >= 64 || !uploaded[c.device]) {
      upload_stress_constants();
      upload_rheology_constants();
      upload_thermal_constants();
      DP_CUDA(cudaDeviceSynchronize());  // the copies are on the default stream; ours does not wait on it
      if (c.device >= 0 && c.device < 64) uploaded[c.device] = true;
    }
    if (!c.th_buf) dalloc(&c.th_buf, kThPack * nel + TV_COUNT * nn);
    const int heated = o->heated ? 1 : 0;
    const int amax = 2 * L.ncr;
    double* Told = th_vec(c, TV_TOLD);
    double* Tbc = th_vec(c, TV_TBC);
    double* dg = th_vec(c, TV_DIAG);
    double* b = th_vec(c, TV_B);
    double* stage = th_vec(c, TV_STAGE);
    const cudaMemcpyKind kin = kind_in(mem);
    DP_CUDA(cudaMemcpyAsync(stage, T, sizeof(double) * nn, kin, c.stream));
    launch_gather_ref2lat(c, stage, Told, 1);
    DP_CUDA(cudaMemcpyAsync(stage, rho_node, sizeof(double) * nn, kin, c.stream));
    double* rho = th_vec(c, TV_X);  // x is initialised by k_th_init after the assembly
    launch_gather_ref2lat(c, stage, rho, 1);
    ++g_klaunch;
    k_th_bc<<<(int)div_up(nn, 256), 256, 0, c.stream>>>(Tbc, nn, L.A(), amax, heated, o->Ttop, o->Tbot);
    DP_CUDA(cudaMemsetAsync(dg, 0, sizeof(double) * nn, c.stream));
    DP_CUDA(cudaMemsetAsync(b, 0, sizeof(double) * nn, c.stream));
    ThAsmArgs a;
    a.theta_lat = c.theta_lat; a.r_lat = c.r_lat; a.rho_lat = rho; a.Told = Told; a.Tbc = Tbc;
    a.Ae = c.th_buf; a.diag = dg; a.b = b; a.K = o->K; a.Cp = o->Cp; a.dt = o->dt;
    a.nel = (int)nel; a.ncr = L.ncr; a.A = (int)L.A(); a.B = (int)L.B();
    ++g_klaunch;
    k_th_assemble<<<(int)div_up(nel, 128), 128, 0, c.stream>>>(a);
    DP_LAUNCH_CHECK();
    const int itmax = o->itmax > 0 ? o->itmax : (int)std::min<int64_t>(nn, INT32_MAX);
    ++g_klaunch;
    k_th_init<<<red_grid(nn), kRedThreads, 0, c.stream>>>(b, dg, th_vec(c, TV_X), th_vec(c, TV_R), th_vec(c, TV_Z),
                                                        th_vec(c, TV_P), th_vec(c, TV_Q), nn, L.A(), amax, heated,
                                                        c.scal, c.partial, c.counter, o->rtol, o->atol, itmax);
    DP_LAUNCH_CHECK();
    // the CG loop: one graph per context and wall configuration
    if (!c.th_exec || c.th_heated != heated) {
      if (c.th_exec) {
        cudaGraphExecDestroy((cudaGraphExec_t)c.th_exec);
        c.th_exec = nullptr;
      }
      ensure_ctl(c);  // the capture streams of loop bodies
      cudaGraph_t g = nullptr;
      DP_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
      try {
        PdlScope pdl(1);
        th_emit_loop(c, heated);
      } catch (...) {
        // leave the stream out of capture mode before reporting the error
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(c.stream, &partial);
        if (partial) cudaGraphDestroy(partial);
        cudaGetLastError();
        throw;
      }
      DP_CUDA(cudaStreamEndCapture(c.stream, &g));
      cudaGraphExec_t ex = nullptr;
      DP_CUDA(cudaGraphInstantiate(&ex, g, 0));
      cudaGraphDestroy(g);
      c.th_exec = ex;
      c.th_heated = heated;
    }
    DP_CUDA(cudaGraphLaunch((cudaGraphExec_t)c.th_exec, c.stream));
    ++g_klaunch;
    k_th_finish<<<(int)div_up(nn, 256), 256, 0, c.stream>>>(th_vec(c, TV_X), Tbc, stage, nn);
    DP_LAUNCH_CHECK();
    launch_scatter_lat2ref(c, stage, Told, 1);
    DP_CUDA(cudaMemcpyAsync(T, Told, sizeof(double) * nn, kind_out(mem), c.stream));
    DP_CUDA(cudaMemcpyAsync(c.h_scal, c.scal, sizeof(double) * 64, cudaMemcpyDeviceToHost, c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    const double it = c.h_scal[TH_IT];
    const double rel = c.h_scal[TH_BB] > 0.0 ? std::sqrt(c.h_scal[TH_RR] / c.h_scal[TH_BB]) : 0.0;
    if (iterations) *iterations = (int32_t)it;
    if (relres) *relres = rel;
    if (!std::isfinite(rel)) return (int)DP_BREAKDOWN;
    return (c.h_scal[TH_RR] > c.h_scal[TH_TOL2]) ? (int)DP_NOT_CONVERGED : (int)DP_OK;
  });
}
