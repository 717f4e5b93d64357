// Schur-complement PCG (outer) with an inner K-solve on the device.
//
// Outer loop: StokesPcCG, src/IterativeSolvers.jl:94-168, step for step:
//   U0 = K^-1 (F + G P0); r = -G^T U0; rm0space!(r); tol = ||r|| * rtol
//   d = r .* pc; q = d
//   repeat: rm0space!(q); rd = r.d; y = G q; z = K^-1 y; Sq = G^T z;
//           alpha = rd / q.Sq; P += alpha q; U += alpha z; r -= alpha Sq;
//           rm0space!(r); stop if ||r|| < tol and it >= itmin;
//           d = r .* pc; beta = (r - rlast).d / rd (Polak-Ribiere); q = d + beta q
// The scalars stay on the device (kernels read them from a scalar table); the
// host reads ||r||^2 and q.Sq once per outer iteration for the stopping test
// and the breakdown check (q.Sq <= 0 or non-finite -> DP_BREAKDOWN).
//
// Inner solve K z = y (the reference's LU back-substitution,
// PardisoSolvers.jl:274-278): PCG preconditioned with one V-cycle of the
// Galerkin multigrid (or point Jacobi), to ||y - K z|| <= inner_rtol ||y||.
// FP32-refined mode: FP64 iterative refinement around an FP32 PCG on the
// FP32 copy of Ke with an FP32 hierarchy -- the residual y - K z, the
// correction update and every outer-loop quantity stay FP64.
//
// Rigid-rotation removal: updatevelocity2 (StokesSolver.jl:170-184) with
// volume_integral (FSE.jl:412-464): omega = int rho u_theta / int rho r,
// u_theta -= omega r.
#include <cmath>
#include <vector>

#include "kernels.cuh"
#include "mg.cuh"
#include "reduce.cuh"
#include "solver.cuh"

namespace dp {

// scalar-table slots
enum Slot {
  S_RD = 0, S_QSQ = 1, S_SUMQ = 2, S_SUMR = 3, S_RR = 4, S_BNUM = 5,
  S_AM = 6, S_MOM = 7, S_TMP = 8, S_TMP2 = 9,
  S_RZ0 = 10, S_RZ1 = 11, S_PAP = 12, S_IRR = 13, S_YY = 14,
};

static int nb256(int64_t n) { return (int)div_up(n, 256); }

// ---- outer vector kernels -----------------------------------------------------
__global__ void k_sub_mean(double* __restrict__ a, int64_t n, const double* __restrict__ sum) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] -= *sum / (double)n;
}

// rlast = r; alpha = rd/qSq; P += alpha q; r -= alpha Sq; sum(r) -> scal[S_SUMR]
__global__ void __launch_bounds__(kRedThreads) k_schur_update_p(double* __restrict__ P, double* __restrict__ r,
                                                                 double* __restrict__ rlast, const double* __restrict__ q,
                                                                 const double* __restrict__ Sq, int64_t n,
                                                                 double* scal, double* partial, unsigned int* counter) {
  grid_dep_wait();
  const double alpha = scal[S_RD] / scal[S_QSQ];
  DD s{0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    const double ri = r[i];
    rlast[i] = ri;
    P[i] += alpha * q[i];
    const double rn = ri - alpha * Sq[i];
    r[i] = rn;
    dd_add(s, rn);
  }
  DD v[1] = {s};
  double* o[1] = {scal + S_SUMR};
  grid_finish_dd<1>(v, partial, counter, o);
}

__global__ void k_axpy_slot(double* __restrict__ U, const double* __restrict__ z, int64_t n, const double* scal) {
  grid_dep_wait();
  const double alpha = scal[S_RD] / scal[S_QSQ];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) U[i] += alpha * z[i];
}

// r -= mean(r); d = r*pc; ||r||^2 -> S_RR; (r - rlast).d -> S_BNUM
__global__ void __launch_bounds__(kRedThreads) k_schur_center(double* __restrict__ r, const double* __restrict__ rlast,
                                                               const double* __restrict__ pc, double* __restrict__ d,
                                                               int64_t n, double* scal, double* partial,
                                                               unsigned int* counter) {
  grid_dep_wait();
  const double m = scal[S_SUMR] / (double)n;
  DD s0{0.0, 0.0}, s1{0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    const double ri = r[i] - m;
    r[i] = ri;
    const double di = ri * pc[i];
    d[i] = di;
    dd_add_prod(s0, ri, ri);
    dd_add_prod(s1, ri - rlast[i], di);
  }
  DD v[2] = {s0, s1};
  double* o[2] = {scal + S_RR, scal + S_BNUM};
  grid_finish_dd<2>(v, partial, counter, o);
}

// Element-block mass preconditioner (discontinuous pressure): d_e = M_e^-1 r_e.
__global__ void k_mass_blk(const double* __restrict__ r, const double* __restrict__ Minv, double* __restrict__ d,
                           int nel) {
  grid_dep_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  const double r0 = r[3 * (size_t)e], r1 = r[3 * (size_t)e + 1], r2 = r[3 * (size_t)e + 2];
  const double a = Minv[e], b = Minv[nel + e], c = Minv[2 * (size_t)nel + e];
  const double dd = Minv[3 * (size_t)nel + e], f = Minv[4 * (size_t)nel + e], g = Minv[5 * (size_t)nel + e];
  d[3 * (size_t)e] = a * r0 + b * r1 + c * r2;
  d[3 * (size_t)e + 1] = b * r0 + dd * r1 + f * r2;
  d[3 * (size_t)e + 2] = c * r0 + f * r1 + g * r2;
}

// k_schur_center with d = M^-1 r per element block
__global__ void __launch_bounds__(kRedThreads) k_schur_center_blk(double* __restrict__ r, const double* __restrict__ rlast,
                                                                   const double* __restrict__ Minv, double* __restrict__ d,
                                                                   int nel, double* scal, double* partial,
                                                                   unsigned int* counter) {
  grid_dep_wait();
  const double m = scal[S_SUMR] / (3.0 * (double)nel);
  DD s0{0.0, 0.0}, s1{0.0, 0.0};
  for (int e = blockIdx.x * kRedThreads + threadIdx.x; e < nel; e += gridDim.x * kRedThreads) {
    double rv[3];
    for (int k = 0; k < 3; ++k) {
      rv[k] = r[3 * (size_t)e + k] - m;
      r[3 * (size_t)e + k] = rv[k];
    }
    const double a = Minv[e], b = Minv[nel + e], c = Minv[2 * (size_t)nel + e];
    const double dd = Minv[3 * (size_t)nel + e], f = Minv[4 * (size_t)nel + e], g = Minv[5 * (size_t)nel + e];
    const double dv[3] = {a * rv[0] + b * rv[1] + c * rv[2], b * rv[0] + dd * rv[1] + f * rv[2],
                          c * rv[0] + f * rv[1] + g * rv[2]};
    for (int k = 0; k < 3; ++k) {
      d[3 * (size_t)e + k] = dv[k];
      dd_add_prod(s0, rv[k], rv[k]);
      dd_add_prod(s1, rv[k] - rlast[3 * (size_t)e + k], dv[k]);
    }
  }
  DD v[2] = {s0, s1};
  double* o[2] = {scal + S_RR, scal + S_BNUM};
  grid_finish_dd<2>(v, partial, counter, o);
}

// q = d + beta q, beta = BNUM / RD; sum(q) -> S_SUMQ (for the next rm0space!)
__global__ void __launch_bounds__(kRedThreads) k_q_update(double* __restrict__ q, const double* __restrict__ d, int64_t n,
                                                           double* scal, double* partial, unsigned int* counter) {
  grid_dep_wait();
  const double beta = scal[S_BNUM] / scal[S_RD];
  DD s{0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    const double qi = d[i] + beta * q[i];
    q[i] = qi;
    dd_add(s, qi);
  }
  DD v[1] = {s};
  double* o[1] = {scal + S_SUMQ};
  grid_finish_dd<1>(v, partial, counter, o);
}

// q -= mean(q); rd = r.d -> S_RD
__global__ void __launch_bounds__(kRedThreads) k_q_center_rd(double* __restrict__ q, const double* __restrict__ r,
                                                              const double* __restrict__ d, int64_t n, double* scal,
                                                              double* partial, unsigned int* counter) {
  grid_dep_wait();
  const double m = scal[S_SUMQ] / (double)n;
  DD s{0.0, 0.0};
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    q[i] -= m;
    dd_add_prod(s, r[i], d[i]);
  }
  DD v[1] = {s};
  double* o[1] = {scal + S_RD};
  grid_finish_dd<1>(v, partial, counter, o);
}

__global__ void k_mul_into(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                           int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] * b[i];
}
__global__ void k_neg(double* __restrict__ a, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) a[i] = -a[i];
}
__global__ void k_add(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i] + b[i];
}

// ---- inner PCG kernels (templated on the vector precision) --------------------
// x += alpha p; r -= alpha Ap; alpha = scal[rz]/scal[pAp]; ||r||^2 -> scal[S_IRR]
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_pcg_update(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                                                             const T* __restrict__ Ap, int64_t n, double* scal, int rz_slot,
                                                             double* partial, unsigned int* counter) {
  grid_dep_wait();
  const double pap = scal[S_PAP];
  const double alpha = (pap > 0.0 && isfinite(pap)) ? scal[rz_slot] / pap : 0.0;   // breakdown: no update
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    x[i] += (T)(alpha * (double)p[i]);
    const T ri = (T)((double)r[i] - alpha * (double)Ap[i]);
    r[i] = ri;
    s += (double)ri * (double)ri;
  }
  double v[1] = {s};
  double* o[1] = {scal + S_IRR};
  grid_finish<1>(v, partial, counter, o);
}

// p = z + beta p, beta = scal[new]/scal[old]
template <typename T>
__global__ void k_pcg_dir(T* __restrict__ p, const T* __restrict__ z, int64_t n, const double* scal, int new_slot,
                          int old_slot) {
  grid_dep_wait();
  const double beta = scal[new_slot] / scal[old_slot];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = (T)((double)z[i] + beta * (double)p[i]);
}


__global__ void k_f32_to_f64(const float* __restrict__ a, double* __restrict__ b, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}
__global__ void k_bj_host_mixed(const float* __restrict__ dinv, const double* __restrict__ r, double* __restrict__ z,
                                int64_t nnod) {
  grid_dep_wait();
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnod) return;
  double z0, z1;
  bj_apply<float>(dinv, n, r[2 * n], r[2 * n + 1], z0, z1);
  z[2 * n] = z0;
  z[2 * n + 1] = z1;
}

template <typename T>
__global__ void k_scale_copy(const double* __restrict__ a, T* __restrict__ b, double s, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) b[i] = (T)(s * a[i]);
}
template <typename T>
__global__ void k_add_scaled(double* __restrict__ z, const T* __restrict__ e, double s, int64_t n) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) z[i] += s * (double)e[i];
}
__global__ void k_residual(const double* __restrict__ y, double* __restrict__ Kz, int64_t n) {  // Kz <- y - Kz
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) Kz[i] = y[i] - Kz[i];
}

template <typename T>
static void dot_t(Ctx& c, const T* a, const T* b, int64_t n, int slot);
template <>
void dot_t<double>(Ctx& c, const double* a, const double* b, int64_t n, int slot) { launch_dot(c, a, b, n, slot); }
template <>
void dot_t<float>(Ctx& c, const float* a, const float* b, int64_t n, int slot) { launch_dot_f(c, a, b, n, slot); }

static double read_slot(Ctx& c, int slot) {
  DP_CUDA(cudaMemcpyAsync(c.h_scal + slot, c.scal + slot, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
  DP_CUDA(cudaStreamSynchronize(c.stream));
  return c.h_scal[slot];
}
static void read_slots(Ctx& c, int first, int count) {
  DP_CUDA(cudaMemcpyAsync(c.h_scal + first, c.scal + first, sizeof(double) * count, cudaMemcpyDeviceToHost, c.stream));
  DP_CUDA(cudaStreamSynchronize(c.stream));
}

// Preconditioned CG on the masked K (precision T), x = 0 start.
// Work vectors: r, z, p, Ap (T, length n).  Returns iterations.
template <typename T>
static int pcg(Ctx& c, const T* Kmat, const T* b, T* x, T* r, T* z, T* p, T* Ap, double rtol, int itmax,
               int pc_kind, const MGOptions& mgo, double* out_relres) {
  const Level& L = c.fine;
  const int64_t n = 2 * L.nnod;
  DP_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * n, c.stream));
  DP_CUDA(cudaMemcpyAsync(r, b, sizeof(T) * n, cudaMemcpyDeviceToDevice, c.stream));
  dot_t<T>(c, b, b, n, S_YY);
  const double bb = read_slot(c, S_YY);
  if (!(bb > 0.0)) {
    if (out_relres) *out_relres = 0.0;
    return 0;
  }
  const double tol2 = rtol * rtol * bb;
  auto precond = [&](const T* rin, T* zout) {
    if (pc_kind == 0) {
      if (std::is_same<T, double>::value && c.mg_prec == 1) {
        // FP64 vectors, FP32 hierarchy: unscaled conversion (host loop is a debugging path)
        float* r32 = (float*)c.work[W_F_R];
        float* z32 = (float*)c.work[W_F_Z];
        klaunch(k_scale_copy<float>, nb256(n), 256, 0, c.stream, (const double*)rin, r32, 1.0, n);
        mg_apply_f(c, r32, z32, mgo);
        klaunch(k_f32_to_f64, nb256(n), 256, 0, c.stream, z32, (double*)zout, n);
      } else if (std::is_same<T, double>::value) {
        mg_apply(c, (const double*)rin, (double*)zout, mgo);
      } else {
        mg_apply_f(c, (const float*)rin, (float*)zout, mgo);
      }
    } else if (c.mg_prec == 1 && std::is_same<T, double>::value) {
      klaunch(k_bj_host_mixed, nb256(L.nnod), 256, 0, c.stream, c.mg[0].dinv32, (const double*)rin, (double*)zout, L.nnod);
    } else {
      const T* dinv = std::is_same<T, double>::value ? (const T*)c.mg[0].dinv64 : (const T*)c.mg[0].dinv32;
      klaunch(k_bj<T>, nb256(L.nnod), 256, 0, c.stream, dinv, rin, zout, L.nnod);
    }
  };
  precond(r, z);
  DP_CUDA(cudaMemcpyAsync(p, z, sizeof(T) * n, cudaMemcpyDeviceToDevice, c.stream));
  dot_t<T>(c, r, z, n, S_RZ0);
  int it = 0;
  double rr = bb;
  for (it = 1; it <= itmax; ++it) {
    const int cur = (it & 1) ? S_RZ0 : S_RZ1;
    const int nxt = (it & 1) ? S_RZ1 : S_RZ0;
    launch_apply_K<T, T>(L, Kmat, p, Ap, c.stream);
    dot_t<T>(c, p, Ap, n, S_PAP);
    klaunch(k_pcg_update<T>, red_grid(n), kRedThreads, 0, c.stream, x, r, p, Ap, n, c.scal, cur, c.partial, c.counter);
    DP_LAUNCH_CHECK();
    rr = read_slot(c, S_IRR);
    if (!std::isfinite(rr)) break;
    if (rr <= tol2) break;
    precond(r, z);
    dot_t<T>(c, r, z, n, nxt);
    klaunch(k_pcg_dir<T>, nb256(n), 256, 0, c.stream, p, z, n, c.scal, nxt, cur);
    DP_LAUNCH_CHECK();
  }
  if (out_relres) *out_relres = std::sqrt(rr / bb);
  return std::min(it, itmax);
}

// Inner solve K z = y (FP64 in/out).
int inner_solve(Ctx& c, const double* y, double* z, const SolveCfg& cfg, InnerStats& st) {
  const Level& L = c.fine;
  const int64_t n = 2 * L.nnod;
  double* w = (double*)c.work[W_IN_R];
  double* wz = (double*)c.work[W_IN_Z];
  double* wp = (double*)c.work[W_IN_P];
  double* wAp = (double*)c.work[W_IN_AP];
  if (cfg.precision <= 1) {
    double rel = 0.0;
    const int its = pcg<double>(c, c.K64, y, z, w, wz, wp, wAp, cfg.inner_rtol, cfg.inner_itmax, cfg.inner_pc, cfg.mg,
                                &rel);
    st.its += its;
    st.last_relres = rel;
    return its;
  }
  // FP32-refined: z = 0; res = y; repeat { e = K32^-1 (res/s) ; z += s e; res = y - K64 z }
  float* fb = (float*)c.work[W_F_B];
  float* fx = (float*)c.work[W_F_X];
  float* fr = (float*)c.work[W_F_R];
  float* fz = (float*)c.work[W_F_Z];
  float* fp = (float*)c.work[W_F_P];
  float* fAp = (float*)c.work[W_F_AP];
  double* res = (double*)c.work[W_RES];
  DP_CUDA(cudaMemsetAsync(z, 0, sizeof(double) * n, c.stream));
  DP_CUDA(cudaMemcpyAsync(res, y, sizeof(double) * n, cudaMemcpyDeviceToDevice, c.stream));
  launch_dot(c, y, y, n, S_TMP);
  const double yy = read_slot(c, S_TMP);
  if (!(yy > 0.0)) { st.last_relres = 0.0; return 0; }
  double rel = 1.0;
  int total = 0;
  for (int ref = 0; ref < cfg.max_refine; ++ref) {
    const double s = std::sqrt(rel * rel * yy);
    klaunch(k_scale_copy<float>, nb256(n), 256, 0, c.stream, res, fb, 1.0 / s, n);
    double rel32 = 0.0;
    total += pcg<float>(c, c.K32, fb, fx, fr, fz, fp, fAp, cfg.inner_rtol32, cfg.inner_itmax, cfg.inner_pc, cfg.mg,
                        &rel32);
    klaunch(k_add_scaled<float>, nb256(n), 256, 0, c.stream, z, fx, s, n);
    launch_apply_K<double, double>(L, c.K64, z, res, c.stream);
    klaunch(k_residual, nb256(n), 256, 0, c.stream, y, res, n);
    DP_LAUNCH_CHECK();
    launch_dot(c, res, res, n, S_TMP);
    rel = std::sqrt(read_slot(c, S_TMP) / yy);
    if (!(rel > cfg.inner_rtol)) break;
  }
  st.its += total;
  st.last_relres = rel;
  return total;
}

// ---- rigid-rotation removal ----------------------------------------------------
// per element: sum_ip (N . V_el) * r_ip * detJ * w_ip with V = Uth*rho (am) and r*rho (mom)
__global__ void __launch_bounds__(kRedThreads) k_rot_integrals(const double* __restrict__ U, const double* __restrict__ rho,
                                                                const double* __restrict__ th_lat,
                                                                const double* __restrict__ r_lat, int nel, int ncr, int A,
                                                                int B, double* scal, double* partial,
                                                                unsigned int* counter) {
  grid_dep_wait();
  DD am{0.0, 0.0}, mom{0.0, 0.0};
  for (int e = blockIdx.x * kRedThreads + threadIdx.x; e < nel; e += gridDim.x * kRedThreads) {
    int nd[6];
    element_nodes_mg(e, ncr, A, B, nd);
    double th[3], rr[3];
    for (int k = 0; k < 3; ++k) { th[k] = th_lat[nd[k]]; rr[k] = r_lat[nd[k]]; }
    const double PI = 3.14159265358979323846;
    if (fabs(th[0] - th[1]) + fabs(th[1] - th[2]) + fabs(th[2] - th[0]) > PI)
      for (int k = 0; k < 3; ++k)
        if (th[k] < PI) th[k] += 2.0 * PI;
    const double detJ = (th[1] - th[0]) * (rr[2] - rr[0]) - (th[2] - th[0]) * (rr[1] - rr[0]);
    double va[6], vm[6];
    for (int k = 0; k < 6; ++k) {
      va[k] = U[2 * nd[k]] * rho[nd[k]];
      vm[k] = r_lat[nd[k]] * rho[nd[k]];
    }
    for (int ip = 0; ip < 6; ++ip) {
      const double r_ip = rr[0] * c_N3[ip][0] + rr[1] * c_N3[ip][1] + rr[2] * c_N3[ip][2];
      const double om = r_ip * detJ * c_w[ip];
      double sa = 0.0, sm = 0.0;
      for (int k = 0; k < 6; ++k) { sa += va[k] * c_N[ip][k]; sm += vm[k] * c_N[ip][k]; }
      dd_add_prod(am, sa, om);
      dd_add_prod(mom, sm, om);
    }
  }
  DD v[2] = {am, mom};
  double* o[2] = {scal + S_AM, scal + S_MOM};
  grid_finish_dd<2>(v, partial, counter, o);
}

__global__ void k_rot_remove(double* __restrict__ U, const double* __restrict__ r_lat, int64_t nnod, const double* scal) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nnod) return;
  const double om = scal[S_AM] / scal[S_MOM];
  U[2 * i] -= om * r_lat[i];
}

// U_cart = TT U per node: [c s; -s c] (StokesSolver.jl:159, :214-241)
__global__ void k_to_cartesian(const double* __restrict__ U, const double* __restrict__ th, double* __restrict__ Uc,
                               int64_t nnod) {
  grid_dep_wait();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nnod) return;
  double s, c;
  sincos(th[i], &s, &c);
  const double ut = U[2 * i], ur = U[2 * i + 1];
  Uc[2 * i] = c * ut + s * ur;
  Uc[2 * i + 1] = -s * ut + c * ur;
}

// ---- the full solve ---------------------------------------------------------------
int schur_pcg(Ctx& c, const SolveCfg& cfg, double* U, double* P, SolveResult& res) {
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
  InnerStats st;

  // Rhs = F + G P ; U = K^-1 Rhs   (IterativeSolvers.jl:101-111)
  // Pressure gauge: constant pressure is in the null space of G under free slip,
  // so P is defined up to a constant.  StokesPcCG starts from P = 0 and adds
  // only mean-free directions (IterativeSolvers.jl:101, rm0space! of q), so its
  // P has zero mean; a given initial P (a guess) has its mean removed first so
  // that the answer carries the same gauge.  It changes nothing else (G 1 = 0).
  if (!cfg.use_guess) {
    DP_CUDA(cudaMemsetAsync(P, 0, sizeof(double) * nP, c.stream));
  } else {
    launch_sum_c(c, P, nP, S_TMP2);
    klaunch(k_sub_mean, nb256(nP), 256, 0, c.stream, P, nP, (const double*)(c.scal + S_TMP2));
  }
  launch_apply_G(c, P, y);
  klaunch(k_add, nb256(nU), 256, 0, c.stream, c.F, y, rhs, nU);
  DP_LAUNCH_CHECK();
  inner_solve(c, rhs, U, cfg, st);
  // r = -G^T U; rm0space!(r)
  launch_apply_GT(c, U, r);
  klaunch(k_neg, nb256(nP), 256, 0, c.stream, r, nP);
  launch_sum_c(c, r, nP, S_SUMR);
  klaunch(k_sub_mean, nb256(nP), 256, 0, c.stream, r, nP, c.scal + S_SUMR);
  launch_dot_c(c, r, r, nP, S_RR);
  DP_LAUNCH_CHECK();
  const double r0 = std::sqrt(read_slot(c, S_RR));
  res.r0 = r0;
  if (!std::isfinite(r0)) {   // the initial inner solve failed: breakdown, not a zero residual
    res.status = 2;
    res.iterations = 0;
    res.relres = r0;
    res.inner_its = st.its;
    return res.status;
  }
  const double tol = r0 * cfg.rtol;
  // d = r .* pc (or M^-1 r); q = d
  if (cfg.schur_pc == 1) {
    klaunch(k_mass_blk, nb256(L.nel), 256, 0, c.stream, r, c.Minv, d, (int)L.nel);
  } else {
    klaunch(k_mul_into, nb256(nP), 256, 0, c.stream, r, c.pc, d, nP);
  }
  DP_CUDA(cudaMemcpyAsync(q, d, sizeof(double) * nP, cudaMemcpyDeviceToDevice, c.stream));
  launch_sum_c(c, q, nP, S_SUMQ);
  res.status = 1;  // not converged until shown otherwise
  res.iterations = 0;
  double rnorm = r0;
  if (r0 == 0.0) res.status = 0;
  for (int it = 1; it <= cfg.itmax && r0 > 0.0; ++it) {
    // rm0space!(q); rd = r.d
    klaunch(k_q_center_rd, red_grid(nP), kRedThreads, 0, c.stream, q, r, d, nP, c.scal, c.partial, c.counter);
    // y = G q ; z = K^-1 y ; Sq = G^T z ; qSq
    launch_apply_G(c, q, y);
    inner_solve(c, y, z, cfg, st);
    launch_apply_GT(c, z, Sq);
    launch_dot_c(c, q, Sq, nP, S_QSQ);
    // P += alpha q; U += alpha z; r -= alpha Sq
    klaunch(k_schur_update_p, red_grid(nP), kRedThreads, 0, c.stream, P, r, rlast, q, Sq, nP, c.scal, c.partial, c.counter);
    klaunch(k_axpy_slot, nb256(nU), 256, 0, c.stream, U, z, nU, c.scal);
    // rm0space!(r); d = r .* pc; ||r||; (r - rlast).d
    if (cfg.schur_pc == 1)
      klaunch(k_schur_center_blk, red_grid(L.nel), kRedThreads, 0, c.stream, r, rlast, c.Minv, d, (int)L.nel, c.scal,
                                                                         c.partial, c.counter);
    else
      klaunch(k_schur_center, red_grid(nP), kRedThreads, 0, c.stream, r, rlast, c.pc, d, nP, c.scal, c.partial, c.counter);
    DP_LAUNCH_CHECK();
    read_slots(c, 0, 6);
    const double qSq = c.h_scal[S_QSQ], rd = c.h_scal[S_RD];
    rnorm = std::sqrt(c.h_scal[S_RR]);
    res.iterations = it;
    if (cfg.verbose >= 2)
      std::fprintf(stderr, "[dp] it %d ||r||/r0 %.3e inner its %lld (rel %.2e)\n", it, rnorm / r0,
                   (long long)st.its, st.last_relres);
    if (!(qSq > 0.0) || !std::isfinite(qSq) || !std::isfinite(rd) || !std::isfinite(rnorm)) {
      res.status = 2;
      break;
    }
    if (rnorm < tol && it >= cfg.itmin) {
      res.status = 0;
      break;
    }
    // q = d + beta q
    klaunch(k_q_update, red_grid(nP), kRedThreads, 0, c.stream, q, d, nP, c.scal, c.partial, c.counter);
    DP_LAUNCH_CHECK();
  }
  res.relres = r0 > 0.0 ? rnorm / r0 : 0.0;
  res.inner_its = st.its;

  // residual diagnostics on the raw solution: ||K U - F - G P|| / ||F||, ||G^T U||
  launch_apply_K<double, double>(L, c.K64, U, rhs, c.stream);   // rhs <- K U
  launch_apply_G(c, P, y);                                      // y <- G P
  klaunch(k_add, nb256(nU), 256, 0, c.stream, c.F, y, y, nU);        // y <- F + G P
  klaunch(k_residual, nb256(nU), 256, 0, c.stream, y, rhs, nU);      // rhs <- F + G P - K U
  DP_LAUNCH_CHECK();
  launch_dot(c, rhs, rhs, nU, S_TMP);
  launch_dot(c, c.F, c.F, nU, S_TMP2);
  read_slots(c, S_TMP, 2);
  res.mom_residual = std::sqrt(c.h_scal[S_TMP] / std::max(c.h_scal[S_TMP2], 1e-300));
  launch_apply_GT(c, U, Sq);
  launch_sum_c(c, Sq, nP, S_SUMR);
  klaunch(k_sub_mean, nb256(nP), 256, 0, c.stream, Sq, nP, c.scal + S_SUMR);
  launch_dot_c(c, Sq, Sq, nP, S_TMP);
  res.div_residual = r0 > 0.0 ? std::sqrt(read_slot(c, S_TMP)) / r0 : 0.0;

  // rigid-rotation removal (updatevelocity2)
  res.omega = 0.0;
  if (cfg.remove_rotation) {
    klaunch(k_rot_integrals, red_grid(L.nel), kRedThreads, 0, c.stream, U, c.rho_lat, c.theta_lat, c.r_lat, (int)L.nel, L.ncr,
                                                                   (int)L.A(), (int)L.B(), c.scal, c.partial, c.counter);
    klaunch(k_rot_remove, nb256(L.nnod), 256, 0, c.stream, U, c.r_lat, L.nnod, c.scal);
    DP_LAUNCH_CHECK();
    read_slots(c, S_AM, 2);
    res.omega = c.h_scal[S_AM] / c.h_scal[S_MOM];
  }
  return res.status;
}

void to_cartesian(Ctx& c, const double* U, double* Uc) {
  klaunch(k_to_cartesian, nb256(c.fine.nnod), 256, 0, c.stream, U, c.theta_lat, Uc, c.fine.nnod);
  DP_LAUNCH_CHECK();
}

}  // namespace dp
