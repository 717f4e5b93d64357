// Per-IP viscosity update, Arrhenius law with Drucker-Prager plasticity:
// getviscosity!(::Arrhenius, T, P, epsII, tauII, e2n, r) (src/Rheology/
// Rheology.jl:348-403), the producer of the eta.ip the Stokes assembly reads.
//
// One thread per element, 7-point IPs (Quadrature.jl:109-138): T_ip and the
// radius z_ip by the P2 shape functions, P_ip by the linear ones at the three
// vertices plus |min P| (a device reduction), a depth factor lambda (1e1
// between max r - 2780 km and max r - 660 km, 1e-3 below, 1e0 above), eta_TP =
// clamp(lambda eta0 exp((Ea + P Va) / (R T) - Ea / (R T0)), 1e18, 1e25)
// (getviscosity :171-173).  Where cohesion, friction angle and epsII are all
// non-zero the plastic branch applies: yield stress cosd(phi) C + sind(phi) P
// (druckerPrager :338-344) and, if it is below tauII, eta = clamp(tau_y /
// (2 epsII), 1e18, 1e25); otherwise the previous eta is kept, as the
// reference does.  eta is read and written in place.
#include "kernels.cuh"
#include "reduce.cuh"

namespace dp {

constexpr int S_MINP = 40, S_MAXR = 41;  // scalar-table slots of the two reductions

__constant__ double c_N6s[7][6];  // P2 N at the 7 IPs (sf_N_tri6, Quadrature.jl:264-285)

static void upload_rheology_constants() {
  double N6[7][6];
  const double g1 = (6.0 - std::sqrt(15.0)) / 21.0, g2 = (6.0 + std::sqrt(15.0)) / 21.0;
  const double ip[7][2] = {{1.0 / 3.0, 1.0 / 3.0}, {1.0 - 2.0 * g1, g1}, {g1, 1.0 - 2.0 * g1}, {g1, g1},
                           {1.0 - 2.0 * g2, g2},   {g2, 1.0 - 2.0 * g2}, {g2, g2}};
  for (int q = 0; q < 7; ++q) {
    const double r = ip[q][0], s = ip[q][1], t = 1.0 - r - s;
    const double n[6] = {t * (2.0 * t - 1.0), r * (2.0 * r - 1.0), s * (2.0 * s - 1.0),
                         4.0 * r * t, 4.0 * r * s, 4.0 * s * t};
    for (int k = 0; k < 6; ++k) N6[q][k] = n[k];
  }
  DP_CUDA(cudaMemcpyToSymbol(c_N6s, N6, sizeof(N6)));
}

// per-block min of P and max of r -> partial[b], partial[nb + b]
__global__ void __launch_bounds__(kRedThreads) k_minmax_partial(const double* __restrict__ P, int64_t np,
                                                                const double* __restrict__ r, int64_t nn,
                                                                double* __restrict__ partial) {
  double mn = INFINITY, mx = -INFINITY;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += (int64_t)gridDim.x * blockDim.x)
    mn = fmin(mn, P[i]);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x)
    mx = fmax(mx, r[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  __shared__ double smn[kRedThreads / 32], smx[kRedThreads / 32];
  if ((threadIdx.x & 31) == 0) {
    smn[threadIdx.x >> 5] = mn;
    smx[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kRedThreads / 32; ++w) {
      mn = fmin(mn, smn[w]);
      mx = fmax(mx, smx[w]);
    }
    partial[blockIdx.x] = mn;
    partial[gridDim.x + blockIdx.x] = mx;
  }
}

__global__ void k_minmax_final(const double* __restrict__ partial, int nb, double* __restrict__ scal) {
  double mn = INFINITY, mx = -INFINITY;
  for (int b = 0; b < nb; ++b) {
    mn = fmin(mn, partial[b]);
    mx = fmax(mx, partial[nb + b]);
  }
  scal[S_MINP] = fabs(mn);
  scal[S_MAXR] = mx;
}

struct ArrheniusArgs {
  double eta0, R, Ea, Va, T0, sphi, cphi, phi;
};

// T, P (vertex entries; others unused), r: lattice order.  epsII, tauII, coh,
// eta: nel x 7 element-fastest.
__global__ void __launch_bounds__(128) k_viscosity_arrhenius(const double* __restrict__ T, const double* __restrict__ P,
                                                             const double* __restrict__ r,
                                                             const double* __restrict__ epsII,
                                                             const double* __restrict__ tauII,
                                                             const double* __restrict__ coh, double* __restrict__ eta,
                                                             const double* __restrict__ scal, ArrheniusArgs law,
                                                             int nel, int ncr, int A, int B) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  int64_t nd[6];
  element_nodes(e, ncr, A, B, nd);
  double Te[6], re[6], Pe[3];
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    Te[k] = T[nd[k]];
    re[k] = r[nd[k]];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) Pe[k] = P[nd[k]];
  const double minP = scal[S_MINP], maxr = scal[S_MAXR];
  const size_t st = (size_t)nel;
  for (int ip = 0; ip < 7; ++ip) {
    double T_ip = 0.0, z_ip = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      T_ip += Te[k] * c_N6s[ip][k];
      z_ip += re[k] * c_N6s[ip][k];
    }
    const double P_ip = Pe[0] * c_N3s[ip][0] + Pe[1] * c_N3s[ip][1] + Pe[2] * c_N3s[ip][2] + minP;
    const double lam = z_ip < maxr - 2780e3 ? 1e-3 : (z_ip > maxr - 660e3 ? 1e0 : 1e1);
    const double etaTP =
        fmin(fmax(lam * law.eta0 * exp((law.Ea + P_ip * law.Va) / law.R / T_ip - law.Ea / law.R / law.T0), 1e18), 1e25);
    const size_t i = (size_t)ip * st + e;
    const double e2 = epsII[i], c = coh[i];
    if (c > 0.0 && law.phi > 0.0 && e2 != 0.0) {
      const double tau_y = law.cphi * c + law.sphi * P_ip;
      if (tau_y < tauII[i]) eta[i] = fmax(1e18, fmin(1e25, 0.5 * tau_y / e2));
    } else {
      eta[i] = etaTP;
    }
  }
}

// k_viscosity_arrhenius on the inputs staged by the last dp_viscosity_arrhenius
// call (kernel timing; eta is updated in place, and a second pass over it
// writes the same values).
void launch_viscosity_staged(Ctx& c) {
  const int64_t nel = c.fine.nel, nn = c.fine.nnod;
  double* e2 = c.rheo_buf;
  double* Tl = e2 + 28 * nel;
  ArrheniusArgs a;
  a.eta0 = c.rheo_law[0]; a.R = c.rheo_law[1]; a.Ea = c.rheo_law[2]; a.Va = c.rheo_law[3];
  a.T0 = c.rheo_law[4]; a.sphi = c.rheo_law[5]; a.cphi = c.rheo_law[6]; a.phi = c.rheo_law[7];
  ++g_klaunch;
  k_viscosity_arrhenius<<<(int)div_up(nel, 128), 128, 0, c.stream>>>(Tl, Tl + nn, Tl + 2 * nn, e2, e2 + 7 * nel,
                                                                      e2 + 14 * nel, e2 + 21 * nel, c.scal, a,
                                                                      (int)nel, c.fine.ncr, (int)c.fine.A(),
                                                                      (int)c.fine.B());
  DP_LAUNCH_CHECK();
}

}  // namespace dp

using namespace dp;

extern "C" int dp_viscosity_arrhenius(dp_ctx* h, const dp_arrhenius* law, const double* T_node, const double* P_vertex,
                                      int64_t nvert, const double* r_node, const double* epsII, const double* tauII,
                                      const double* cohesion, double* eta_ip, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!law || !T_node || !P_vertex || !r_node || !epsII || !tauII || !cohesion || !eta_ip)
      throw BadArg("null argument");
    const int64_t nel = c.fine.nel, nn = c.fine.nnod;
    const int64_t nv = (int64_t)(c.fine.ncr + 1) * c.fine.nct;
    if (nvert != nv) throw BadArg("P_vertex must hold the " + std::to_string(nv) + " vertex values");
    if (!(law->T0 > 0.0) || !(law->R > 0.0)) throw BadArg("T0 and R must be positive");
    static bool uploaded[64] = {false};
    if (c.device < 0 || c.device >= 64 || !uploaded[c.device]) {
      upload_rheology_constants();
      upload_stress_constants();
      DP_CUDA(cudaDeviceSynchronize());  // the copies are on the default stream; ours does not wait on it
      if (c.device >= 0 && c.device < 64) uploaded[c.device] = true;
    }
    if (!c.rheo_buf) dalloc(&c.rheo_buf, 28 * nel + 4 * nn);
    double* e2 = c.rheo_buf;
    double* t2 = e2 + 7 * nel;
    double* co = t2 + 7 * nel;
    double* et = co + 7 * nel;
    double* Tl = et + 7 * nel;
    double* Pl = Tl + nn;
    double* rl = Pl + nn;
    double* stage = rl + nn;  // nnod: reference-numbered input before the permutation
    const cudaMemcpyKind kin = kind_in(mem);
    DP_CUDA(cudaMemcpyAsync(e2, epsII, sizeof(double) * 7 * nel, kin, c.stream));
    DP_CUDA(cudaMemcpyAsync(t2, tauII, sizeof(double) * 7 * nel, kin, c.stream));
    DP_CUDA(cudaMemcpyAsync(co, cohesion, sizeof(double) * 7 * nel, kin, c.stream));
    DP_CUDA(cudaMemcpyAsync(et, eta_ip, sizeof(double) * 7 * nel, kin, c.stream));
    DP_CUDA(cudaMemcpyAsync(stage, T_node, sizeof(double) * nn, kin, c.stream));
    launch_gather_ref2lat(c, stage, Tl, 1);
    DP_CUDA(cudaMemcpyAsync(stage, r_node, sizeof(double) * nn, kin, c.stream));
    launch_gather_ref2lat(c, stage, rl, 1);
    // vertices are the first nvert nodes of the reference numbering
    DP_CUDA(cudaMemsetAsync(stage, 0, sizeof(double) * nn, c.stream));
    DP_CUDA(cudaMemcpyAsync(stage, P_vertex, sizeof(double) * nv, kin, c.stream));
    launch_gather_ref2lat(c, stage, Pl, 1);
    // |min P| over the vertices (reference numbering) and max r
    ++g_klaunch;
    k_minmax_partial<<<kRedBlocks, kRedThreads, 0, c.stream>>>(stage, nv, rl, nn, c.partial);
    ++g_klaunch;
    k_minmax_final<<<1, 1, 0, c.stream>>>(c.partial, kRedBlocks, c.scal);
    ArrheniusArgs a;
    a.eta0 = law->eta0; a.R = law->R; a.Ea = law->Ea; a.Va = law->Va; a.T0 = law->T0; a.phi = law->phi_deg;
    a.sphi = std::sin(law->phi_deg * (3.14159265358979323846 / 180.0));
    a.cphi = std::cos(law->phi_deg * (3.14159265358979323846 / 180.0));
    const double keep[8] = {a.eta0, a.R, a.Ea, a.Va, a.T0, a.sphi, a.cphi, a.phi};
    for (int i = 0; i < 8; ++i) c.rheo_law[i] = keep[i];
    ++g_klaunch;
    k_viscosity_arrhenius<<<(int)div_up(nel, 128), 128, 0, c.stream>>>(Tl, Pl, rl, e2, t2, co, et, c.scal, a, (int)nel,
                                                                        c.fine.ncr, (int)c.fine.A(), (int)c.fine.B());
    DP_LAUNCH_CHECK();
    DP_CUDA(cudaMemcpyAsync(eta_ip, et, sizeof(double) * 7 * nel, kind_out(mem), c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}
