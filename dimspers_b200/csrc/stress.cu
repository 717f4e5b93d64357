// Strain-rate / stress post-processor: stress! (src/Stress/StressCalculation.jl:
// 23-249), called after each Stokes solve with the Cartesian velocity
// (MAIN.jl:241-243, nip = 7: MAIN.jl:94, :164).
//
// One thread per element (FP64).  Per 7-point IP: the curved inverse Jacobian
// of the (theta, r)-linear element (the same geometry as the assembly), the P2
// derivatives dN/dx, dN/dz, the strain rate (exx, ezz, exz = (dux/dz +
// duz/dx) / 2) and its second invariant, and the deviatoric stress with its
// invariant: isotropic eta (4/3, -2/3, 2) or, with a tensor, the reference's
// anisotropic formula (:219-233, including its factors: eta13 * exz in tau_xx,
// eta23 * 2 exz in tau_zz, eta33 * exz in tau_xz).  Outputs are the reference's
// nel x 7 matrices (element fastest), eight of them in a row.
#include "kernels.cuh"

namespace dp {

__constant__ double c_N3s[7][3];     // linear N3 at the 7 IPs (Quadrature.jl:109-138)
__constant__ double c_dNs[7][2][6];  // P2 dN/d(r, s) at the 7 IPs (sf_dN_tri6, :287-307)

static void upload_stress_constants() {
  double N3[7][3], dN[7][2][6];
  const double g1 = (6.0 - std::sqrt(15.0)) / 21.0, g2 = (6.0 + std::sqrt(15.0)) / 21.0;
  const double ip[7][2] = {{1.0 / 3.0, 1.0 / 3.0}, {1.0 - 2.0 * g1, g1}, {g1, 1.0 - 2.0 * g1}, {g1, g1},
                           {1.0 - 2.0 * g2, g2},   {g2, 1.0 - 2.0 * g2}, {g2, g2}};
  for (int q = 0; q < 7; ++q) {
    const double r = ip[q][0], s = ip[q][1], t = 1.0 - r - s;
    N3[q][0] = t; N3[q][1] = r; N3[q][2] = s;
    const double dr[6] = {-(4.0 * t - 1.0), 4.0 * r - 1.0, 0.0, 4.0 * (t - r), 4.0 * s, -4.0 * s};
    const double ds[6] = {-(4.0 * t - 1.0), 0.0, 4.0 * s - 1.0, -4.0 * r, 4.0 * r, 4.0 * (t - s)};
    for (int k = 0; k < 6; ++k) {
      dN[q][0][k] = dr[k];
      dN[q][1][k] = ds[k];
    }
  }
  DP_CUDA(cudaMemcpyToSymbol(c_N3s, N3, sizeof(N3)));
  DP_CUDA(cudaMemcpyToSymbol(c_dNs, dN, sizeof(dN)));
}

// U: Cartesian velocity, lattice order, interleaved (ux, uz).  eta: 7*nel
// (ip-major), C: 42*nel ((field*7 + ip)*nel + e) or null.  out: 56*nel.
__global__ void __launch_bounds__(128) k_stress(const double* __restrict__ U, const double* __restrict__ theta_lat,
                                                const double* __restrict__ r_lat, const double* __restrict__ eta,
                                                const double* __restrict__ C, double* __restrict__ out, int nel,
                                                int ncr, int A, int B) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  const int q = e >> 1, t = e & 1;
  const int ir = q % ncr, it = q / ncr;
  const int a0 = 2 * ir, b0 = 2 * it;
  int aa[6], bb[6];
  if (t == 0) {
    aa[0] = a0; aa[1] = a0; aa[2] = a0 + 2; aa[3] = a0; aa[4] = a0 + 1; aa[5] = a0 + 1;
    bb[0] = b0; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 1; bb[4] = b0 + 1; bb[5] = b0;
  } else {
    aa[0] = a0; aa[1] = a0 + 2; aa[2] = a0 + 2; aa[3] = a0 + 1; aa[4] = a0 + 2; aa[5] = a0 + 1;
    bb[0] = b0 + 2; bb[1] = b0 + 2; bb[2] = b0; bb[3] = b0 + 2; bb[4] = b0 + 1; bb[5] = b0 + 1;
  }
  int nd[6];
  double ux[6], uz[6];
  const double2* U2 = reinterpret_cast<const double2*>(U);
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    nd[k] = aa[k] + A * (bb[k] >= B ? bb[k] - B : bb[k]);
    const double2 v = U2[nd[k]];
    ux[k] = v.x;
    uz[k] = v.y;
  }
  // vertex coordinates + fixangles! (Utilities.jl:45-61)
  double th[3], rr[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    th[k] = theta_lat[nd[k]];
    rr[k] = r_lat[nd[k]];
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
  const double Jt0 = -th[0] + th[1], Jt1 = -th[0] + th[2];
  const double Jr0 = -rr[0] + rr[1], Jr1 = -rr[0] + rr[2];
  const double invdet = 1.0 / (Jt0 * Jr1 - Jt1 * Jr0);
  const double R21 = rr[1] - rr[0], R31 = rr[2] - rr[0];
  const double T31 = th[2] - th[0], T21 = th[1] - th[0];
  const size_t st = (size_t)nel;
  for (int ip = 0; ip < 7; ++ip) {
    const double th_ip = th[0] * c_N3s[ip][0] + th[1] * c_N3s[ip][1] + th[2] * c_N3s[ip][2];
    const double r_ip = rr[0] * c_N3s[ip][0] + rr[1] * c_N3s[ip][1] + rr[2] * c_N3s[ip][2];
    double s, c;
    sincos(th_ip, &s, &c);
    const double cr = c / r_ip, sr = s / r_ip;
    const double a11 = R31 * cr - T31 * s, a12 = -R21 * cr + T21 * s;
    const double a21 = -R31 * sr - T31 * c, a22 = R21 * sr + T21 * c;
    double exx = 0.0, ezz = 0.0, duxdz = 0.0, duzdx = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double dx = (a11 * c_dNs[ip][0][k] + a12 * c_dNs[ip][1][k]) * invdet;
      const double dz = (a21 * c_dNs[ip][0][k] + a22 * c_dNs[ip][1][k]) * invdet;
      exx += dx * ux[k];
      ezz += dz * uz[k];
      duxdz += dz * ux[k];
      duzdx += dx * uz[k];
    }
    const double exz = 0.5 * (duxdz + duzdx);
    const double et = eta[(size_t)ip * st + e];
    double txx, tzz, txz;
    if (C) {
      const double c11 = C[(size_t)(0 * 7 + ip) * st + e] * et, c33 = C[(size_t)(1 * 7 + ip) * st + e] * et;
      const double c55 = C[(size_t)(2 * 7 + ip) * st + e] * et, c13 = C[(size_t)(3 * 7 + ip) * st + e] * et;
      const double c15 = C[(size_t)(4 * 7 + ip) * st + e] * et, c35 = C[(size_t)(5 * 7 + ip) * st + e] * et;
      const double pa = -exx / 3.0 + 2.0 * ezz / 3.0, pb = 2.0 * exx / 3.0 - ezz / 3.0;
      txx = c13 * pa + c11 * pb + c15 * exz;
      tzz = c33 * pa + c13 * pb + c35 * 2.0 * exz;
      txz = c35 * pa + c15 * pb + c55 * exz;
    } else {
      txx = et * (4.0 / 3.0 * exx - 2.0 / 3.0 * ezz);
      tzz = et * (-2.0 / 3.0 * exx + 4.0 / 3.0 * ezz);
      txz = et * 2.0 * exz;
    }
    double* o = out + (size_t)ip * st + e;
    const size_t blk = 7 * st;
    o[0 * blk] = exx;
    o[1 * blk] = ezz;
    o[2 * blk] = exz;
    o[3 * blk] = sqrt(0.5 * (exx * exx + ezz * ezz) + exz * exz);
    o[4 * blk] = txx;
    o[5 * blk] = tzz;
    o[6 * blk] = txz;
    o[7 * blk] = sqrt(0.5 * (txx * txx + tzz * tzz) + txz * txz);
  }
}

// k_stress on the inputs staged by the last dp_stress call (kernel timing).
void launch_stress_staged(Ctx& c, bool tensor) {
  const int64_t nel = c.fine.nel;
  double* eta = c.stress_buf;
  double* C = eta + 7 * nel;
  double* o = C + 42 * nel;
  ++g_klaunch;
  k_stress<<<(int)div_up(nel, 128), 128, 0, c.stream>>>((const double*)c.work[W_RES], c.theta_lat, c.r_lat, eta,
                                                         tensor ? C : nullptr, o, (int)nel, c.fine.ncr,
                                                         (int)c.fine.A(), (int)c.fine.B());
  DP_LAUNCH_CHECK();
}

}  // namespace dp

using namespace dp;

extern "C" int dp_stress(dp_ctx* h, const double* Ucart, const double* eta_ip, int64_t ld_eta,
                         const double* const* C6, int64_t ld_C, double* out, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!Ucart || !eta_ip || !out) throw BadArg("null argument");
    const int64_t nel = c.fine.nel, nn = c.fine.nnod;
    if (ld_eta < nel || (C6 && ld_C < nel)) throw BadArg("leading dimension below nel");
    static bool uploaded[64] = {false};
    if (c.device < 0 || c.device >= 64 || !uploaded[c.device]) {
      upload_stress_constants();
      DP_CUDA(cudaDeviceSynchronize());  // the copies are on the default stream; ours does not wait on it
      if (c.device >= 0 && c.device < 64) uploaded[c.device] = true;
    }
    if (!c.stress_buf) dalloc(&c.stress_buf, (7 + 42 + 56) * nel);
    double* eta = c.stress_buf;
    double* C = eta + 7 * nel;
    double* o = C + 42 * nel;
    const cudaMemcpyKind kin = kind_in(mem);
    // nel x 7 column-major (element fastest) -> 7 contiguous columns
    DP_CUDA(cudaMemcpy2DAsync(eta, sizeof(double) * nel, eta_ip, sizeof(double) * ld_eta, sizeof(double) * nel, 7,
                              kin, c.stream));
    if (C6) {
      for (int f = 0; f < 6; ++f) {
        if (!C6[f]) throw BadArg("null tensor field");
        DP_CUDA(cudaMemcpy2DAsync(C + (size_t)f * 7 * nel, sizeof(double) * nel, C6[f], sizeof(double) * ld_C,
                                  sizeof(double) * nel, 7, kin, c.stream));
      }
    }
    // velocity: reference numbering -> lattice
    double* stage = (double*)c.work[W_UC];
    double* ulat = (double*)c.work[W_RES];
    DP_CUDA(cudaMemcpyAsync(stage, Ucart, sizeof(double) * 2 * nn, kin, c.stream));
    launch_gather_ref2lat(c, stage, ulat, 2);
    ++g_klaunch;
    k_stress<<<(int)div_up(nel, 128), 128, 0, c.stream>>>(ulat, c.theta_lat, c.r_lat, eta, C6 ? C : nullptr, o,
                                                           (int)nel, c.fine.ncr, (int)c.fine.A(), (int)c.fine.B());
    DP_LAUNCH_CHECK();
    c.stress_tensor = C6 != nullptr;
    DP_CUDA(cudaMemcpyAsync(out, o, sizeof(double) * 56 * nel, kind_out(mem), c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}
