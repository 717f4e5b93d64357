// Element assembly of the Stokes blocks on the device, one element per thread.
//
// Follows src/Stokes/StokesSolver.jl:
//   _fill_R_J!            :522-541  linear (theta, r) Jacobian of the 3 vertices
//   _ip_loop!             :587-638  6 Stokes IPs; eta read at IP 1..6 (:608)
//   _element_density      :1017-1038  rho_ip = NP . rho(vertices)
//   _derivative_weights!  :641-686  curved inverse Jacobian (x = r sin, z = r cos),
//                                   omega = r_ip * detJ * w_ip
//   _fill_Kblk!           :688-810  Ke += omega * B^T D B (packed lower, 78)
//   _fill_Gblk!           :812-823  Ge += omega * NP_i * dN_k/dx|dz (12x3)
//   _fill_Mblk!           :825-836  Me += (omega/eta) NP_i NP_j (packed, 6)
//   _fill_Fbblk!          :838-845  fe += omega * g * rho_ip * N_k * (sin, cos)
// and then, per element instead of on the global sparse matrices,
//   _prepare_matrices     :192-201  K <- TT^T K TT, G <- TT^T G, F <- TT^T F
//   _apply_bcs / free_slip          rows/cols of wall u_r zeroed
// The lumped pressure preconditioner 1/rowsum(M) (IterativeSolvers.jl:238-240)
// is produced in the same pass.
//
// The 132 per-element accumulators live in shared memory (one column per
// thread, conflict-free), which keeps the register count low enough for
// several CTAs per SM; assembly runs once per solve and is FP64 throughout
// (the refined path stores a rounded FP32 copy of Ke).
#include "kernels.cuh"

namespace dp {

__constant__ double c_N[6][6];       // P2 N at the 6 IPs
__constant__ double c_dN[6][2][6];   // P2 dN/d(r,s)
__constant__ double c_N3[6][3];      // linear N3 = pressure NP
__constant__ double c_w[6];          // weights (x0.5)

void upload_quadrature_constants() {
  // ip_triangle6 (Quadrature.jl:80-107), sf_N_tri6 / sf_dN_tri6 (:264-307)
  const double g1 = (8.0 - std::sqrt(10.0) + std::sqrt(38.0 - 44.0 * std::sqrt(2.0 / 5.0))) / 18.0;
  const double g2 = (8.0 - std::sqrt(10.0) - std::sqrt(38.0 - 44.0 * std::sqrt(2.0 / 5.0))) / 18.0;
  const double ipx[6][2] = {{1.0 - 2.0 * g1, g1}, {g1, 1.0 - 2.0 * g1}, {g1, g1},
                            {1.0 - 2.0 * g2, g2}, {g2, 1.0 - 2.0 * g2}, {g2, g2}};
  const double w1 = (620.0 + std::sqrt(213125.0 - 53320.0 * std::sqrt(10.0))) / 3720.0;
  const double w2 = (620.0 - std::sqrt(213125.0 - 53320.0 * std::sqrt(10.0))) / 3720.0;
  double N[6][6], dN[6][2][6], N3[6][3], w[6];
  for (int ip = 0; ip < 6; ++ip) {
    const double r = ipx[ip][0], s = ipx[ip][1], t = 1.0 - r - s;
    N[ip][0] = t * (2.0 * t - 1.0);
    N[ip][1] = r * (2.0 * r - 1.0);
    N[ip][2] = s * (2.0 * s - 1.0);
    N[ip][3] = 4.0 * r * t;
    N[ip][4] = 4.0 * r * s;
    N[ip][5] = 4.0 * s * t;
    const double dr[6] = {-(4.0 * t - 1.0), 4.0 * r - 1.0, 0.0, 4.0 * (t - r), 4.0 * s, -4.0 * s};
    const double ds[6] = {-(4.0 * t - 1.0), 0.0, 4.0 * s - 1.0, -4.0 * r, 4.0 * r, 4.0 * (t - s)};
    for (int k = 0; k < 6; ++k) { dN[ip][0][k] = dr[k]; dN[ip][1][k] = ds[k]; }
    N3[ip][0] = t; N3[ip][1] = r; N3[ip][2] = s;
    w[ip] = 0.5 * (ip < 3 ? w1 : w2);
  }
  DP_CUDA(cudaMemcpyToSymbol(c_N, N, sizeof(N)));
  DP_CUDA(cudaMemcpyToSymbol(c_dN, dN, sizeof(dN)));
  DP_CUDA(cudaMemcpyToSymbol(c_N3, N3, sizeof(N3)));
  DP_CUDA(cudaMemcpyToSymbol(c_w, w, sizeof(w)));
}

// directRotation2D (anisotropy.jl:503-536) of the frame tensor
// (a, c, e, h) = (4/3, 4/3, 1/delta, -2/3) by rotmatrix(dx, dy) (:287-292).
// Output order: C11, C33, C55, C13, C15, C35 (StiffnessTensor fields).
__host__ __device__ inline void ti_tensor(double delta, double dx, double dy, double out[6]) {
  const double a = 4.0 / 3.0, c = 4.0 / 3.0, h = -2.0 / 3.0;
  const double e = 1.0 / delta;
  const double inv = 1.0 / sqrt(dy * dy + dx * dx);
  const double cs = dx * inv, sn = dy * inv;
  const double x1 = cs, y2 = cs, x2 = sn, y1 = -sn;
  const double x1x1 = x1 * x1, x2x2 = x2 * x2, y1y1 = y1 * y1, y2y2 = y2 * y2;
  const double m = x1 * y2 + x2 * y1;
  out[0] = (c * x2x2 + h * x1x1 + 4 * e * x1x1) * x2x2 + (a * x1x1 + h * x2x2) * x1x1;
  out[1] = (c * y2y2 + h * y1y1 + 4 * e * y1y1) * y2y2 + (a * y1y1 + h * y2y2) * y1y1;
  out[2] = (c * x2 * y2 + h * x1 * y1) * x2 * y2 + m * m * e + (a * x1 * y1 + h * x2 * y2) * x1 * y1;
  out[3] = ((c * x2x2 + h * x1x1) * y2 + 4 * e * x1 * x2 * y1) * y2 + (a * x1x1 + h * x2x2) * y1y1;
  out[4] = ((c * x2x2 + h * x1x1) * y2 + 2 * m * e * x1) * x2 + (a * x1x1 + h * x2x2) * x1 * y1;
  out[5] = ((c * y2y2 + h * y1y1) * x2 + 2 * m * e * y1) * y2 + (a * y1y1 + h * y2y2) * x1 * y1;
}

struct AsmArgs {
  int ncr, nct, nel, A, B, pressure, mat_kind, pin;
  const double* theta_lat;
  const double* r_lat;
  const double* rho_lat;
  const double* eta;   // 6*nel
  const double* C;     // FULL 36*nel | TI 3*nel
  double g;
  double* K64;         // 78*nel (may be null)
  float* K32;          // 78*nel (may be null)
  double* Gp;          // 36*nel
  double* F;           // 2*nnod, accumulated with atomics (zeroed by caller)
  double* Fe;          // deterministic mode: element RHS, Fe[(2k + c) nel + e] (F then by k_node_gather)
  double* pcsum;       // npres: disc -> 1/rowsum written; cont -> rowsum accumulated
  double* Minv;        // 6*nel: inverse of the element mass block (discontinuous pressure)
  double* mfD;         // 36*nel or null: omega * Q^T D Q per IP, entry-major (matrix-free apply)
  CartOut cart;
};

constexpr int kAsmThreads = 64;
constexpr int kAcc = kKe + kGe + kMe + kFe;  // 132

__global__ void __launch_bounds__(kAsmThreads) k_assemble(AsmArgs p) {
  extern __shared__ double sm[];
  const int tid = threadIdx.x;
  const int e = blockIdx.x * kAsmThreads + tid;
  if (e >= p.nel) return;  // no block-level synchronisation below
  double* acc = sm + tid;
#define ACC(i) acc[(i) * kAsmThreads]
  for (int i = 0; i < kAcc; ++i) ACC(i) = 0.0;

  // lattice nodes of the element
  const int q = e >> 1, t = e & 1;
  const int ir = q % p.ncr, it = q / p.ncr;
  int na[6], nb[6];
  {
    const int a0 = 2 * ir, b0 = 2 * it;
    if (t == 0) {
      const int aa[6] = {a0, a0, a0 + 2, a0, a0 + 1, a0 + 1};
      const int bb[6] = {b0, b0 + 2, b0, b0 + 1, b0 + 1, b0};
      for (int k = 0; k < 6; ++k) { na[k] = aa[k]; nb[k] = bb[k]; }
    } else {
      const int aa[6] = {a0, a0 + 2, a0 + 2, a0 + 1, a0 + 2, a0 + 1};
      const int bb[6] = {b0 + 2, b0 + 2, b0, b0 + 2, b0 + 1, b0 + 1};
      for (int k = 0; k < 6; ++k) { na[k] = aa[k]; nb[k] = bb[k]; }
    }
  }
  int nd[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) nd[k] = na[k] + p.A * (nb[k] >= p.B ? nb[k] - p.B : nb[k]);

  // vertex coordinates + fixangles! (Utilities.jl:45-61)
  double th[3], rr[3], rho[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    th[k] = p.theta_lat[nd[k]];
    rr[k] = p.r_lat[nd[k]];
    rho[k] = p.rho_lat[nd[k]];
  }
  {
    const double PI = 3.14159265358979323846;
    const double a1 = fabs(th[0] - th[1]), a2 = fabs(th[1] - th[2]), a3 = fabs(th[2] - th[0]);
    if ((a1 + a2 + a3) > PI) {
#pragma unroll
      for (int k = 0; k < 3; ++k)
        if (th[k] < PI) th[k] += 2.0 * PI;
    }
  }
  // _fill_R_J! (:522-541); J = VCOORD' * dN3ds'
  const double Jt0 = -th[0] + th[1], Jt1 = -th[0] + th[2];
  const double Jr0 = -rr[0] + rr[1], Jr1 = -rr[0] + rr[2];
  const double detJ = Jt0 * Jr1 - Jt1 * Jr0;
  const double R31 = rr[2] - rr[0], R21 = rr[1] - rr[0];
  const double T31 = th[2] - th[0], T21 = th[1] - th[0];

  double Cel[6];
  if (p.mat_kind == MAT_TI) ti_tensor(p.C[e], p.C[p.nel + e], p.C[2 * p.nel + e], Cel);

  // matrix-free form: the element is its ring's reference element (it = 0)
  // rotated by phi = theta(v0) - theta(v0 of the reference); its polar operator
  // is sum_ip om B0^T (Q^T D Q) B0 with Q the engineering-strain rotation by phi
  double qc = 1.0, qs = 0.0;
  const size_t emf = (size_t)e;
  if (p.mfD) {
    const int bref = (t == 0) ? 0 : 2;            // vertex 0 of the reference element
    sincos(th[0] - p.theta_lat[2 * ir + p.A * bref], &qs, &qc);
  }

  for (int ip = 0; ip < 6; ++ip) {
    const double th_ip = th[0] * c_N3[ip][0] + th[1] * c_N3[ip][1] + th[2] * c_N3[ip][2];
    const double r_ip = rr[0] * c_N3[ip][0] + rr[1] * c_N3[ip][1] + rr[2] * c_N3[ip][2];
    const double dens = rho[0] * c_N3[ip][0] + rho[1] * c_N3[ip][1] + rho[2] * c_N3[ip][2];
    const double visc = p.eta[(size_t)ip * p.nel + e];
    const double fg = p.g * dens;
    double s, c;
    sincos(th_ip, &s, &c);
    const double inv = 1.0 / r_ip / detJ;
    const double ix0 = (R31 * c - T31 * s * r_ip) * inv;
    const double ix1 = (-R21 * c + T21 * s * r_ip) * inv;
    const double iz0 = (-R31 * s - T31 * c * r_ip) * inv;
    const double iz1 = (R21 * s + T21 * c * r_ip) * inv;
    const double om = r_ip * detJ * c_w[ip];
    double dx[6], dz[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      dx[k] = ix0 * c_dN[ip][0][k] + ix1 * c_dN[ip][1][k];
      dz[k] = iz0 * c_dN[ip][0][k] + iz1 * c_dN[ip][1][k];
    }
    // D (Voigt xx, zz, xz), symmetric: d11 d12 d13 / d22 d23 / d33
    double d11, d12, d13, d22, d23, d33;
    if (p.mat_kind == MAT_ISO) {
      d11 = d22 = (4.0 / 3.0) * visc;
      d12 = (-2.0 / 3.0) * visc;
      d33 = visc;
      d13 = d23 = 0.0;
    } else {
      double cc[6];
      if (p.mat_kind == MAT_FULL) {
#pragma unroll
        for (int f = 0; f < 6; ++f) cc[f] = p.C[((size_t)f * 6 + ip) * p.nel + e];
      } else {
#pragma unroll
        for (int f = 0; f < 6; ++f) cc[f] = Cel[f];
      }
      d11 = cc[0] * visc; d22 = cc[1] * visc; d33 = cc[2] * visc;
      d12 = cc[3] * visc; d13 = cc[4] * visc; d23 = cc[5] * visc;
    }
    if (p.mfD) {
      // om * Q^T D Q, Q = [c^2 s^2 cs; s^2 c^2 -cs; -2cs 2cs c^2-s^2]
      const double cc2 = qc * qc, ss2 = qs * qs, cs = qc * qs;
      const double Q[3][3] = {{cc2, ss2, cs}, {ss2, cc2, -cs}, {-2.0 * cs, 2.0 * cs, cc2 - ss2}};
      const double Dm[3][3] = {{d11, d12, d13}, {d12, d22, d23}, {d13, d23, d33}};
      double M[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i][j] = Dm[i][0] * Q[0][j] + Dm[i][1] * Q[1][j] + Dm[i][2] * Q[2][j];
      double R[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = Q[0][i] * M[0][j] + Q[1][i] * M[1][j] + Q[2][i] * M[2][j];
      const size_t st = (size_t)p.nel;
      double* o = p.mfD + (size_t)(ip * 6) * st + emf;
      o[0 * st] = om * R[0][0];
      o[1 * st] = om * R[0][1];
      o[2 * st] = om * R[0][2];
      o[3 * st] = om * R[1][1];
      o[4 * st] = om * R[1][2];
      o[5 * st] = om * R[2][2];
    }
    // omega * D * B columns: DBx_i = D (dx_i, 0, dz_i), DBz_i = D (0, dz_i, dx_i)
    double bx0[6], bx1[6], bx2[6], bz0[6], bz1[6], bz2[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      const double x = om * dx[i], z = om * dz[i];
      bx0[i] = d11 * x + d13 * z; bx1[i] = d12 * x + d23 * z; bx2[i] = d13 * x + d33 * z;
      bz0[i] = d12 * z + d13 * x; bz1[i] = d22 * z + d23 * x; bz2[i] = d23 * z + d33 * x;
    }
    // Ke lower packed: column 2i rows (2j, 2j+1) j>=i; column 2i+1 rows 2j (j>i), 2j+1 (j>=i)
#pragma unroll
    for (int i = 0; i < 6; ++i) {
#pragma unroll
      for (int j = i; j < 6; ++j) {
        ACC(packed_index12(2 * j, 2 * i)) += dx[j] * bx0[i] + dz[j] * bx2[i];
        ACC(packed_index12(2 * j + 1, 2 * i)) += dz[j] * bx1[i] + dx[j] * bx2[i];
        if (j > i) ACC(packed_index12(2 * j, 2 * i + 1)) += dx[j] * bz0[i] + dz[j] * bz2[i];
        ACC(packed_index12(2 * j + 1, 2 * i + 1)) += dz[j] * bz1[i] + dx[j] * bz2[i];
      }
    }
    // Ge (12x3 column-major)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double tt = om * c_N3[ip][i];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        ACC(kKe + i * 12 + 2 * k) += tt * dx[k];
        ACC(kKe + i * 12 + 2 * k + 1) += tt * dz[k];
      }
    }
    // Me packed lower 3x3: (0,0),(1,0),(2,0),(1,1),(2,1),(2,2)
    {
      const double w3 = om / visc;
      const double* NP = c_N3[ip];
      ACC(kKe + kGe + 0) += w3 * NP[0] * NP[0];
      ACC(kKe + kGe + 1) += w3 * NP[1] * NP[0];
      ACC(kKe + kGe + 2) += w3 * NP[2] * NP[0];
      ACC(kKe + kGe + 3) += w3 * NP[1] * NP[1];
      ACC(kKe + kGe + 4) += w3 * NP[2] * NP[1];
      ACC(kKe + kGe + 5) += w3 * NP[2] * NP[2];
    }
    // Fb
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      const double cte = om * fg * c_N[ip][k];
      ACC(kKe + kGe + kMe + 2 * k) += s * cte;
      ACC(kKe + kGe + kMe + 2 * k + 1) += c * cte;
    }
  }

  // optional Cartesian reference-layout outputs (column-major 78 x nel etc.)
  if (p.cart.Ke) for (int i = 0; i < kKe; ++i) p.cart.Ke[(size_t)e * kKe + i] = ACC(i);
  if (p.cart.Ge) for (int i = 0; i < kGe; ++i) p.cart.Ge[(size_t)e * kGe + i] = ACC(kKe + i);
  if (p.cart.Me) for (int i = 0; i < kMe; ++i) p.cart.Me[(size_t)e * kMe + i] = ACC(kKe + kGe + i);
  if (p.cart.Fb) for (int i = 0; i < kFe; ++i) p.cart.Fb[(size_t)e * kFe + i] = ACC(kKe + kGe + kMe + i);

  // rotation to polar DOFs: TT_k = [c s; -s c] per node (StokesSolver.jl:214-241)
  double cs[6], sn[6];
  bool fixed[6], fixt[6];  // u_r / u_theta constrained
  const int amax = 2 * p.ncr;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    sincos(p.theta_lat[nd[k]], &sn[k], &cs[k]);
    const int bk = nb[k] >= p.B ? nb[k] - p.B : nb[k];
    fixed[k] = dof_fixed(na[k], bk, 1, amax, p.pin);
    fixt[k] = dof_fixed(na[k], bk, 0, amax, p.pin);
  }
  // K: block (j,i) -> T_j^T K_ji T_i, written to packed lower
  for (int i = 0; i < 6; ++i) {
    for (int j = i; j < 6; ++j) {
      double k00 = ACC(packed_index12(2 * j, 2 * i));
      double k10 = ACC(packed_index12(2 * j + 1, 2 * i));
      double k11 = ACC(packed_index12(2 * j + 1, 2 * i + 1));
      double k01 = (j > i) ? ACC(packed_index12(2 * j, 2 * i + 1)) : k10;
      // M1 = K_ji T_i
      const double m00 = k00 * cs[i] - k01 * sn[i], m01 = k00 * sn[i] + k01 * cs[i];
      const double m10 = k10 * cs[i] - k11 * sn[i], m11 = k10 * sn[i] + k11 * cs[i];
      // T_j^T M1
      double r00 = cs[j] * m00 - sn[j] * m10, r01 = cs[j] * m01 - sn[j] * m11;
      double r10 = sn[j] * m00 + cs[j] * m10, r11 = sn[j] * m01 + cs[j] * m11;
      if (fixed[i]) { r01 = 0.0; r11 = 0.0; }
      if (fixed[j]) { r10 = 0.0; r11 = 0.0; }
      if (fixt[i]) { r00 = 0.0; r10 = 0.0; }
      if (fixt[j]) { r00 = 0.0; r01 = 0.0; }
      ACC(packed_index12(2 * j, 2 * i)) = r00;
      ACC(packed_index12(2 * j + 1, 2 * i)) = r10;
      ACC(packed_index12(2 * j + 1, 2 * i + 1)) = r11;
      if (j > i) ACC(packed_index12(2 * j, 2 * i + 1)) = r01;
    }
  }
  if (p.K64)
    for (int i = 0; i < kKe; ++i) p.K64[kidx64(i, e)] = ACC(i);
  if (p.K32)
    for (int i = 0; i < kKe; ++i) p.K32[kidx32(i, e)] = (float)ACC(i);
  // G rows and F: T_k^T applied per node, wall u_r rows zeroed
#pragma unroll
  for (int k = 0; k < 6; ++k) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double gx = ACC(kKe + i * 12 + 2 * k), gz = ACC(kKe + i * 12 + 2 * k + 1);
      p.Gp[(size_t)(i * 12 + 2 * k) * p.nel + e] = fixt[k] ? 0.0 : cs[k] * gx - sn[k] * gz;
      p.Gp[(size_t)(i * 12 + 2 * k + 1) * p.nel + e] = fixed[k] ? 0.0 : sn[k] * gx + cs[k] * gz;
    }
    const double fx = ACC(kKe + kGe + kMe + 2 * k), fz = ACC(kKe + kGe + kMe + 2 * k + 1);
    if (p.Fe) {
      p.Fe[(size_t)(2 * k) * p.nel + e] = fixt[k] ? 0.0 : cs[k] * fx - sn[k] * fz;
      p.Fe[(size_t)(2 * k + 1) * p.nel + e] = fixed[k] ? 0.0 : sn[k] * fx + cs[k] * fz;
    } else {
      if (!fixt[k]) atomicAdd(&p.F[2 * (size_t)nd[k]], cs[k] * fx - sn[k] * fz);
      if (!fixed[k]) atomicAdd(&p.F[2 * (size_t)nd[k] + 1], sn[k] * fx + cs[k] * fz);
    }
  }
  // lumped mass rows
  {
    const double m00 = ACC(kKe + kGe + 0), m10 = ACC(kKe + kGe + 1), m20 = ACC(kKe + kGe + 2);
    const double m11 = ACC(kKe + kGe + 3), m21 = ACC(kKe + kGe + 4), m22 = ACC(kKe + kGe + 5);
    const double row[3] = {m00 + m10 + m20, m10 + m11 + m21, m20 + m21 + m22};
    if (p.pressure == 1) {
      for (int i = 0; i < 3; ++i) p.pcsum[3 * (size_t)e + i] = 1.0 / row[i];
      // exact inverse of the symmetric 3x3 element block M_e (the whole of M for
      // discontinuous pressure), packed (00, 10, 20, 11, 21, 22)
      const double c00 = m11 * m22 - m21 * m21, c10 = -(m10 * m22 - m21 * m20), c20 = m10 * m21 - m11 * m20;
      const double c11 = m00 * m22 - m20 * m20, c21 = -(m00 * m21 - m10 * m20), c22 = m00 * m11 - m10 * m10;
      const double det = m00 * c00 + m10 * c10 + m20 * c20;
      const double id = 1.0 / det;
      p.Minv[(size_t)0 * p.nel + e] = c00 * id;
      p.Minv[(size_t)1 * p.nel + e] = c10 * id;
      p.Minv[(size_t)2 * p.nel + e] = c20 * id;
      p.Minv[(size_t)3 * p.nel + e] = c11 * id;
      p.Minv[(size_t)4 * p.nel + e] = c21 * id;
      p.Minv[(size_t)5 * p.nel + e] = c22 * id;
    } else {
      int64_t pd[3];
      element_pdofs_cont(e, p.ncr, p.nct, pd);
      for (int i = 0; i < 3; ++i) atomicAdd(&p.pcsum[pd[i]], row[i]);
    }
  }
#undef ACC
}

// Per ring (ir, t) of the matrix-free apply (ring = 2 ir + t): the reference
// element's (it = 0) Cartesian shape-function derivatives at the 6 IPs and its
// node rotations, value-major so that consecutive rings are consecutive:
// tab[(ip * 12 + k) * nring + ring] = dN_k/dx, [(ip * 12 + 6 + k) * nring + ring]
// = dN_k/dz, [(72 + 2k) * nring + ring] = cos theta_k, [(73 + 2k) ..] = sin.
// Same formulas as k_assemble.
__global__ void k_mf_table(int ncr, int A, const double* __restrict__ theta_lat, const double* __restrict__ r_lat,
                           double* __restrict__ tab) {
  const int ring = blockIdx.x * blockDim.x + threadIdx.x;
  if (ring >= 2 * ncr) return;
  const int ir = ring >> 1, t = ring & 1;
  const int a0 = 2 * ir, b0 = 0;
  int na[6], nb[6];
  if (t == 0) {
    const int aa[6] = {a0, a0, a0 + 2, a0, a0 + 1, a0 + 1};
    const int bb[6] = {b0, b0 + 2, b0, b0 + 1, b0 + 1, b0};
    for (int k = 0; k < 6; ++k) { na[k] = aa[k]; nb[k] = bb[k]; }
  } else {
    const int aa[6] = {a0, a0 + 2, a0 + 2, a0 + 1, a0 + 2, a0 + 1};
    const int bb[6] = {b0 + 2, b0 + 2, b0, b0 + 2, b0 + 1, b0 + 1};
    for (int k = 0; k < 6; ++k) { na[k] = aa[k]; nb[k] = bb[k]; }
  }
  int nd[6];
  for (int k = 0; k < 6; ++k) nd[k] = na[k] + A * nb[k];
  double th[3], rr[3];
  for (int k = 0; k < 3; ++k) {
    th[k] = theta_lat[nd[k]];
    rr[k] = r_lat[nd[k]];
  }
  const double Jt0 = -th[0] + th[1], Jt1 = -th[0] + th[2];
  const double Jr0 = -rr[0] + rr[1], Jr1 = -rr[0] + rr[2];
  const double detJ = Jt0 * Jr1 - Jt1 * Jr0;
  const double R31 = rr[2] - rr[0], R21 = rr[1] - rr[0];
  const double T31 = th[2] - th[0], T21 = th[1] - th[0];
  const int nring = 2 * ncr;
  double* o = tab + ring;
  for (int ip = 0; ip < 6; ++ip) {
    const double th_ip = th[0] * c_N3[ip][0] + th[1] * c_N3[ip][1] + th[2] * c_N3[ip][2];
    const double r_ip = rr[0] * c_N3[ip][0] + rr[1] * c_N3[ip][1] + rr[2] * c_N3[ip][2];
    double s, c;
    sincos(th_ip, &s, &c);
    const double inv = 1.0 / r_ip / detJ;
    const double ix0 = (R31 * c - T31 * s * r_ip) * inv;
    const double ix1 = (-R21 * c + T21 * s * r_ip) * inv;
    const double iz0 = (-R31 * s - T31 * c * r_ip) * inv;
    const double iz1 = (R21 * s + T21 * c * r_ip) * inv;
    for (int k = 0; k < 6; ++k) {
      o[(size_t)(ip * 12 + k) * nring] = ix0 * c_dN[ip][0][k] + ix1 * c_dN[ip][1][k];
      o[(size_t)(ip * 12 + 6 + k) * nring] = iz0 * c_dN[ip][0][k] + iz1 * c_dN[ip][1][k];
    }
  }
  for (int k = 0; k < 6; ++k) {
    double s, c;
    sincos(theta_lat[nd[k]], &s, &c);
    o[(size_t)(72 + 2 * k) * nring] = c;
    o[(size_t)(73 + 2 * k) * nring] = s;
  }
}

void launch_assemble(Ctx& c, int precision, const CartOut* cart) {
  const Level& L = c.fine;
  AsmArgs a{};
  a.ncr = L.ncr; a.nct = L.nct; a.nel = (int)L.nel; a.A = (int)L.A(); a.B = (int)L.B();
  a.pressure = c.mesh.pressure;
  a.mat_kind = c.mat_kind;
  a.pin = L.pin;
  a.theta_lat = c.theta_lat; a.r_lat = c.r_lat; a.rho_lat = c.rho_lat;
  a.eta = c.eta; a.C = c.C; a.g = c.g;
  a.K64 = c.K64;
  a.K32 = precision >= 1 ? c.K32 : nullptr;
  a.Gp = c.Gp; a.F = c.F; a.pcsum = c.pc; a.Minv = c.Minv;
  a.Fe = static_cast<double*>(L.det);
  a.mfD = c.mfD64;
  if (cart) a.cart = *cart;
  const size_t smem = sizeof(double) * kAcc * kAsmThreads;
  static bool attr_set = false;
  if (!attr_set) {
    DP_CUDA(cudaFuncSetAttribute(k_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  if (!a.Fe) DP_CUDA(cudaMemsetAsync(c.F, 0, sizeof(double) * 2 * L.nnod, c.stream));
  if (c.mesh.pressure == 0) DP_CUDA(cudaMemsetAsync(c.pc, 0, sizeof(double) * c.mesh.npres, c.stream));
  const int grid = (int)div_up(L.nel, kAsmThreads);
  ++g_klaunch;
  k_assemble<<<grid, kAsmThreads, smem, c.stream>>>(a);
  DP_LAUNCH_CHECK();
  if (a.Fe) launch_node_gather<double>(L, a.Fe, c.F, 2, 2, c.stream);
  if (c.mfT64) {
    ++g_klaunch;
    k_mf_table<<<(int)div_up(2 * L.ncr, 64), 64, 0, c.stream>>>(L.ncr, (int)L.A(), c.theta_lat, c.r_lat, c.mfT64);
    DP_LAUNCH_CHECK();
  }
  if (c.mesh.pressure == 0) launch_pc_invert(c, c.pc, c.mesh.npres);
}

__global__ void k_ti_fill(int nel, const double* delta, const double* dx, const double* dy, double* C) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  C[e] = delta[e];
  C[nel + e] = dx[e];
  C[2 * (size_t)nel + e] = dy[e];
}

void launch_ti_tensor_fill(Ctx& c, const double* delta, const double* dx, const double* dy) {
  const int nel = (int)c.fine.nel;
  ++g_klaunch;
  k_ti_fill<<<(int)div_up(nel, 256), 256, 0, c.stream>>>(nel, delta, dx, dy, c.C);
  DP_LAUNCH_CHECK();
}

// Major eigenvector (vx, vy) and the eigenvalues of L = F F^T (FSE.jl:143-161,
// eigval_order :189), F in Julia 2x2 column-major order F11, F21, F12, F22.
// The eigenvector is taken from whichever row of L - lmax I is longer; a
// multiple of the identity gives (1, 0).  lmin = det(L) / lmax (no
// cancellation for elongated ellipsoids).
__device__ __forceinline__ void fse_axes(double f11, double f21, double f12, double f22, double& vx, double& vy,
                                         double& lmax, double& lmin) {
  const double l11 = f11 * f11 + f12 * f12;
  const double l12 = f11 * f21 + f12 * f22;
  const double l22 = f21 * f21 + f22 * f22;
  const double half_tr = 0.5 * (l11 + l22);
  const double disc = sqrt(0.25 * (l11 - l22) * (l11 - l22) + l12 * l12);
  lmax = half_tr + disc;
  const double ax = l12, ay = lmax - l11, bx = lmax - l22, by = l12;
  const bool use_a = (ax * ax + ay * ay) >= (bx * bx + by * by);
  vx = use_a ? ax : bx;
  vy = use_a ? ay : by;
  const double n = sqrt(vx * vx + vy * vy);
  if (n == 0.0) { vx = 1.0; vy = 0.0; } else { vx /= n; vy /= n; }
  const double det = f11 * f22 - f12 * f21;
  lmin = lmax > 0.0 ? det * det / lmax : 0.0;
}

// Major eigenvector of L = F F^T per element.
__global__ void k_fse_director(int64_t nel, const double* F, double* dxo, double* dyo) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nel) return;
  double vx, vy, l1, l2;
  fse_axes(F[4 * e + 0], F[4 * e + 1], F[4 * e + 2], F[4 * e + 3], vx, vy, l1, l2);
  dxo[e] = vx;
  dyo[e] = vy;
}

void launch_fse_director(Ctx& c, const double* F, double* dx, double* dy, int64_t nel) {
  ++g_klaunch;
  k_fse_director<<<(int)div_up(nel, 256), 256, 0, c.stream>>>(nel, F, dx, dy);
  DP_LAUNCH_CHECK();
}

}  // namespace dp
