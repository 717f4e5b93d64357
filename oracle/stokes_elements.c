/* Stokes element blocks of the annulus in plain C (FP64; test
 * infrastructure): a second, independent restatement of the element
 * assembly beside oracle/assembly.py, threaded over elements with OpenMP.
 *
 * Follows src/Stokes/StokesSolver.jl:
 *   _fill_R_J!            :522-541   J from the linear (theta, r) map
 *   _derivative_weights!  :641-686   curved inverse Jacobian, omega = r detJ w
 *   _fill_Kblk! (aniso)   :744-810   78 packed lower entries, the loop order
 *   _fill_Gblk!           :812-823   12 x 3 column-major
 *   _fill_Mblk!           :825-836   (omega / eta) NP NP, 6 packed lower
 *   _fill_Fbblk!          :838-845   omega g rho_ip N (sin, cos)
 *   _element_density      :1017-1038 rho_ip from the three vertex values
 * with the 6-point rule and the P2 / P1 shape functions of
 * src/Algebra/Quadrature.jl:80-107, 166-180, 264-307.
 *
 * Layouts follow the NumPy oracle: th, r, rho_v are (3, nel) and the outputs
 * (78|36|6|12, nel), element index fastest; eta_ip and the six tensor fields
 * (C11, C33, C55, C13, C15, C35) are (nel, ld) column-major, IPs 1..6 read.
 * C6 == NULL is the isotropic D = eta [4/3 -2/3 0; -2/3 4/3 0; 0 0 1].
 *
 * Build: gcc -O2 -fopenmp -shared -fPIC -o oracle/libstokes_elements.so oracle/stokes_elements.c -lm
 */
#include <math.h>
#include <stdint.h>

static void quadrature(double ip[6][2], double w[6]) {
  const double g1 = (8.0 - sqrt(10.0) + sqrt(38.0 - 44.0 * sqrt(2.0 / 5.0))) / 18.0;
  const double g2 = (8.0 - sqrt(10.0) - sqrt(38.0 - 44.0 * sqrt(2.0 / 5.0))) / 18.0;
  const double w1 = (620.0 + sqrt(213125.0 - 53320.0 * sqrt(10.0))) / 3720.0;
  const double w2 = (620.0 - sqrt(213125.0 - 53320.0 * sqrt(10.0))) / 3720.0;
  const double pts[6][2] = {{1.0 - 2.0 * g1, g1}, {g1, 1.0 - 2.0 * g1}, {g1, g1},
                            {1.0 - 2.0 * g2, g2}, {g2, 1.0 - 2.0 * g2}, {g2, g2}};
  for (int q = 0; q < 6; ++q) {
    ip[q][0] = pts[q][0];
    ip[q][1] = pts[q][1];
    w[q] = 0.5 * (q < 3 ? w1 : w2);
  }
}

static void shape(double r, double s, double N[6], double dN[2][6], double N3[3]) {
  const double t = 1.0 - r - s;
  N[0] = t * (2.0 * t - 1.0); N[1] = r * (2.0 * r - 1.0); N[2] = s * (2.0 * s - 1.0);
  N[3] = 4.0 * r * t; N[4] = 4.0 * r * s; N[5] = 4.0 * s * t;
  dN[0][0] = -(4.0 * t - 1.0); dN[0][1] = 4.0 * r - 1.0; dN[0][2] = 0.0;
  dN[0][3] = 4.0 * (t - r); dN[0][4] = 4.0 * s; dN[0][5] = -4.0 * s;
  dN[1][0] = -(4.0 * t - 1.0); dN[1][1] = 0.0; dN[1][2] = 4.0 * s - 1.0;
  dN[1][3] = -4.0 * r; dN[1][4] = 4.0 * r; dN[1][5] = 4.0 * (t - s);
  N3[0] = t; N3[1] = r; N3[2] = s;
}

int dpo_element_matrices(int64_t nel, const double* th, const double* r, const double* eta_ip, int64_t ld_eta,
                         const double* const* C6, int64_t ld_C, const double* rho_v, double g, double* Kp,
                         double* Ge, double* Me, double* Fb) {
  if (nel < 0 || ld_eta < nel || (C6 && ld_C < nel)) return 1;
  double ip[6][2], w[6], N[6][6], dN[6][2][6], N3[6][3];
  quadrature(ip, w);
  for (int q = 0; q < 6; ++q) shape(ip[q][0], ip[q][1], N[q], dN[q], N3[q]);
  static const int PACK3[6][2] = {{0, 0}, {1, 0}, {2, 0}, {1, 1}, {2, 1}, {2, 2}};
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < nel; ++e) {
    const double t0 = th[e], t1 = th[nel + e], t2 = th[2 * nel + e];
    const double r0 = r[e], r1 = r[nel + e], r2 = r[2 * nel + e];
    const double Jt0 = -t0 + t1, Jt1 = -t0 + t2, Jr0 = -r0 + r1, Jr1 = -r0 + r2;
    const double detJ = Jt0 * Jr1 - Jt1 * Jr0;
    const double R31 = r2 - r0, R21 = r1 - r0, T31 = t2 - t0, T21 = t1 - t0;
    double K[78] = {0}, G[36] = {0}, M[6] = {0}, F[12] = {0};
    for (int q = 0; q < 6; ++q) {
      const double th_ip = t0 * N3[q][0] + t1 * N3[q][1] + t2 * N3[q][2];
      const double r_ip = r0 * N3[q][0] + r1 * N3[q][1] + r2 * N3[q][2];
      const double dens = rho_v[e] * N3[q][0] + rho_v[nel + e] * N3[q][1] + rho_v[2 * nel + e] * N3[q][2];
      const double visc = eta_ip[(int64_t)q * ld_eta + e];
      const double fg = g * dens;
      const double s = sin(th_ip), c = cos(th_ip);
      const double inv = 1.0 / r_ip / detJ;
      const double ix0 = (R31 * c - T31 * s * r_ip) * inv, ix1 = (-R21 * c + T21 * s * r_ip) * inv;
      const double iz0 = (-R31 * s - T31 * c * r_ip) * inv, iz1 = (R21 * s + T21 * c * r_ip) * inv;
      const double om = r_ip * detJ * w[q];
      double dx[6], dz[6];
      for (int k = 0; k < 6; ++k) {
        dx[k] = ix0 * dN[q][0][k] + ix1 * dN[q][1][k];
        dz[k] = iz0 * dN[q][0][k] + iz1 * dN[q][1][k];
      }
      double e11, e13, e15, e33, e35, e55;
      if (C6) {
        const int64_t i = (int64_t)q * ld_C + e;
        e11 = C6[0][i] * visc; e33 = C6[1][i] * visc; e55 = C6[2][i] * visc;
        e13 = C6[3][i] * visc; e15 = C6[4][i] * visc; e35 = C6[5][i] * visc;
      } else {
        e11 = 4.0 / 3.0 * visc; e33 = 4.0 / 3.0 * visc; e55 = 1.0 * visc;
        e13 = -2.0 / 3.0 * visc; e15 = 0.0 * visc; e35 = 0.0 * visc;
      }
      int idx = 0;  /* the 78 entries in _fill_Kblk!'s loop order */
      for (int i = 0; i < 6; ++i) {
        const double xi = dx[i], zi = dz[i];
        for (int j = i; j < 6; ++j) {
          const double xj = dx[j], zj = dz[j];
          K[idx++] += om * (xi * (e11 * xj + e15 * zj) + zi * (e15 * xj + e55 * zj));
          K[idx++] += om * (xi * (e13 * zj + e15 * xj) + zi * (e35 * zj + e55 * xj));
        }
        for (int j = i; j < 6; ++j) {
          const double xj = dx[j], zj = dz[j];
          if (j > i) K[idx++] += om * (xi * (e15 * xj + e55 * zj) + zi * (e13 * xj + e35 * zj));
          K[idx++] += om * (xi * (e35 * zj + e55 * xj) + zi * (e33 * zj + e35 * xj));
        }
      }
      for (int i = 0; i < 3; ++i) {
        const double t = om * N3[q][i];
        for (int k = 0; k < 6; ++k) {
          G[i * 12 + 2 * k] += t * dx[k];
          G[i * 12 + 2 * k + 1] += t * dz[k];
        }
      }
      const double w3 = om / visc;
      for (int k = 0; k < 6; ++k) M[k] += w3 * N3[q][PACK3[k][0]] * N3[q][PACK3[k][1]];
      for (int k = 0; k < 6; ++k) {
        const double cte = om * fg * N[q][k];
        F[2 * k] += s * cte;
        F[2 * k + 1] += c * cte;
      }
    }
    for (int k = 0; k < 78; ++k) Kp[(int64_t)k * nel + e] = K[k];
    for (int k = 0; k < 36; ++k) Ge[(int64_t)k * nel + e] = G[k];
    for (int k = 0; k < 6; ++k) Me[(int64_t)k * nel + e] = M[k];
    for (int k = 0; k < 12; ++k) Fb[(int64_t)k * nel + e] = F[k];
  }
  return 0;
}
