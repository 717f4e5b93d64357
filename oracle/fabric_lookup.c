/* DEM viscous-tensor lookup per IP in plain C (FP64; test infrastructure): a
 * second restatement of anisotropic_tensor (src/Rheology/anisotropy.jl:
 * 140-285) beside oracle/fabric.py, for the CPU baseline.
 *
 * Per element and IP 1..6: argminsorted (:110-118) over a1a2_blk for r1 and
 * over the sorted a2a3_blk for r2, row sblk (i1 - 1) + permutation_blk[i2] of
 * the table, its C11, C33, max(C55, w), C13 rotated by rotmatrix(vx1, vy1)
 * (:287-292) with directRotation2D (:503-536), eta55 floored at w; IP 7 the
 * mean of IPs 1..6.  Inputs (nel, 6) and outputs (nel, 7) column-major; the
 * table C is (nrows, 9) column-major; permutation_blk 1-based.
 *
 * Build: gcc -O2 -fopenmp -shared -fPIC -o oracle/libfabric_lookup.so oracle/fabric_lookup.c -lm
 */
#include <math.h>
#include <stdint.h>
#include <omp.h>

static int argminsorted(double r, const double* b, int64_t m) {
  for (int64_t i = 0; i + 1 < m; ++i)
    if (fabs(r - b[i]) < fabs(r - b[i + 1])) return (int)i;
  return (int)(m - 1);
}

static double jmax(double v, double w) { return v != v ? v : (v > w ? v : w); }

int dpo_anisotropic_tensor(int64_t nel, const double* vx1, const double* vy1, const double* r1, const double* r2,
                           const double* C, int64_t nrows, const double* a1a2, int64_t n1, const double* a2a3,
                           const int64_t* perm, int64_t sblk, double w, double* const* out, int nthreads) {
  if (n1 < 1 || sblk < 1 || n1 * sblk > nrows) return 1;
  for (int64_t k = 0; k < sblk; ++k)
    if (perm[k] < 1 || perm[k] > sblk) return 1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < nel; ++e) {
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int ip = 0; ip < 6; ++ip) {
      const int64_t i = (int64_t)ip * nel + e;
      const int64_t i1 = argminsorted(r1[i], a1a2, n1);
      const int64_t i2 = perm[argminsorted(r2[i], a2a3, sblk)];
      const int64_t row = sblk * i1 + i2 - 1;
      const double a = C[row], c = C[2 * nrows + row], ee = jmax(C[4 * nrows + row], w), h = C[7 * nrows + row];
      const double x = vx1[i], y = vy1[i];
      const double hh = 1.0 / sqrt(y * y + x * x);
      const double x1 = x * hh, y2 = x * hh, x2 = y * hh, y1 = -(y * hh);
      const double x1x1 = x1 * x1, x2x2 = x2 * x2, y1y1 = y1 * y1, y2y2 = y2 * y2, m = x1 * y2 + x2 * y1;
      double n[6];
      n[0] = (c * x2x2 + h * x1x1 + 4 * ee * x1x1) * x2x2 + (a * x1x1 + h * x2x2) * x1x1;
      n[1] = (c * y2y2 + h * y1y1 + 4 * ee * y1y1) * y2y2 + (a * y1y1 + h * y2y2) * y1y1;
      n[2] = jmax((c * x2 * y2 + h * x1 * y1) * x2 * y2 + m * m * ee + (a * x1 * y1 + h * x2 * y2) * x1 * y1, w);
      n[3] = ((c * x2x2 + h * x1x1) * y2 + 4 * ee * x1 * x2 * y1) * y2 + (a * x1x1 + h * x2x2) * y1y1;
      n[4] = ((c * x2x2 + h * x1x1) * y2 + 2 * m * ee * x1) * x2 + (a * x1x1 + h * x2x2) * x1 * y1;
      n[5] = ((c * y2y2 + h * y1y1) * x2 + 2 * m * ee * y1) * y2 + (a * y1y1 + h * y2y2) * x1 * y1;
      for (int k = 0; k < 6; ++k) {
        out[k][i] = n[k];
        acc[k] += n[k];
      }
    }
    for (int k = 0; k < 6; ++k) out[k][(int64_t)6 * nel + e] = acc[k] * (1.0 / 6.0);
  }
  return 0;
}
