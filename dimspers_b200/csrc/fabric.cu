// Per-IP finite-strain ellipsoid and DEM viscous tensor: getFSE / _FSE
// (src/Stress/FSE.jl:131-161) and anisotropic_tensor (src/Rheology/
// anisotropy.jl:140-285), the producers of the StiffnessTensor fields the
// Stokes assembly reads (MAIN.jl:262-269).
//
// k_fse_ip: one thread per (IP, element), the closed-form eigen-decomposition
// of L = F F^T shared with the per-element director.
// k_dem_tensor: one warp per (IP, 32 elements), IP 7 the mean of IPs 1..6
// through shared memory.  Per
// IP the nearest DEM row by the reference's argminsorted scans (first i with
// |r - b[i]| < |r - b[i+1]|, the same comparisons on the same values, so the
// row chosen is the reference's), then directRotation2D by the FSE axis.  The
// table (100 rows in the reference's DEM files) stays in L1/L2.
#include "kernels.cuh"

namespace dp {

struct DemDev {
  const double* C;        // nrows x 9 column-major
  const double* b1;       // a1a2_blk (n1)
  const double* b2;       // a2a3_blk (sblk, sorted)
  const int64_t* perm;    // 1-based (sblk)
  int64_t nrows;
  int n1, sblk;
  double w;
};

// F: 4 doubles per (ip, e) at (ip * nel + e) * 4; out: field-major 6 x n
// (vx1, vx2, vy1, vy2, a1, a2), n = 6 nel (ip * nel + e).
__global__ void __launch_bounds__(256) k_fse_ip(const double* __restrict__ F, double* __restrict__ out, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 f0 = reinterpret_cast<const double2*>(F)[2 * i];
  const double2 f1 = reinterpret_cast<const double2*>(F)[2 * i + 1];
  double vx, vy, l1, l2;
  fse_axes(f0.x, f0.y, f1.x, f1.y, vx, vy, l1, l2);
  out[i] = vx;
  out[n + i] = -vy;  // minor axis, perpendicular to the major one
  out[2 * n + i] = vy;
  out[3 * n + i] = vx;
  out[4 * n + i] = sqrt(fabs(l1));
  out[5 * n + i] = sqrt(fabs(l2));
}

// argminsorted (anisotropy.jl:110-118), 0-based
__device__ __forceinline__ int argmin_sorted(double r, const double* __restrict__ b, int m) {
  double prev = fabs(r - b[0]);
  for (int i = 0; i < m - 1; ++i) {
    const double nxt = fabs(r - b[i + 1]);
    if (prev < nxt) return i;
    prev = nxt;
  }
  return m - 1;
}

// Julia's max for a value that may be NaN against a finite floor
__device__ __forceinline__ double jmax(double v, double w) { return v != v ? v : (v > w ? v : w); }

// directRotation2D (anisotropy.jl:503-536) of the tensor (a = C11, c = C33,
// e = C55, h = C13) by R = (cos, sin, -sin)
__device__ __forceinline__ void direct_rotation_2d(double cosa, double sina, double a, double c, double e, double h,
                                                   double n[6]) {
  const double x1 = cosa, y2 = cosa, x2 = sina, y1 = -sina;
  const double x1x1 = x1 * x1, x2x2 = x2 * x2, y1y1 = y1 * y1, y2y2 = y2 * y2;
  const double m = x1 * y2 + x2 * y1;
  n[0] = (c * x2x2 + h * x1x1 + 4 * e * x1x1) * x2x2 + (a * x1x1 + h * x2x2) * x1x1;
  n[1] = (c * y2y2 + h * y1y1 + 4 * e * y1y1) * y2y2 + (a * y1y1 + h * y2y2) * y1y1;
  n[2] = (c * x2 * y2 + h * x1 * y1) * x2 * y2 + m * m * e + (a * x1 * y1 + h * x2 * y2) * x1 * y1;
  n[3] = ((c * x2x2 + h * x1x1) * y2 + 4 * e * x1 * x2 * y1) * y2 + (a * x1x1 + h * x2x2) * y1y1;
  n[4] = ((c * x2x2 + h * x1x1) * y2 + 2 * m * e * x1) * x2 + (a * x1x1 + h * x2x2) * x1 * y1;
  n[5] = ((c * y2y2 + h * y1y1) * x2 + 2 * m * e * y1) * y2 + (a * y1y1 + h * y2y2) * x1 * y1;
}

constexpr int kDemEl = 32;  // elements per CTA: warps 0..5 one IP each, warp 6 the IP-7 mean

// in: field-major 4 x 6 nel (vx1, vy1, r1, r2; ip * nel + e); out: 6 x 7 nel.
// Every load and store is a coalesced row of an element-fastest matrix.
__global__ void __launch_bounds__(kDemEl * 7) k_dem_tensor(const double* __restrict__ in, double* __restrict__ out,
                                                           DemDev d, int nel) {
  __shared__ double sh[6][6][kDemEl];  // field, ip, element
  const int tx = threadIdx.x, ip = threadIdx.y;
  const int e = blockIdx.x * kDemEl + tx;
  const bool valid = e < nel;
  const size_t st = (size_t)nel, n6 = 6 * st, n7 = 7 * st;
  if (valid && ip < 6) {
    const size_t i = (size_t)ip * st + e;
    const double x = in[i], y = in[n6 + i], r1 = in[2 * n6 + i], r2 = in[3 * n6 + i];
    const int i1 = argmin_sorted(r1, d.b1, d.n1);
    const int64_t i2 = d.perm[argmin_sorted(r2, d.b2, d.sblk)];  // 1-based, checked on the host
    const int64_t row = (int64_t)d.sblk * i1 + i2 - 1;
    const double a = d.C[row], c = d.C[2 * d.nrows + row];
    const double ee = jmax(d.C[4 * d.nrows + row], d.w), h = d.C[7 * d.nrows + row];
    const double hh = 1.0 / sqrt(y * y + x * x);  // rotmatrix (anisotropy.jl:287-292)
    double n[6];
    direct_rotation_2d(x * hh, y * hh, a, c, ee, h, n);
    n[2] = jmax(n[2], d.w);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      out[k * n7 + i] = n[k];
      sh[k][ip][tx] = n[k];
    }
  }
  __syncthreads();
  if (valid && ip == 6) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double acc = 0.0;
#pragma unroll
      for (int q = 0; q < 6; ++q) acc += sh[k][q][tx];
      out[k * n7 + 6 * st + e] = acc * (1.0 / 6.0);
    }
  }
}

static DemDev staged_dem(Ctx& c, double* tab) {
  DemDev d;
  d.C = tab;
  d.b1 = tab + 9 * c.fabric_dem[0];
  d.b2 = d.b1 + c.fabric_dem[1];
  d.perm = reinterpret_cast<const int64_t*>(d.b2 + c.fabric_dem[2]);
  d.nrows = c.fabric_dem[0];
  d.n1 = (int)c.fabric_dem[1];
  d.sblk = (int)c.fabric_dem[2];
  d.w = c.fabric_w;
  return d;
}

static void launch_k_dem_tensor(Ctx& c, const double* in, double* o, const DemDev& d) {
  const int64_t nel = c.fine.nel;
  ++g_klaunch;
  k_dem_tensor<<<(int)div_up(nel, kDemEl), dim3(kDemEl, 7), 0, c.stream>>>(in, o, d, (int)nel);
  DP_LAUNCH_CHECK();
}

// k_dem_tensor on the inputs and table staged by the last
// dp_anisotropic_tensor call (kernel timing)
void launch_dem_staged(Ctx& c) {
  const int64_t nel = c.fine.nel;
  double* in = c.fabric_buf;
  launch_k_dem_tensor(c, in, in + 24 * nel, staged_dem(c, in + 66 * nel));
}

static double* fabric_scratch(Ctx& c, int64_t n) {
  if (c.fabric_cap < n) {
    cudaFree(c.fabric_buf);
    c.fabric_buf = nullptr;
    c.fabric_cap = 0;
    dalloc(&c.fabric_buf, (size_t)n);
    c.fabric_cap = n;
  }
  return c.fabric_buf;
}

}  // namespace dp

using namespace dp;

extern "C" int dp_fse(dp_ctx* h, const double* F, double* const* fse, int64_t ld_out, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!F || !fse) throw BadArg("null argument");
    for (int f = 0; f < 6; ++f)
      if (!fse[f]) throw BadArg("null output field");
    const int64_t nel = c.fine.nel, n = 6 * nel;
    if (ld_out < nel) throw BadArg("leading dimension below nel");
    double* buf = fabric_scratch(c, 4 * n + 6 * n);
    c.fabric_dem[0] = 0;  // the staged DEM table is overwritten
    double* dF = buf;
    double* o = buf + 4 * n;
    DP_CUDA(cudaMemcpyAsync(dF, F, sizeof(double) * 4 * n, kind_in(mem), c.stream));
    ++g_klaunch;
    k_fse_ip<<<(int)div_up(n, 256), 256, 0, c.stream>>>(dF, o, n);
    DP_LAUNCH_CHECK();
    for (int f = 0; f < 6; ++f)
      DP_CUDA(cudaMemcpy2DAsync(fse[f], sizeof(double) * ld_out, o + (size_t)f * n, sizeof(double) * nel,
                                sizeof(double) * nel, 6, kind_out(mem), c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

extern "C" int dp_anisotropic_tensor(dp_ctx* h, const dp_dem* dem, const double* vx1, const double* vy1,
                                     const double* r1, const double* r2, int64_t ld_in, double* const* C6_out,
                                     int64_t ld_out, int32_t mem) {
  if (!h) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (!dem || !vx1 || !vy1 || !r1 || !r2 || !C6_out) throw BadArg("null argument");
    for (int f = 0; f < 6; ++f)
      if (!C6_out[f]) throw BadArg("null output field");
    if (!dem->C || !dem->a1a2_blk || !dem->a2a3_blk || !dem->permutation_blk) throw BadArg("null DEM table");
    if (dem->sblk < 1 || dem->n_a1a2 < 1 || dem->sblk > (1 << 20) || dem->n_a1a2 > (1 << 20))
      throw BadArg("DEM block sizes out of range");
    if (dem->n_a1a2 * dem->sblk > dem->nrows) throw BadArg("n_a1a2 * sblk exceeds the DEM rows");
    for (int64_t k = 0; k < dem->sblk; ++k)
      if (dem->permutation_blk[k] < 1 || dem->permutation_blk[k] > dem->sblk)
        throw BadArg("permutation_blk entries must lie in 1..sblk");
    if (!std::isfinite(dem->w)) throw BadArg("cut-off w must be finite");
    const int64_t nel = c.fine.nel;
    if (ld_in < nel || ld_out < nel) throw BadArg("leading dimension below nel");
    const int64_t ntab = 9 * dem->nrows + dem->n_a1a2 + 2 * dem->sblk;
    double* buf = fabric_scratch(c, 24 * nel + 42 * nel + ntab);
    double* in = buf;
    double* o = in + 24 * nel;
    double* tab = o + 42 * nel;
    const cudaMemcpyKind kin = kind_in(mem);
    const double* src[4] = {vx1, vy1, r1, r2};
    for (int f = 0; f < 4; ++f)
      DP_CUDA(cudaMemcpy2DAsync(in + (size_t)f * 6 * nel, sizeof(double) * nel, src[f], sizeof(double) * ld_in,
                                sizeof(double) * nel, 6, kin, c.stream));
    c.fabric_dem[0] = dem->nrows;
    c.fabric_dem[1] = dem->n_a1a2;
    c.fabric_dem[2] = dem->sblk;
    c.fabric_w = dem->w;
    const DemDev d = staged_dem(c, tab);
    DP_CUDA(cudaMemcpyAsync(tab, dem->C, sizeof(double) * 9 * dem->nrows, cudaMemcpyHostToDevice, c.stream));
    DP_CUDA(cudaMemcpyAsync((void*)d.b1, dem->a1a2_blk, sizeof(double) * dem->n_a1a2, cudaMemcpyHostToDevice,
                            c.stream));
    DP_CUDA(cudaMemcpyAsync((void*)d.b2, dem->a2a3_blk, sizeof(double) * dem->sblk, cudaMemcpyHostToDevice,
                            c.stream));
    DP_CUDA(cudaMemcpyAsync((void*)d.perm, dem->permutation_blk, sizeof(int64_t) * dem->sblk,
                            cudaMemcpyHostToDevice, c.stream));
    launch_k_dem_tensor(c, in, o, d);
    for (int f = 0; f < 6; ++f)
      DP_CUDA(cudaMemcpy2DAsync(C6_out[f], sizeof(double) * ld_out, o + (size_t)f * 7 * nel, sizeof(double) * nel,
                                sizeof(double) * nel, 7, kind_out(mem), c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}
