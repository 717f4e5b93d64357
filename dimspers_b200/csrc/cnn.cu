// Learned initial guess for the Schur PCG: a small convolutional network on
// the polar grid of the half-resolution mesh's vertices (nrg = ncr/2 + 1
// radial x ntg = nct/2 angular points, periodic in theta), with hand-written
// forward, backward and Adam kernels.
//
// Network: L dilated 3x3 convolutions (zero padding in r, periodic in theta),
// ReLU after every layer but the last; inputs 4 channels (buoyancy rho,
// log10 eta, cos 2phi, sin 2phi of the director), output 1 channel: the
// pressure divided by g (Stokes is linear in the body force, so P/g does not
// depend on the Rayleigh number).  Activations are [batch][channel][r][theta]
// (theta fastest).  Each forward / data-gradient thread owns one grid point
// and all output channels, so every input value it loads is reused C times;
// weights sit in shared memory.  FP32 arithmetic: at C <= 32 and 65 x 512
// points a layer is ~0.6 GFLOP per sample, which CUDA cores cover in tens of
// microseconds.
//
// The predicted grid pressure is prolongated bilinearly to the pressure DOFs
// (discontinuous: the element's vertex values; continuous: vertex values) and
// handed to dp_solve with use_guess = 2, which keeps it only if it lowers the
// initial Schur residual.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

namespace dp {

constexpr int kCnnMaxC = 32;
constexpr int kCnnMaxLayers = 12;

struct Cnn {
  int nrg = 0, ntg = 0, C = 16, L = 6, cin = 4, device = 0;
  int bf16 = 1;                 // 1: BF16 tensor-core convolutions (FP32 accumulate), 0: FP32 CUDA cores
  __nv_bfloat16* wk = nullptr;  // the BF16 B operand of the current tensor-core convolution
  int dil[kCnnMaxLayers];
  int bmax = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  // parameters: per layer W[cout][cin][3][3] then b[cout], concatenated
  std::vector<int64_t> woff, boff;
  int64_t nparam = 0;
  float* param = nullptr;
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  int64_t step = 0;
  std::vector<float*> act;   // act[0] = input (external), act[l+1] = output of layer l
  float* dbuf0 = nullptr;    // gradient buffers (max size)
  float* dbuf1 = nullptr;
  double* partial = nullptr;
  unsigned int* counter = nullptr;
  double* loss = nullptr;
  double* h_loss = nullptr;
  int cin_of(int l) const { return l == 0 ? cin : C; }
  int cout_of(int l) const { return l == L - 1 ? 1 : C; }
  ~Cnn() {
    cudaFree(param); cudaFree(grad); cudaFree(adam_m); cudaFree(adam_v);
    for (size_t i = 1; i < act.size(); ++i) cudaFree(act[i]);
    cudaFree(dbuf0); cudaFree(dbuf1); cudaFree(partial); cudaFree(counter); cudaFree(loss); cudaFree(wk);
    cudaFreeHost(h_loss);
    if (stream) cudaStreamDestroy(stream);
  }
};

// ---- kernels -------------------------------------------------------------------
// Y[b][co][i][j] = b[co] + sum_ci sum_taps W[co][ci][ti][tj] X[b][ci][i+(ti-1)d][j+(tj-1)d]
template <int COUT>
__global__ void __launch_bounds__(256) k_conv_fwd(const float* __restrict__ X, const float* __restrict__ W,
                                                  const float* __restrict__ bias, float* __restrict__ Y, int cin,
                                                  int nrg, int ntg, int dil, int relu) {
  extern __shared__ float sw[];  // COUT * cin * 9 + COUT
  const int nw = COUT * cin * 9;
  for (int k = threadIdx.x; k < nw + COUT; k += blockDim.x) sw[k] = k < nw ? W[k] : bias[k - nw];
  __syncthreads();
  const int b = blockIdx.z, i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntg) return;
  float acc[COUT];
#pragma unroll
  for (int co = 0; co < COUT; ++co) acc[co] = sw[nw + co];
  const int64_t plane = (int64_t)nrg * ntg;
  for (int ci = 0; ci < cin; ++ci) {
    const float* Xc = X + ((int64_t)b * cin + ci) * plane;
#pragma unroll
    for (int ti = 0; ti < 3; ++ti) {
      const int ii = i + (ti - 1) * dil;
      if (ii < 0 || ii >= nrg) continue;
#pragma unroll
      for (int tj = 0; tj < 3; ++tj) {
        int jj = j + (tj - 1) * dil;
        jj = ((jj % ntg) + ntg) % ntg;
        const float xv = Xc[(int64_t)ii * ntg + jj];
#pragma unroll
        for (int co = 0; co < COUT; ++co) acc[co] += sw[(co * cin + ci) * 9 + ti * 3 + tj] * xv;
      }
    }
  }
#pragma unroll
  for (int co = 0; co < COUT; ++co) {
    float v = acc[co];
    if (relu && v < 0.f) v = 0.f;
    Y[((int64_t)b * COUT + co) * plane + (int64_t)i * ntg + j] = v;
  }
}

// ---- BF16 tensor-core convolutions (mma.sync m16n8k16, FP32 accumulation) ----------
// The forward convolution and the data gradient are both implicit GEMMs over
// the grid points: out[p][n] = sum_tap sum_k in[k][p + s*tap] * B[tap][n][k],
// with s = +1 (forward: k = input channel, n = output channel) or s = -1 (data
// gradient: k = output channel, n = input channel).  One warp computes 16
// consecutive theta points of one row times all NT*8 output columns; the K
// loop runs over the 9 taps and blocks of 16 channels.  A fragments are
// gathered from the FP32 activations and rounded to BF16; the B operand is
// the layer's weights rounded to BF16, laid out [tap][n][k] with a row stride
// of kpad + 8 elements, so the k pairs read from shared memory by a warp fall
// in distinct banks.
constexpr int kTcWarps = 4;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);   // .x (low half) = lo
  return *reinterpret_cast<const uint32_t*>(&v);
}

// D += A B for one 16x8x16 tile: A rows = grid points, columns = k; B = k x n.
// Fragment layout (PTX ISA, mma.m16n8k16 with .bf16): a[0] = (row g, k 2t..2t+1),
// a[1] = (row g+8, k 2t..2t+1), a[2] = (row g, k 2t+8..2t+9), a[3] = (row g+8,
// k 2t+8..2t+9); b0 = (k 2t..2t+1, col g), b1 = (k 2t+8..2t+9, col g); d[0..1] =
// (row g, col 2t..2t+1), d[2..3] = (row g+8, col 2t..2t+1), with g = lane/4,
// t = lane%4.
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// B operand of one layer: Bk[tap][n][k] (row stride kpad + 8) from W[co][ci][tap];
// forward n = co, k = ci; data gradient n = ci, k = co.  Zero outside the layer.
__global__ void k_conv_weights_bf16(const float* __restrict__ W, __nv_bfloat16* __restrict__ Bk, int cin, int cout,
                                    int npad, int kpad, int transpose) {
  const int ks = kpad + 8;
  const int total = 9 * npad * ks;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int tap = idx / (npad * ks), rem = idx % (npad * ks), n = rem / ks, k = rem % ks;
    const int co = transpose ? k : n, ci = transpose ? n : k;
    float v = 0.f;
    if (k < kpad && co < cout && ci < cin) v = W[(co * cin + ci) * 9 + tap];
    Bk[idx] = __float2bfloat16_rn(v);
  }
}

// out[b][n][i][j] = bias[n] + sum_tap sum_k X[b][k][i + s(ti-1)d][j + s(tj-1)d] Bk[tap][n][k]
// (zero rows outside [0, nrg), periodic in j), ReLU optional.  ntg % 16 == 0.
template <int NT>
__global__ void __launch_bounds__(kTcWarps * 32) k_conv_tc(const float* __restrict__ X,
                                                           const __nv_bfloat16* __restrict__ Bk,
                                                           const float* __restrict__ bias, float* __restrict__ Y,
                                                           int kch, int kpad, int nch, int nrg, int ntg, int dil,
                                                           int sgn, int relu) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __nv_bfloat16* sb = reinterpret_cast<__nv_bfloat16*>(smem_raw);
  const int ks = kpad + 8;
  const int nb_words = (9 * NT * 8 * ks) / 2;
  const uint32_t* gsrc = reinterpret_cast<const uint32_t*>(Bk);
  uint32_t* sdst = reinterpret_cast<uint32_t*>(sb);
  for (int w = threadIdx.x; w < nb_words; w += blockDim.x) sdst[w] = gsrc[w];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int b = blockIdx.z, i = blockIdx.y;
  const int j0 = (blockIdx.x * kTcWarps + warp) * 16;
  if (j0 >= ntg) return;                      // whole warps only (ntg is a multiple of 16)
  const int64_t plane = (int64_t)nrg * ntg;
  const float* Xb = X + (int64_t)b * kch * plane;
  float acc[NT][4];
#pragma unroll
  for (int nt = 0; nt < NT; ++nt)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
  for (int ti = 0; ti < 3; ++ti) {
    const int ii = i + sgn * (ti - 1) * dil;
    if (ii < 0 || ii >= nrg) continue;        // the same for the whole warp
    const float* row = Xb + (int64_t)ii * ntg;
    for (int tj = 0; tj < 3; ++tj) {
      int ja = j0 + g + sgn * (tj - 1) * dil;
      int jb = ja + 8;
      ja = ((ja % ntg) + ntg) % ntg;
      jb = ((jb % ntg) + ntg) % ntg;
      const __nv_bfloat16* bt = sb + (ti * 3 + tj) * NT * 8 * ks;
      for (int k0 = 0; k0 < kpad; k0 += 16) {
        const int c0 = k0 + 2 * t, c1 = c0 + 1, c2 = c0 + 8, c3 = c0 + 9;
        const float x0a = c0 < kch ? row[(int64_t)c0 * plane + ja] : 0.f;
        const float x1a = c1 < kch ? row[(int64_t)c1 * plane + ja] : 0.f;
        const float x0b = c0 < kch ? row[(int64_t)c0 * plane + jb] : 0.f;
        const float x1b = c1 < kch ? row[(int64_t)c1 * plane + jb] : 0.f;
        const float x2a = c2 < kch ? row[(int64_t)c2 * plane + ja] : 0.f;
        const float x3a = c3 < kch ? row[(int64_t)c3 * plane + ja] : 0.f;
        const float x2b = c2 < kch ? row[(int64_t)c2 * plane + jb] : 0.f;
        const float x3b = c3 < kch ? row[(int64_t)c3 * plane + jb] : 0.f;
        const uint32_t a[4] = {pack_bf16(x0a, x1a), pack_bf16(x0b, x1b), pack_bf16(x2a, x3a), pack_bf16(x2b, x3b)};
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const __nv_bfloat16* bn = bt + (nt * 8 + g) * ks + k0 + 2 * t;
          const uint32_t b0 = *reinterpret_cast<const uint32_t*>(bn);
          const uint32_t b1 = *reinterpret_cast<const uint32_t*>(bn + 8);
          mma_bf16_16816(acc[nt], a, b0, b1);
        }
      }
    }
  }
  float* Yb = Y + (int64_t)b * nch * plane + (int64_t)i * ntg;
#pragma unroll
  for (int nt = 0; nt < NT; ++nt) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int n = nt * 8 + 2 * t + (q & 1);
      const int j = j0 + g + ((q & 2) ? 8 : 0);
      if (n < nch) {
        float v = acc[nt][q] + (bias ? bias[n] : 0.f);
        if (relu && v < 0.f) v = 0.f;
        Yb[(int64_t)n * plane + j] = v;
      }
    }
  }
}

// dX[b][ci][i][j] = sum_co sum_taps W[co][ci][tap] dY[b][co][i-(ti-1)d][j-(tj-1)d]
template <int CIN>
__global__ void __launch_bounds__(256) k_conv_bwd_data(const float* __restrict__ dY, const float* __restrict__ W,
                                                       float* __restrict__ dX, int cout, int nrg, int ntg, int dil) {
  extern __shared__ float sw[];  // cout * CIN * 9
  const int nw = cout * CIN * 9;
  for (int k = threadIdx.x; k < nw; k += blockDim.x) sw[k] = W[k];
  __syncthreads();
  const int b = blockIdx.z, i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= ntg) return;
  float acc[CIN];
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.f;
  const int64_t plane = (int64_t)nrg * ntg;
  for (int co = 0; co < cout; ++co) {
    const float* Dc = dY + ((int64_t)b * cout + co) * plane;
#pragma unroll
    for (int ti = 0; ti < 3; ++ti) {
      const int ii = i - (ti - 1) * dil;
      if (ii < 0 || ii >= nrg) continue;
#pragma unroll
      for (int tj = 0; tj < 3; ++tj) {
        int jj = j - (tj - 1) * dil;
        jj = ((jj % ntg) + ntg) % ntg;
        const float dv = Dc[(int64_t)ii * ntg + jj];
#pragma unroll
        for (int ci = 0; ci < CIN; ++ci) acc[ci] += sw[(co * CIN + ci) * 9 + ti * 3 + tj] * dv;
      }
    }
  }
#pragma unroll
  for (int ci = 0; ci < CIN; ++ci) dX[((int64_t)b * CIN + ci) * plane + (int64_t)i * ntg + j] = acc[ci];
}

// One block per (co, ci): dW[co][ci][taps] (and db[co] when ci == 0) reduced over
// batch and grid points in a fixed order (deterministic).
__global__ void __launch_bounds__(256) k_conv_bwd_w(const float* __restrict__ X, const float* __restrict__ dY,
                                                    float* __restrict__ dW, float* __restrict__ db, int cin, int cout,
                                                    int nb, int nrg, int ntg, int dil) {
  const int co = blockIdx.x / cin, ci = blockIdx.x % cin;
  const int64_t plane = (int64_t)nrg * ntg;
  float acc[10];
#pragma unroll
  for (int k = 0; k < 10; ++k) acc[k] = 0.f;
  const int64_t npos = (int64_t)nb * plane;
  for (int64_t pidx = threadIdx.x; pidx < npos; pidx += blockDim.x) {
    const int b = (int)(pidx / plane);
    const int64_t rem = pidx % plane;
    const int i = (int)(rem / ntg), j = (int)(rem % ntg);
    const float g = dY[((int64_t)b * cout + co) * plane + rem];
    if (g == 0.f) continue;
    const float* Xc = X + ((int64_t)b * cin + ci) * plane;
#pragma unroll
    for (int ti = 0; ti < 3; ++ti) {
      const int ii = i + (ti - 1) * dil;
      if (ii < 0 || ii >= nrg) continue;
#pragma unroll
      for (int tj = 0; tj < 3; ++tj) {
        int jj = j + (tj - 1) * dil;
        jj = ((jj % ntg) + ntg) % ntg;
        acc[ti * 3 + tj] += g * Xc[(int64_t)ii * ntg + jj];
      }
    }
    acc[9] += g;
  }
  __shared__ float sh[10][8];
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    float v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 10) {
    float v = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sh[threadIdx.x][w];
    if (threadIdx.x < 9) dW[(co * cin + ci) * 9 + threadIdx.x] = v;
    else if (ci == 0) db[co] = v;
  }
}

// gradient through ReLU: d *= (a > 0)
__global__ void k_relu_bwd(float* __restrict__ d, const float* __restrict__ a, int64_t n) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n && !(a[i] > 0.f)) d[i] = 0.f;
}

// MSE loss L = mean (y - t)^2 and dL/dy
__global__ void __launch_bounds__(kRedThreads) k_mse(const float* __restrict__ y, const float* __restrict__ t,
                                                     float* __restrict__ g, int64_t n, double* partial,
                                                     unsigned int* counter, double* out) {
  double s = 0.0;
  const float inv = 2.0f / (float)n;
  for (int64_t i = blockIdx.x * (int64_t)kRedThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kRedThreads) {
    const float d = y[i] - t[i];
    g[i] = inv * d;
    s += (double)d * (double)d;
  }
  double v[1] = {s / (double)n};
  double* o[1] = {out};
  grid_finish<1>(v, partial, counter, o);
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ---- host: layer dispatch ----------------------------------------------------------
template <int N>
static void conv_fwd_n(Cnn& n, int l, const float* X, float* Y, int nb) {
  const int cin = n.cin_of(l);
  const size_t smem = sizeof(float) * (N * cin * 9 + N);
  dim3 grid((unsigned)div_up(n.ntg, 256), (unsigned)n.nrg, (unsigned)nb);
  ++g_klaunch;
  k_conv_fwd<N><<<grid, 256, smem, n.stream>>>(X, n.param + n.woff[l], n.param + n.boff[l], Y, cin, n.nrg, n.ntg,
                                                 n.dil[l], l < n.L - 1 ? 1 : 0);
}
static void conv_fwd(Cnn& n, int l, const float* X, float* Y, int nb) {
  switch (n.cout_of(l)) {
    case 1: conv_fwd_n<1>(n, l, X, Y, nb); break;
    case 8: conv_fwd_n<8>(n, l, X, Y, nb); break;
    case 16: conv_fwd_n<16>(n, l, X, Y, nb); break;
    case 32: conv_fwd_n<32>(n, l, X, Y, nb); break;
    default: throw std::runtime_error("unsupported channel count");
  }
  DP_LAUNCH_CHECK();
}
template <int N>
static void conv_bwd_data_n(Cnn& n, int l, const float* dY, float* dX, int nb) {
  const int cout = n.cout_of(l);
  const size_t smem = sizeof(float) * (cout * N * 9);
  dim3 grid((unsigned)div_up(n.ntg, 256), (unsigned)n.nrg, (unsigned)nb);
  ++g_klaunch;
  k_conv_bwd_data<N><<<grid, 256, smem, n.stream>>>(dY, n.param + n.woff[l], dX, cout, n.nrg, n.ntg, n.dil[l]);
}
static void conv_bwd_data(Cnn& n, int l, const float* dY, float* dX, int nb) {
  switch (n.cin_of(l)) {
    case 4: conv_bwd_data_n<4>(n, l, dY, dX, nb); break;
    case 8: conv_bwd_data_n<8>(n, l, dY, dX, nb); break;
    case 16: conv_bwd_data_n<16>(n, l, dY, dX, nb); break;
    case 32: conv_bwd_data_n<32>(n, l, dY, dX, nb); break;
    default: throw std::runtime_error("unsupported channel count");
  }
  DP_LAUNCH_CHECK();
}

// ---- tensor-core dispatch ------------------------------------------------------------
static int pad16(int c) { return (c + 15) / 16 * 16; }
static int ntiles(int c) { return (c + 7) / 8; }
// elements of a layer's B operand: forward (n = cout, k = cin) or data gradient (n = cin, k = cout)
static int64_t wk_elems(int cin, int cout, bool transpose) {
  const int nch = transpose ? cin : cout, kch = transpose ? cout : cin;
  return 9LL * ntiles(nch) * 8 * (pad16(kch) + 8);
}
static bool tc_ok(const Cnn& n) { return n.bf16 && n.ntg % 16 == 0; }

template <int NT>
static void conv_tc_n(Cnn& n, const float* X, const __nv_bfloat16* Bk, const float* bias, float* Y, int kch, int nch,
                      int dil, int sgn, int relu, int nb) {
  const int kpad = pad16(kch);
  const size_t smem = sizeof(__nv_bfloat16) * 9 * NT * 8 * (kpad + 8);
  dim3 grid((unsigned)div_up(n.ntg, 16 * kTcWarps), (unsigned)n.nrg, (unsigned)nb);
  ++g_klaunch;
  k_conv_tc<NT><<<grid, kTcWarps * 32, smem, n.stream>>>(X, Bk, bias, Y, kch, kpad, nch, n.nrg, n.ntg, dil, sgn,
                                                          relu);
  DP_LAUNCH_CHECK();
}
static void conv_tc(Cnn& n, const float* X, const __nv_bfloat16* Bk, const float* bias, float* Y, int kch, int nch,
                    int dil, int sgn, int relu, int nb) {
  switch (ntiles(nch)) {
    case 1: conv_tc_n<1>(n, X, Bk, bias, Y, kch, nch, dil, sgn, relu, nb); break;
    case 2: conv_tc_n<2>(n, X, Bk, bias, Y, kch, nch, dil, sgn, relu, nb); break;
    case 4: conv_tc_n<4>(n, X, Bk, bias, Y, kch, nch, dil, sgn, relu, nb); break;
    default: throw std::runtime_error("unsupported channel count");
  }
}
// rounds layer l's weights to the BF16 B operand (forward or data gradient) in n.wk
static const __nv_bfloat16* conv_weights(Cnn& n, int l, bool transpose) {
  const int cin = n.cin_of(l), cout = n.cout_of(l);
  const int nch = transpose ? cin : cout, kch = transpose ? cout : cin;
  const int64_t total = wk_elems(cin, cout, transpose);
  ++g_klaunch;
  k_conv_weights_bf16<<<(int)std::min<int64_t>(div_up(total, 256), 1024), 256, 0, n.stream>>>(
      n.param + n.woff[l], n.wk, cin, cout, ntiles(nch) * 8, pad16(kch), transpose ? 1 : 0);
  DP_LAUNCH_CHECK();
  return n.wk;
}

static void cnn_forward(Cnn& n, const float* x, int nb) {
  n.act[0] = const_cast<float*>(x);
  for (int l = 0; l < n.L; ++l) {
    if (tc_ok(n)) {
      const __nv_bfloat16* Bk = conv_weights(n, l, false);
      conv_tc(n, n.act[l], Bk, n.param + n.boff[l], n.act[l + 1], n.cin_of(l), n.cout_of(l), n.dil[l], 1,
              l < n.L - 1 ? 1 : 0, nb);
    } else {
      conv_fwd(n, l, n.act[l], n.act[l + 1], nb);
    }
  }
}

// forward + backward; returns the device loss in n.loss
static void cnn_fwd_bwd(Cnn& n, const float* x, const float* t, int nb) {
  cnn_forward(n, x, nb);
  const int64_t plane = (int64_t)n.nrg * n.ntg;
  const int64_t nout = (int64_t)nb * plane;
  float* g = n.dbuf0;
  float* g2 = n.dbuf1;
  ++g_klaunch;
  k_mse<<<red_grid(nout), kRedThreads, 0, n.stream>>>(n.act[n.L], t, g, nout, n.partial, n.counter, n.loss);
  DP_LAUNCH_CHECK();
  for (int l = n.L - 1; l >= 0; --l) {
    const int cin = n.cin_of(l), cout = n.cout_of(l);
    if (l < n.L - 1) {
      ++g_klaunch;
      k_relu_bwd<<<(int)div_up(nb * cout * plane, 256), 256, 0, n.stream>>>(g, n.act[l + 1], nb * cout * plane);
    }
    ++g_klaunch;
    k_conv_bwd_w<<<cout * cin, 256, 0, n.stream>>>(n.act[l], g, n.grad + n.woff[l], n.grad + n.boff[l], cin, cout, nb,
                                                   n.nrg, n.ntg, n.dil[l]);
    DP_LAUNCH_CHECK();
    if (l > 0) {
      if (tc_ok(n)) {
        const __nv_bfloat16* Bk = conv_weights(n, l, true);
        conv_tc(n, g, Bk, nullptr, g2, cout, cin, n.dil[l], -1, 0, nb);
      } else {
        conv_bwd_data(n, l, g, g2, nb);
      }
      std::swap(g, g2);
    }
  }
}

// ---- input features and the prolongation of the predicted pressure -----------------
// grid point (i, j) = fine vertex (2i, 2j) = lattice node (4i, 4j); features from the
// element of type 0 in fine cell (min(2i, ncr-1), 2j)
__global__ void k_cnn_inputs(const double* __restrict__ rho_lat, const double* __restrict__ eta,
                             const double* __restrict__ C, int mat_kind, int nel, int ncr, int nct, int A,
                             float* __restrict__ X, int nrg, int ntg) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
  if (j >= ntg) return;
  const int a = 4 * i, b = 4 * j;
  const int ir = min(2 * i, ncr - 1), it = 2 * j;
  const int e = 2 * (ir + ncr * it);
  double le = 0.0;
  for (int ip = 0; ip < 6; ++ip) le += log10(eta[(size_t)ip * nel + e]);
  double c2 = 1.0, s2 = 0.0;
  if (mat_kind == MAT_TI) {
    const double dx = C[nel + e], dy = C[2 * (size_t)nel + e];
    const double nn = dx * dx + dy * dy;
    if (nn > 0) { c2 = (dx * dx - dy * dy) / nn; s2 = 2.0 * dx * dy / nn; }
  }
  const int64_t plane = (int64_t)nrg * ntg, off = (int64_t)i * ntg + j;
  X[off] = (float)rho_lat[a + (int64_t)A * b];
  X[plane + off] = (float)(le / 6.0);
  X[2 * plane + off] = (float)c2;
  X[3 * plane + off] = (float)s2;
}

// bilinear value of the grid field at fine vertex (ir, it) = grid (ir/2, it/2)
__device__ inline double grid_at(const float* p, int ir, int it, int nrg, int ntg) {
  const int i0 = ir >> 1, j0 = it >> 1;
  const int i1 = (ir & 1) ? min(i0 + 1, nrg - 1) : i0;
  const int j1 = (it & 1) ? (j0 + 1 == ntg ? 0 : j0 + 1) : j0;
  return 0.25 * ((double)p[(int64_t)i0 * ntg + j0] + (double)p[(int64_t)i1 * ntg + j0] +
                 (double)p[(int64_t)i0 * ntg + j1] + (double)p[(int64_t)i1 * ntg + j1]);
}

__global__ void k_guess_prolong(const float* __restrict__ pg, int nrg, int ntg, double scale, int ncr, int nct,
                                int pressure, double* __restrict__ P, int nel) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nel) return;
  const int q = e >> 1, t = e & 1;
  const int ir = q % ncr, it = q / ncr;
  const int it1 = it + 1 == nct ? 0 : it + 1;
  int vr[3], vt[3];
  if (t == 0) { vr[0] = ir; vt[0] = it; vr[1] = ir; vt[1] = it1; vr[2] = ir + 1; vt[2] = it; }
  else { vr[0] = ir; vt[0] = it1; vr[1] = ir + 1; vt[1] = it1; vr[2] = ir + 1; vt[2] = it; }
  for (int k = 0; k < 3; ++k) {
    const double v = scale * grid_at(pg, vr[k], vt[k], nrg, ntg);
    if (pressure == 1) P[3 * (int64_t)e + k] = v;
    else P[vr[k] + (int64_t)(ncr + 1) * vt[k]] = v;  // shared vertices get identical values
  }
}

}  // namespace dp

struct dp_cnn {
  dp::Cnn n;
};

using namespace dp;

extern "C" {

int dp_cnn_create(int32_t nrg, int32_t ntg, int32_t channels, int32_t layers, const int32_t* dilations,
                  int32_t max_batch, int32_t device, dp_cnn** out) {
  if (!out) return DP_BAD_ARG;
  *out = nullptr;
  dp_cnn* h = nullptr;
  int st = guarded(nullptr, [&] {
    if (nrg < 2 || ntg < 3 || layers < 2 || layers > kCnnMaxLayers || max_batch < 1)
      throw BadArg("invalid network shape");
    if (channels != 8 && channels != 16 && channels != 32) throw BadArg("channels must be 8, 16 or 32");
    h = new dp_cnn();
    Cnn& n = h->n;
    n.nrg = nrg; n.ntg = ntg; n.C = channels; n.L = layers; n.device = device; n.bmax = max_batch;
    for (int l = 0; l < layers; ++l) {
      n.dil[l] = dilations ? dilations[l] : 1;
      if (n.dil[l] < 1 || n.dil[l] >= nrg) throw BadArg("invalid dilation");
    }
    DP_CUDA(cudaSetDevice(device));
    DP_CUDA(cudaStreamCreateWithFlags(&n.stream, cudaStreamNonBlocking));
    int64_t off = 0;
    for (int l = 0; l < layers; ++l) {
      n.woff.push_back(off);
      off += (int64_t)n.cout_of(l) * n.cin_of(l) * 9;
      n.boff.push_back(off);
      off += n.cout_of(l);
    }
    n.nparam = off;
    DP_CUDA(cudaMalloc(&n.param, sizeof(float) * off));
    DP_CUDA(cudaMalloc(&n.grad, sizeof(float) * off));
    DP_CUDA(cudaMalloc(&n.adam_m, sizeof(float) * off));
    DP_CUDA(cudaMalloc(&n.adam_v, sizeof(float) * off));
    DP_CUDA(cudaMemset(n.param, 0, sizeof(float) * off));
    DP_CUDA(cudaMemset(n.adam_m, 0, sizeof(float) * off));
    DP_CUDA(cudaMemset(n.adam_v, 0, sizeof(float) * off));
    const int64_t plane = (int64_t)nrg * ntg;
    n.act.assign(layers + 1, nullptr);
    for (int l = 0; l < layers; ++l) DP_CUDA(cudaMalloc(&n.act[l + 1], sizeof(float) * max_batch * n.cout_of(l) * plane));
    const int64_t gmax = (int64_t)max_batch * std::max(channels, 4) * plane;
    DP_CUDA(cudaMalloc(&n.dbuf0, sizeof(float) * gmax));
    DP_CUDA(cudaMalloc(&n.dbuf1, sizeof(float) * gmax));
    int64_t wmax = 0;
    for (int l = 0; l < layers; ++l)
      wmax = std::max({wmax, wk_elems(n.cin_of(l), n.cout_of(l), false), wk_elems(n.cin_of(l), n.cout_of(l), true)});
    DP_CUDA(cudaMalloc(&n.wk, sizeof(__nv_bfloat16) * wmax));
    DP_CUDA(cudaMalloc(&n.partial, sizeof(double) * 4 * kRedBlocks));
    DP_CUDA(cudaMalloc(&n.counter, sizeof(unsigned int)));
    DP_CUDA(cudaMemset(n.counter, 0, sizeof(unsigned int)));
    DP_CUDA(cudaMalloc(&n.loss, sizeof(double)));
    DP_CUDA(cudaMallocHost(&n.h_loss, sizeof(double)));
    return (int)DP_OK;
  });
  if (st != DP_OK) {
    delete h;
    return st;
  }
  *out = h;
  return DP_OK;
}

void dp_cnn_destroy(dp_cnn* h) {
  if (!h) return;
  cudaSetDevice(h->n.device);
  if (h->n.stream) cudaStreamSynchronize(h->n.stream);
  delete h;
}

int64_t dp_cnn_num_params(const dp_cnn* h) { return h ? h->n.nparam : -1; }

int dp_cnn_set_math(dp_cnn* h, int32_t bf16) {
  if (!h || bf16 < 0 || bf16 > 1) return DP_BAD_ARG;
  h->n.bf16 = bf16;
  return DP_OK;
}

int dp_cnn_set_params(dp_cnn* h, const float* p, int64_t n) {
  if (!h || !p || n != h->n.nparam) return DP_BAD_ARG;
  return guarded(nullptr, [&] {
    DP_CUDA(cudaSetDevice(h->n.device));
    DP_CUDA(cudaMemcpy(h->n.param, p, sizeof(float) * n, cudaMemcpyHostToDevice));
    DP_CUDA(cudaMemset(h->n.adam_m, 0, sizeof(float) * n));
    DP_CUDA(cudaMemset(h->n.adam_v, 0, sizeof(float) * n));
    h->n.step = 0;
    return (int)DP_OK;
  });
}

int dp_cnn_get_params(dp_cnn* h, float* p, float* g, int64_t n) {
  if (!h || n != h->n.nparam) return DP_BAD_ARG;
  return guarded(nullptr, [&] {
    DP_CUDA(cudaSetDevice(h->n.device));
    if (p) DP_CUDA(cudaMemcpy(p, h->n.param, sizeof(float) * n, cudaMemcpyDeviceToHost));
    if (g) DP_CUDA(cudaMemcpy(g, h->n.grad, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return (int)DP_OK;
  });
}

int dp_cnn_forward(dp_cnn* h, const float* x, float* y, int32_t nb) {
  if (!h || !x || !y || nb < 1 || nb > h->n.bmax) return DP_BAD_ARG;
  return guarded(nullptr, [&] {
    Cnn& n = h->n;
    DP_CUDA(cudaSetDevice(n.device));
    cnn_forward(n, x, nb);
    DP_CUDA(cudaMemcpyAsync(y, n.act[n.L], sizeof(float) * nb * (int64_t)n.nrg * n.ntg, cudaMemcpyDeviceToDevice,
                            n.stream));
    DP_CUDA(cudaStreamSynchronize(n.stream));
    return (int)DP_OK;
  });
}

int dp_cnn_gradients(dp_cnn* h, const float* x, const float* t, int32_t nb, double* loss) {
  if (!h || !x || !t || nb < 1 || nb > h->n.bmax) return DP_BAD_ARG;
  return guarded(nullptr, [&] {
    Cnn& n = h->n;
    DP_CUDA(cudaSetDevice(n.device));
    cnn_fwd_bwd(n, x, t, nb);
    DP_CUDA(cudaMemcpyAsync(n.h_loss, n.loss, sizeof(double), cudaMemcpyDeviceToHost, n.stream));
    DP_CUDA(cudaStreamSynchronize(n.stream));
    if (loss) *loss = *n.h_loss;
    return (int)DP_OK;
  });
}

int dp_cnn_train_step(dp_cnn* h, const float* x, const float* t, int32_t nb, float lr, double* loss) {
  if (!h || !x || !t || nb < 1 || nb > h->n.bmax || !(lr > 0.f)) return DP_BAD_ARG;
  return guarded(nullptr, [&] {
    Cnn& n = h->n;
    DP_CUDA(cudaSetDevice(n.device));
    cnn_fwd_bwd(n, x, t, nb);
    n.step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)n.step), c2 = 1.f - std::pow(b2, (float)n.step);
    ++g_klaunch;
    k_adam<<<(int)div_up(n.nparam, 256), 256, 0, n.stream>>>(n.param, n.grad, n.adam_m, n.adam_v, n.nparam, lr, b1,
                                                               b2, 1e-8f, c1, c2);
    DP_LAUNCH_CHECK();
    DP_CUDA(cudaMemcpyAsync(n.h_loss, n.loss, sizeof(double), cudaMemcpyDeviceToHost, n.stream));
    DP_CUDA(cudaStreamSynchronize(n.stream));
    if (loss) *loss = *n.h_loss;
    return (int)DP_OK;
  });
}

int dp_cnn_inputs(dp_ctx* h, float* x, int32_t nrg, int32_t ntg) {
  if (!h || !x) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (c.fine.ncr % 2 || c.fine.nct % 2) throw BadArg("the guess grid needs even cell counts");
    if (nrg != c.fine.ncr / 2 + 1 || ntg != c.fine.nct / 2) throw BadArg("grid must be (ncr/2+1) x (nct/2)");
    if (c.mat_kind == MAT_NONE) throw BadArg("material not set");
    dim3 grid((unsigned)div_up(ntg, 128), (unsigned)nrg);
    ++g_klaunch;
    k_cnn_inputs<<<grid, 128, 0, c.stream>>>(c.rho_lat, c.eta, c.C, c.mat_kind, (int)c.fine.nel, c.fine.ncr,
                                             c.fine.nct, (int)c.fine.A(), x, nrg, ntg);
    DP_LAUNCH_CHECK();
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

int dp_guess_from_grid(dp_ctx* h, const float* pg, int32_t nrg, int32_t ntg, double scale, double* P, int32_t mem) {
  if (!h || !pg || !P) return DP_BAD_ARG;
  Ctx& c = h->c;
  return guarded(&c, [&] {
    DP_CUDA(cudaSetDevice(c.device));
    if (nrg != c.fine.ncr / 2 + 1 || ntg != c.fine.nct / 2) throw BadArg("grid must be (ncr/2+1) x (nct/2)");
    double* dP = (double*)c.work[W_P];
    ++g_klaunch;
    k_guess_prolong<<<(int)div_up(c.fine.nel, 256), 256, 0, c.stream>>>(pg, nrg, ntg, scale, c.fine.ncr, c.fine.nct,
                                                                        c.mesh.pressure, dP, (int)c.fine.nel);
    DP_LAUNCH_CHECK();
    DP_CUDA(cudaMemcpyAsync(P, dP, sizeof(double) * c.mesh.npres, kind_out(mem), c.stream));
    DP_CUDA(cudaStreamSynchronize(c.stream));
    return (int)DP_OK;
  });
}

}  // extern "C"
