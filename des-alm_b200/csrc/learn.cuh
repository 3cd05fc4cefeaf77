// learn.cuh -- the learned initial guess for dual time stepping: a small 3D
// convolutional network that predicts the correction to the linear
// extrapolation 2 q^n - q^{n-1} of the next physical time level, trained
// online on the solutions the solver itself produces.
//
// Network (4 layers, 3x3x3 kernels, zero padding at the grid's edges):
//   15 -> 32 -> 32 -> 32 -> 5 channels, ReLU after the first three layers.
// Inputs per node: q^n, q^n - q^{n-1}, q^{n-1} - q^{n-2} of (p, u, v, w,
// nu_tilde), each divided by its RMS over the grid at that time level;
// output: (q^{n+1} - 2 q^n + q^{n-1}) / s, s = the RMS of q^n - q^{n-1}.  A
// difference channel whose RMS is below 1e-12 of the field's own RMS counts
// as still: its scale is zero, so its features, target and correction are zero.
//
// Activations are BF16, channel-major ([channel][node], nodes in the level's
// i-fastest order); products accumulate in FP32 on the tensor cores (WMMA,
// m16n16k16 BF16).  A convolution is an implicit GEMM: for each of the 27
// stencil offsets the CTA gathers the shifted input tile into shared memory
// and multiplies it by that offset's weight block.  The data gradient of a
// layer is the same kernel with the weights transposed and the stencil
// flipped; the weight gradient is a GEMM that reduces over the nodes.
// Master weights, Adam moments and the loss are FP32 / FP64.
#pragma once
#include <mma.h>
#include <cuda_bf16.h>
#include "common.cuh"

namespace desalm {

using bf16 = __nv_bfloat16;

constexpr int LP_TM = 128;           // nodes per tile
constexpr float LP_YMAX = 8.0f;      // default limit of |output| (in units of s) in the guess
constexpr int LP_LDA = LP_TM + 8;    // shared-memory row stride of a [channel][node] tile

struct LpGrid {
  int im, jm, km;
  long N;
};

// stencil offset o = 0..26 -> (di, dj, dk) in -1..1, o = (dk+1)*9 + (dj+1)*3 + (di+1)
DESALM_DEV void lp_offset(int o, int& di, int& dj, int& dk) {
  dk = o / 9 - 1;
  dj = (o / 3) % 3 - 1;
  di = o % 3 - 1;
}

// Shared-memory layout of k_lp_conv (bytes).
template <int CIN, int COUT_PAD>
struct LpConvSmem {
  static constexpr size_t w = size_t(27) * CIN * COUT_PAD * sizeof(bf16);
  static constexpr size_t a = size_t(CIN) * LP_LDA * sizeof(bf16);
  static constexpr size_t c = size_t(LP_TM) * (COUT_PAD + 4) * sizeof(float);
  static constexpr size_t crd = size_t(LP_TM) * 4 * sizeof(int);
  static constexpr size_t total = w + a + c + crd;
};

// out[co][l] = act(bias[co] + sum_{ci, o} W[o][ci][co] in[ci][l + off(o)]),
// neighbours outside the grid read as zero.  act: ReLU when relu != 0; when
// mask is given the result is multiplied by (mask[co][l] > 0) (the gradient
// through the ReLU that produced mask).  out, when given, gets cout_store
// channels in BF16; out32, when given, the same values in FP32.  Grid-stride over tiles of
// LP_TM nodes; the weights stay in shared memory for the CTA's lifetime.
template <int CIN, int COUT_PAD>
__global__ void __launch_bounds__(256) k_lp_conv(LpGrid G, const bf16* __restrict__ in, const bf16* __restrict__ wk,
                                                 const float* __restrict__ bias, int relu,
                                                 const bf16* __restrict__ mask, bf16* __restrict__ out,
                                                 float* __restrict__ out32, int cout_store) {
  pdl_wait();
  using namespace nvcuda;
  using SM = LpConvSmem<CIN, COUT_PAD>;
  constexpr int NF = COUT_PAD / 16, KC = CIN / 16;
  extern __shared__ __align__(128) unsigned char lp_smem[];
  bf16* Ws = reinterpret_cast<bf16*>(lp_smem);
  bf16* As = reinterpret_cast<bf16*>(lp_smem + SM::w);
  float* Cs = reinterpret_cast<float*>(lp_smem + SM::w + SM::a);
  int* crd = reinterpret_cast<int*>(lp_smem + SM::w + SM::a + SM::c);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int e = tid; e < 27 * CIN * COUT_PAD; e += blockDim.x) Ws[e] = wk[e];
  const long N = G.N;
  const long ntiles = (N + LP_TM - 1) / LP_TM;
  for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long l0 = tile * LP_TM;
    __syncthreads();  // weights loaded / previous tile's reads of As, Cs, crd done
    if (tid < LP_TM) {
      const long l = l0 + tid;
      const int i = int(l % G.im);
      const long r = l / G.im;
      crd[4 * tid + 0] = i;
      crd[4 * tid + 1] = int(r % G.jm);
      crd[4 * tid + 2] = int(r / G.jm);
      crd[4 * tid + 3] = l < N;
    }
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) wmma::fill_fragment(acc[f], 0.0f);
    for (int o = 0; o < 27; ++o) {
      int di, dj, dk;
      lp_offset(o, di, dj, dk);
      const long off = di + (long)G.im * (dj + (long)G.jm * dk);
      __syncthreads();  // crd written / previous offset's fragments loaded
      for (int e = tid; e < CIN * LP_TM; e += blockDim.x) {
        const int c = e / LP_TM, r = e - c * LP_TM;
        const int* cr = crd + 4 * r;
        const int ii = cr[0] + di, jj = cr[1] + dj, kk = cr[2] + dk;
        const bool ok = cr[3] && ii >= 0 && ii < G.im && jj >= 0 && jj < G.jm && kk >= 0 && kk < G.km;
        As[c * LP_LDA + r] = ok ? in[(long)c * N + l0 + r + off] : __float2bfloat16(0.0f);
      }
      __syncthreads();
#pragma unroll
      for (int kc = 0; kc < KC; ++kc) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> a;
        wmma::load_matrix_sync(a, As + kc * 16 * LP_LDA + warp * 16, LP_LDA);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> b;
          wmma::load_matrix_sync(b, Ws + (o * CIN + kc * 16) * COUT_PAD + f * 16, COUT_PAD);
          wmma::mma_sync(acc[f], a, b, acc[f]);
        }
      }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f)
      wmma::store_matrix_sync(Cs + warp * 16 * (COUT_PAD + 4) + f * 16, acc[f], COUT_PAD + 4, wmma::mem_row_major);
    __syncthreads();
    for (int e = tid; e < cout_store * LP_TM; e += blockDim.x) {
      const int co = e / LP_TM, r = e - co * LP_TM;
      const long l = l0 + r;
      if (l >= N) continue;
      float v = Cs[r * (COUT_PAD + 4) + co] + (bias ? bias[co] : 0.0f);
      if (relu) v = fmaxf(v, 0.0f);
      if (mask && !(__bfloat162float(mask[(long)co * N + l]) > 0.0f)) v = 0.0f;
      if (out) out[(long)co * N + l] = __float2bfloat16(v);
      if (out32) out32[(long)co * N + l] = v;
    }
  }
}

// dW[o][ci][co] += sum_l X[ci][l + off(o)] dY[co][l] over this CTA's range of
// nodes (nodes_per_cta, a multiple of LP_TM), FP32 atomics into dW.  Warp w
// owns output fragment w (CIN/16 x COUT_PAD/16 fragments of 16 x 16).
template <int CIN, int COUT_PAD>
__global__ void __launch_bounds__(128) k_lp_wgrad(LpGrid G, const bf16* __restrict__ X, const bf16* __restrict__ dY,
                                                  float* __restrict__ dW, long nodes_per_cta) {
  pdl_wait();
  using namespace nvcuda;
  constexpr int MF = CIN / 16, NF = COUT_PAD / 16, F = MF * NF;
  static_assert(F <= 4, "one output fragment per warp");
  __shared__ __align__(128) bf16 Xs[CIN * LP_LDA];
  __shared__ __align__(128) bf16 Ds[COUT_PAD * LP_LDA];
  __shared__ __align__(128) float Cw[4][16 * 20];
  __shared__ int crd[LP_TM * 4];
  const int tid = threadIdx.x, warp = tid >> 5;
  const long N = G.N;
  const long n0 = blockIdx.x * nodes_per_cta;
  const long n1 = min(N, n0 + nodes_per_cta);
  const int mi = warp / NF, ni = warp % NF;
  for (int o = 0; o < 27; ++o) {
    int di, dj, dk;
    lp_offset(o, di, dj, dk);
    const long off = di + (long)G.im * (dj + (long)G.jm * dk);
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.0f);
    for (long l0 = n0; l0 < n1; l0 += LP_TM) {
      __syncthreads();  // previous chunk's fragments loaded
      if (tid < LP_TM) {
        const long l = l0 + tid;
        const int i = int(l % G.im);
        const long r = l / G.im;
        crd[4 * tid + 0] = i;
        crd[4 * tid + 1] = int(r % G.jm);
        crd[4 * tid + 2] = int(r / G.jm);
        crd[4 * tid + 3] = l < n1;
      }
      __syncthreads();
      for (int e = tid; e < CIN * LP_TM; e += blockDim.x) {
        const int c = e / LP_TM, r = e - c * LP_TM;
        const int* cr = crd + 4 * r;
        const int ii = cr[0] + di, jj = cr[1] + dj, kk = cr[2] + dk;
        const bool ok = cr[3] && ii >= 0 && ii < G.im && jj >= 0 && jj < G.jm && kk >= 0 && kk < G.km;
        Xs[c * LP_LDA + r] = ok ? X[(long)c * N + l0 + r + off] : __float2bfloat16(0.0f);
      }
      for (int e = tid; e < COUT_PAD * LP_TM; e += blockDim.x) {
        const int c = e / LP_TM, r = e - c * LP_TM;
        Ds[c * LP_LDA + r] = crd[4 * r + 3] ? dY[(long)c * N + l0 + r] : __float2bfloat16(0.0f);
      }
      __syncthreads();
      if (warp < F) {
#pragma unroll
        for (int ks = 0; ks < LP_TM / 16; ++ks) {
          wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::row_major> a;   // (ci, node)
          wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::col_major> b;   // (node, co)
          wmma::load_matrix_sync(a, Xs + mi * 16 * LP_LDA + ks * 16, LP_LDA);
          wmma::load_matrix_sync(b, Ds + ni * 16 * LP_LDA + ks * 16, LP_LDA);
          wmma::mma_sync(acc, a, b, acc);
        }
      }
    }
    if (warp < F) {
      wmma::store_matrix_sync(Cw[warp], acc, 20, wmma::mem_row_major);
      __syncwarp();
      const int lane = tid & 31;
      for (int e = lane; e < 256; e += 32) {
        const int r = e / 16, c = e % 16;
        atomicAdd(dW + ((long)o * CIN + mi * 16 + r) * COUT_PAD + ni * 16 + c, Cw[warp][r * 20 + c]);
      }
    }
  }
}

// db[co] += sum_l dY[co][l] (FP32 atomics; blockIdx.y = co)
__global__ void k_lp_bias_grad(long N, const bf16* __restrict__ dY, float* __restrict__ db) {
  pdl_wait();
  __shared__ float sh[256];
  const int co = blockIdx.y;
  float s = 0.0f;
  for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long)gridDim.x * blockDim.x)
    s += __bfloat162float(dY[(long)co * N + l]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(db + co, sh[0]);
}

// Input features from the time levels, in[16][N] BF16 (channel 15 zero):
// channel 3f + {0, 1, 2} = q^n_f, (q^n - q^{n-1})_f, (q^{n-1} - q^{n-2})_f,
// each times rs[channel] (the reciprocal of its RMS).
__global__ void k_lp_features(long N, const double* const* qn, const double* const* qnm1, const double* const* qnm2,
                              const float* __restrict__ rs, bf16* __restrict__ in) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= N) return;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const double a = qn[f][l], b = qnm1[f][l], c = qnm2[f][l];
    in[(long)(3 * f + 0) * N + l] = __float2bfloat16(float(a) * rs[3 * f + 0]);
    in[(long)(3 * f + 1) * N + l] = __float2bfloat16(float(a - b) * rs[3 * f + 1]);
    in[(long)(3 * f + 2) * N + l] = __float2bfloat16(float(b - c) * rs[3 * f + 2]);
  }
  in[15 * N + l] = __float2bfloat16(0.0f);
}

// Sums of squares of the 15 feature channels (before scaling) and of the
// target's second difference, for the RMS scales: acc[16] doubles.
__global__ void k_lp_sumsq(long N, const double* const* qn, const double* const* qnm1, const double* const* qnm2,
                           double* acc) {
  pdl_wait();
  __shared__ double sh[15][128];
  double s[15];
#pragma unroll
  for (int c = 0; c < 15; ++c) s[c] = 0.0;
  for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const double a = qn[f][l], b = qnm1[f][l], c = qnm2[f][l];
      s[3 * f + 0] += a * a;
      s[3 * f + 1] += (a - b) * (a - b);
      s[3 * f + 2] += (b - c) * (b - c);
    }
  }
#pragma unroll
  for (int c = 0; c < 15; ++c) sh[c][threadIdx.x] = s[c];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < 15; ++c) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < 15) atomicAdd(acc + threadIdx.x, sh[threadIdx.x][0]);
}

// Scales from the sums of squares acc[0..14] (one thread block of 32):
// rs[c] = 1 / RMS of channel c (0 for a still or zero channel, and rs[15] = 0),
// rs5[f] = rs[3 f + 1], s5[f] = the RMS of (q^n - q^{n-1})_f or 0.
__global__ void k_lp_scales(long N, const double* __restrict__ acc, float* __restrict__ rs, float* __restrict__ rs5,
                            float* __restrict__ s5) {
  pdl_wait();
  const int c = threadIdx.x;
  if (c >= 16) return;
  float r = 0.0f;
  if (c < 15) {
    const int f = c / 3;
    const double rms = sqrt(acc[c] / double(N));
    const double rq = sqrt(acc[3 * f] / double(N));
    const double floor = c % 3 == 0 ? 1e-30 : fmax(1e-12 * rq, 1e-30);
    r = rms > floor ? float(1.0 / rms) : 0.0f;
    if (c % 3 == 1) {
      rs5[f] = r;
      s5[f] = r > 0.0f ? float(rms) : 0.0f;
    }
  }
  rs[c] = r;
}

// Training target t[f][l] = (q^{n+1} - 2 q^n + q^{n-1})_f / s_f (FP32), with
// q^{n+1} = q, q^n = qn, q^{n-1} = qnm1 and rs5[f] = 1 / s_f.
__global__ void k_lp_target(long N, const double* const* q, const double* const* qn, const double* const* qnm1,
                            const float* __restrict__ rs5, float* __restrict__ t) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= N) return;
#pragma unroll
  for (int f = 0; f < 5; ++f)
    t[(long)f * N + l] = float(q[f][l] - 2.0 * qn[f][l] + qnm1[f][l]) * rs5[f];
}

// Squared error of the network output y against t over the 5 output
// channels: loss partial sums (acc[0], double) and dY = y - t in BF16
// (channels 5..15 of dY stay zero); the factor 2 / (5 N) of the mean goes
// into the gradient scale.
__global__ void k_lp_loss(long N, const float* __restrict__ y, const float* __restrict__ t, bf16* __restrict__ dY,
                          double* acc) {
  pdl_wait();
  __shared__ double sh[256];
  double s = 0.0;
  for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const float d = y[(long)f * N + l] - t[(long)f * N + l];
      s += double(d) * double(d);
      dY[(long)f * N + l] = __float2bfloat16(d);
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(acc, sh[0]);
}

// The guess q = 2 q^n - q^{n-1} + s_f min(max(y_f, -ymax), ymax); a node
// whose network output is not finite keeps the linear extrapolation.
__global__ void k_lp_apply(long N, double* const* q, const double* const* qn, const double* const* qnm1,
                           const float* __restrict__ s5, const float* __restrict__ y, float ymax) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= N) return;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const float c = y[(long)f * N + l];
    const double corr = isfinite(c) ? double(s5[f]) * double(fminf(fmaxf(c, -ymax), ymax)) : 0.0;
    q[f][l] = 2.0 * qn[f][l] - qnm1[f][l] + corr;
  }
}

// FP32 <-> BF16 copies (host-given features, buffer reads)
__global__ void k_lp_f2bf(long n, const float* __restrict__ a, bf16* __restrict__ b) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) b[e] = __float2bfloat16(a[e]);
}

__global__ void k_lp_bf2f(long n, const bf16* __restrict__ a, float* __restrict__ b) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) b[e] = __bfloat162float(a[e]);
}

// One layer's shape in the flat parameter vector: W[co][ci][o] (real
// channels), then b[co].
struct LpLayer {
  int cin, cout;        // real channels
  int cin_pad, cout_pad;
  long woff, boff;      // offsets of W and b in the flat vector
};

// Forward and data-gradient weight blocks from the master weights:
// wf[o][ci][co] = W[co][ci][o], wd[o][co][ci] = W[co][ci][26 - o] (zero in
// the padded channels).
__global__ void k_lp_pack(LpLayer ly, const float* __restrict__ theta, bf16* __restrict__ wf, bf16* __restrict__ wd) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = 27L * ly.cin_pad * ly.cout_pad;
  if (e >= total) return;
  // e indexes wf[o][ci][co]
  const int co = int(e % ly.cout_pad);
  const int ci = int((e / ly.cout_pad) % ly.cin_pad);
  const int o = int(e / ((long)ly.cout_pad * ly.cin_pad));
  float w = 0.0f;
  if (ci < ly.cin && co < ly.cout) w = theta[ly.woff + ((long)co * ly.cin + ci) * 27 + o];
  wf[e] = __float2bfloat16(w);
  // wd[26 - o][co][ci] takes the same weight
  wd[((long)(26 - o) * ly.cout_pad + co) * ly.cin_pad + ci] = __float2bfloat16(w);
}

// Gradient of the flat parameter vector from dW[o][ci][co] and db[co] of one
// layer, times gscale.
__global__ void k_lp_gather_grad(LpLayer ly, const float* __restrict__ dW, const float* __restrict__ db, float gscale,
                                 float* __restrict__ grad) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nw = (long)ly.cout * ly.cin * 27;
  if (e < nw) {
    const int o = int(e % 27);
    const int ci = int((e / 27) % ly.cin);
    const int co = int(e / (27L * ly.cin));
    grad[ly.woff + e] = gscale * dW[((long)o * ly.cin_pad + ci) * ly.cout_pad + co];
  } else if (e < nw + ly.cout) {
    grad[ly.boff + (e - nw)] = gscale * db[e - nw];
  }
}

// Adam (Kingma and Ba, 2015) on the flat parameter vector.
__global__ void k_lp_adam(long n, float* __restrict__ theta, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gi = g[e];
  const float mi = b1 * m[e] + (1.0f - b1) * gi;
  const float vi = b2 * v[e] + (1.0f - b2) * gi * gi;
  m[e] = mi;
  v[e] = vi;
  theta[e] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

}  // namespace desalm
