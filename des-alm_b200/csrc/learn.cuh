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
// Layout: activations and their gradients are BF16, channel-last rows of a
// zero-padded grid ((im+2) x (jm+2) x (km+2) rows, i fastest; 16 or 32
// channels, 32 or 64 bytes a row).  The halo rows stay zero, so the 27
// neighbours of an interior row are the rows at fixed offsets with no bounds
// checks, and the shifted operand of a stencil offset is a contiguous run of
// rows.  The convolution (forward, and the data gradient with the weights
// transposed and the stencil flipped) and the weight gradient are the tcgen05
// kernels of learn_tc.cuh, BF16 products accumulated in FP32 in tensor
// memory; this file holds the layout, the element-wise kernels (features,
// scales, targets, loss, guess), the per-CTA partial reduction, the gradient
// gather and Adam.  Master weights, Adam moments and the loss are FP32 / FP64.
#pragma once
#include <cuda_bf16.h>
#include "common.cuh"

namespace desalm {

using bf16 = __nv_bfloat16;

constexpr int LP_TM = 128;           // rows per tile
constexpr float LP_YMAX = 8.0f;      // default limit of |output| (in units of s) in the guess
constexpr int LP_WROWS = LP_TM + 2;  // rows of a window (di = -1..1)

// The zero-padded grid of the fine level.
struct LpPad {
  int im, jm, km;    // interior extents (the level's nodes)
  int ip, jp, kp;    // padded extents
  long np;           // padded rows
  long p0, p1;       // first interior row and one past the last
  long N;            // interior nodes
};

inline LpPad lp_pad(int im, int jm, int km) {
  LpPad P;
  P.im = im; P.jm = jm; P.km = km;
  P.ip = im + 2; P.jp = jm + 2; P.kp = km + 2;
  P.np = (long)P.ip * P.jp * P.kp;
  P.p0 = 1 + (long)P.ip * (1 + (long)P.jp);
  P.p1 = (long)im + (long)P.ip * (jm + (long)P.jp * km) + 1;
  P.N = (long)im * jm * km;
  return P;
}

// padded row of interior node l (level order, i fastest)
DESALM_DEV long lp_row(const LpPad& P, long l) {
  const long i = l % P.im, r = l / P.im;
  const long j = r % P.jm, k = r / P.jm;
  return (i + 1) + (long)P.ip * ((j + 1) + (long)P.jp * (k + 1));
}

// interior node of padded row p, or -1 for a halo row
DESALM_DEV long lp_node(const LpPad& P, long p) {
  const long ii = p % P.ip, r = p / P.ip;
  const long jj = r % P.jp, kk = r / P.jp;
  if (ii < 1 || ii > P.im || jj < 1 || jj > P.jm || kk < 1 || kk > P.km) return -1;
  return (ii - 1) + (long)P.im * ((jj - 1) + (long)P.jm * (kk - 1));
}

// out[e] = sum over nslot slots of part[slot * len + e]
__global__ void k_lp_reduce(int nslot, long len, const float* __restrict__ part, float* __restrict__ out) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= len) return;
  float s = 0.0f;
  for (int k = 0; k < nslot; ++k) s += part[(long)k * len + e];
  out[e] = s;
}

// Input features from the time levels into the channel-last padded rows
// in[p][16] (BF16; channel 15 zero): channel 3f + {0, 1, 2} = q^n_f,
// (q^n - q^{n-1})_f, (q^{n-1} - q^{n-2})_f, each times rs[channel].
__global__ void k_lp_features(LpPad P, const double* const* qn, const double* const* qnm1, const double* const* qnm2,
                              const float* __restrict__ rs, bf16* __restrict__ in) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= P.N) return;
  uint4 v[2];
  bf16* x = reinterpret_cast<bf16*>(v);
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const double a = qn[f][l], b = qnm1[f][l], c = qnm2[f][l];
    x[3 * f + 0] = __float2bfloat16(float(a) * rs[3 * f + 0]);
    x[3 * f + 1] = __float2bfloat16(float(a - b) * rs[3 * f + 1]);
    x[3 * f + 2] = __float2bfloat16(float(b - c) * rs[3 * f + 2]);
  }
  x[15] = __float2bfloat16(0.0f);
  uint4* dst = reinterpret_cast<uint4*>(in + lp_row(P, l) * 16);
  dst[0] = v[0];
  dst[1] = v[1];
}

// [C][N] FP32 (node order) <-> channel-last padded rows [p][C] BF16
__global__ void k_lp_rows_in(LpPad P, int C, int c0, int nc, const float* __restrict__ a, bf16* __restrict__ rows) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= P.N) return;
  const long p = lp_row(P, l);
  for (int c = 0; c < nc; ++c) rows[p * C + c0 + c] = __float2bfloat16(a[(long)c * P.N + l]);
}

__global__ void k_lp_rows_out(LpPad P, int C, int c0, int nc, const bf16* __restrict__ rows, float* __restrict__ a) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= P.N) return;
  const long p = lp_row(P, l);
  for (int c = 0; c < nc; ++c) a[(long)c * P.N + l] = __bfloat162float(rows[p * C + c0 + c]);
}

// The reductions below leave one row of 16 partial sums per CTA in part
// (part[16 b + c]); k_lp_fold then adds the rows in CTA order, so that every
// sum is the same from run to run.
__global__ void k_lp_fold(const double* __restrict__ part, int nblk, int nc, double* __restrict__ acc) {
  pdl_wait();
  const int c = threadIdx.x;
  if (c >= nc) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[16 * b + c];
  acc[c] = s;
}

// Sums of squares of the 15 feature channels (before scaling): the partial
// sums of the RMS scales (k_lp_fold gives acc[0..14]).
__global__ void k_lp_sumsq(long N, const double* const* qn, const double* const* qnm1, const double* const* qnm2,
                           double* part) {
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
  if (threadIdx.x < 15) part[16 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
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
// channels: loss partial sums (part, column 0) and dY = y - t in BF16 into
// the channel-last padded rows dY[p][16] (channels 5..15 stay zero); the
// factor 2 / (5 N) of the mean goes into the gradient scale.
__global__ void k_lp_loss(LpPad P, const float* __restrict__ y, const float* __restrict__ t, bf16* __restrict__ dY,
                          double* part) {
  pdl_wait();
  __shared__ double sh[256];
  double s = 0.0;
  const long N = P.N;
  for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long)gridDim.x * blockDim.x) {
    bf16* row = dY + lp_row(P, l) * 16;
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const float d = y[(long)f * N + l] - t[(long)f * N + l];
      s += double(d) * double(d);
      row[f] = __float2bfloat16(d);
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[16 * blockIdx.x] = sh[0];
}

// Held-out check of the network on a new sample, before it trains on it:
// partial sums of, per field f, y_f t_f (column f), y_f^2 (5 + f) and t_f^2
// (10 + f), y clipped to [-ymax, ymax] as in the guess.
__global__ void k_lp_dot(long N, const float* __restrict__ y, const float* __restrict__ t, float ymax, double* part) {
  pdl_wait();
  __shared__ double sh[15][128];
  double s[15];
#pragma unroll
  for (int c = 0; c < 15; ++c) s[c] = 0.0;
  for (long l = (long)blockIdx.x * blockDim.x + threadIdx.x; l < N; l += (long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      const float yv = y[(long)f * N + l];
      const double a = isfinite(yv) ? double(fminf(fmaxf(yv, -ymax), ymax)) : 0.0;
      const double b = t[(long)f * N + l];
      s[f] += a * b;
      s[5 + f] += a * a;
      s[10 + f] += b * b;
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
  if (threadIdx.x < 15) part[16 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// Blend of each field's correction: automatic (fixed < 0): the least-squares
// factor alpha_f = <y, t> / <y, y> of the held-out check, limited to [0, 1]
// (0 when the network's output is zero or not finite), so that a network that
// does not help leaves the linear extrapolation; otherwise alpha_f = fixed.
__global__ void k_lp_blend(const double* __restrict__ acc, float fixed, int mask, float* __restrict__ alpha) {
  pdl_wait();
  const int f = threadIdx.x;
  if (f >= 5) return;
  if (!((mask >> f) & 1)) {
    alpha[f] = 0.0f;
    return;
  }
  float a = fixed;
  if (fixed < 0.0f) {
    const double yt = acc[f], yy = acc[5 + f];
    const double r = yy > 0.0 ? yt / yy : 0.0;
    a = isfinite(r) ? float(fmin(fmax(r, 0.0), 1.0)) : 0.0f;
  }
  alpha[f] = a;
}

// The guess q = 2 q^n - q^{n-1} + s_f alpha_f min(max(y_f, -ymax), ymax); a
// node whose network output is not finite keeps the linear extrapolation.
__global__ void k_lp_apply(long N, double* const* q, const double* const* qn, const double* const* qnm1,
                           const float* __restrict__ s5, const float* __restrict__ alpha, const float* __restrict__ y,
                           float ymax) {
  pdl_wait();
  const long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= N) return;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    const float c = y[(long)f * N + l];
    const double corr = isfinite(c) ? double(s5[f] * alpha[f]) * double(fminf(fmaxf(c, -ymax), ymax)) : 0.0;
    q[f][l] = 2.0 * qn[f][l] - qnm1[f][l] + corr;
  }
}

// One layer's shape in the flat parameter vector: W[co][ci][o] (real
// channels), then b[co].
struct LpLayer {
  int cin, cout;        // real channels
  int cin_pad, cout_pad;
  long woff, boff;      // offsets of W and b in the flat vector
};

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
