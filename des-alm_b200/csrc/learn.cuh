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
// rows.  Products accumulate in FP32 on the tensor cores.  The convolution
// (forward, and the data gradient with the weights transposed and the stencil
// flipped) is the tcgen05 kernel of learn_tc.cuh.  The weight gradient here
// is an implicit GEMM on WMMA m16n16k16 BF16 that reduces over the rows: for
// each of the 9 (dj, dk) pairs the CTA copies a window of LP_TM + 2 rows into
// shared memory (16-byte cp.async, double-buffered) and multiplies the window
// shifted by di = -1, 0, 1 rows with the output gradient, with per-CTA
// partial sums and one reduction kernel.  Master weights, Adam moments and
// the loss are FP32 / FP64.
#pragma once
#include <mma.h>
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

DESALM_DEV void lp_cp16(void* smem, const void* gmem, bool ok) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
  const int n = ok ? 16 : 0;  // 0: fill the 16 bytes with zeros
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(gmem), "r"(n) : "memory");
}
DESALM_DEV void lp_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
DESALM_DEV void lp_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Row stride (elements) of a channel-last tile in shared memory: a multiple
// of 32 bytes, so that a window shifted by one row is still a legal WMMA
// operand address.
template <int C>
struct LpStride {
  static constexpr int v = C == 16 ? 16 : 48;
};

// Copy the window of (dj, dk) pair g for the tile starting at padded row
// t0: rows t0 + off(0, dj, dk) - 1 .. + LP_WROWS; rows outside the padded
// grid (only past the end of the last tile) read as zero.
template <int C>
DESALM_DEV void lp_load_window(const LpPad& P, const bf16* __restrict__ src, long t0, int g, bf16* dst, int tid,
                               int nthreads) {
  constexpr int S = LpStride<C>::v, CH = C / 8;
  const int dj = g % 3 - 1, dk = g / 3 - 1;
  const long base = t0 + (long)P.ip * (dj + (long)P.jp * dk) - 1;
  for (int e = tid; e < LP_WROWS * CH; e += nthreads) {
    const int r = e / CH, c = e - r * CH;
    const long row = base + r;
    const bool ok = row >= 0 && row < P.np;
    lp_cp16(dst + r * S + 8 * c, src + (ok ? row : 0) * C + 8 * c, ok);
  }
}

// Shared-memory layout of k_lp_wgrad (bytes): two windows of X, two tiles of D.
template <int CIN, int COUT>
struct LpWgradSmem {
  static constexpr int SA = LpStride<CIN>::v, SD = LpStride<COUT>::v;
  static constexpr size_t win = size_t(LP_WROWS) * SA * sizeof(bf16);
  static constexpr size_t d = size_t(LP_TM) * SD * sizeof(bf16);
  static constexpr size_t total = 2 * win + 2 * d;
};

// Partial weight and bias gradients of one layer over a contiguous range of
// tiles per CTA:
//   part[cta][o][ci][co] = sum_p X[p + off(o)][ci] D[p][co],
//   part[cta][27 CIN COUT + co] = sum_p D[p][co],
// p over the tiles' rows (D is zero on halo rows and past the last interior
// row).  3 * (CIN/16) * (COUT/16) warps; warp w owns the output fragment
// (di, ci block, co block) of every (dj, dk) pair, so each window feeds every
// warp once.
template <int CIN, int COUT>
__global__ void __launch_bounds__(32 * 3 * (CIN / 16) * (COUT / 16))
    k_lp_wgrad(LpPad P, const bf16* __restrict__ X, const bf16* __restrict__ D, float* __restrict__ part) {
  pdl_wait();
  using namespace nvcuda;
  using SM = LpWgradSmem<CIN, COUT>;
  constexpr int MF = CIN / 16, NF = COUT / 16, NW = 3 * MF * NF, NT = 32 * NW;
  constexpr int SA = SM::SA, SD = SM::SD;
  constexpr int WIN = int(SM::win / sizeof(bf16)), DT = int(SM::d / sizeof(bf16));
  constexpr long SLOT = 27L * CIN * COUT + COUT;
  extern __shared__ __align__(128) unsigned char lp_smem[];
  bf16* Win = reinterpret_cast<bf16*>(lp_smem);
  bf16* Dt = reinterpret_cast<bf16*>(lp_smem + 2 * SM::win);
  __shared__ float bsum[NT];
  const int tid = threadIdx.x, warp = tid >> 5;
  const int di = warp % 3, mi = (warp / 3) % MF, ni = warp / (3 * MF);
  const long ntiles = (P.p1 - P.p0 + LP_TM - 1) / LP_TM;
  const long per = (ntiles + gridDim.x - 1) / gridDim.x;
  const long ta = blockIdx.x * per, tb = min(ntiles, ta + per);
  auto load_d = [&](long tile, int b) {
    const long t0 = P.p0 + tile * LP_TM;
    for (int e = tid; e < LP_TM * (COUT / 8); e += NT) {
      const int r = e / (COUT / 8), c = e - r * (COUT / 8);
      const long row = t0 + r;
      const bool ok = row < P.p1;
      lp_cp16(Dt + b * DT + r * SD + 8 * c, D + (ok ? row : 0) * COUT + 8 * c, ok);
    }
  };
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[9];
#pragma unroll
  for (int g = 0; g < 9; ++g) wmma::fill_fragment(acc[g], 0.0f);
  float bs = 0.0f;  // bias partial of channel tid % COUT
  int buf = 0;
  if (ta < tb) {
    lp_load_window<CIN>(P, X, P.p0 + ta * LP_TM, 0, Win, tid, NT);
    load_d(ta, 0);
  }
  lp_cp_commit();
  for (long tile = ta; tile < tb; ++tile) {
    const int db = int((tile - ta) & 1);
#pragma unroll
    for (int g = 0; g < 9; ++g) {
      if (g < 8) {
        lp_load_window<CIN>(P, X, P.p0 + tile * LP_TM, g + 1, Win + (buf ^ 1) * WIN, tid, NT);
      } else if (tile + 1 < tb) {
        lp_load_window<CIN>(P, X, P.p0 + (tile + 1) * LP_TM, 0, Win + (buf ^ 1) * WIN, tid, NT);
        load_d(tile + 1, db ^ 1);
      }
      lp_cp_commit();
      lp_cp_wait<1>();
      __syncthreads();
      const bf16* A0 = Win + buf * WIN + di * SA + mi * 16;
      const bf16* B0 = Dt + db * DT + ni * 16;
#pragma unroll
      for (int ks = 0; ks < LP_TM / 16; ++ks) {
        wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, wmma::col_major> a;  // (ci, row)
        wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, wmma::row_major> b;  // (row, co)
        wmma::load_matrix_sync(a, A0 + ks * 16 * SA, SA);
        wmma::load_matrix_sync(b, B0 + ks * 16 * SD, SD);
        wmma::mma_sync(acc[g], a, b, acc[g]);
      }
      if (g == 0) {
        // bias partial: thread tid sums rows tid / COUT, + NT / COUT, ... of channel tid % COUT
        const bf16* Db = Dt + db * DT;
        for (int r = tid / COUT; r < LP_TM; r += NT / COUT) bs += __bfloat162float(Db[r * SD + tid % COUT]);
      }
      __syncthreads();  // the window (and, after the last pair, the D tile) is read before it is refilled
      buf ^= 1;
    }
  }
  lp_cp_wait<0>();
  float* slot = part + blockIdx.x * SLOT;
#pragma unroll
  for (int g = 0; g < 9; ++g) {
    const int o = 3 * g + di;
    wmma::store_matrix_sync(slot + ((long)o * CIN + mi * 16) * COUT + ni * 16, acc[g], COUT, wmma::mem_row_major);
  }
  bsum[tid] = bs;
  __syncthreads();
  if (tid < COUT) {
    float t = 0.0f;
    for (int r = tid; r < NT; r += COUT) t += bsum[r];
    slot[27L * CIN * COUT + tid] = t;
  }
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
// channels: loss partial sums (acc[0], double) and dY = y - t in BF16 into
// the channel-last padded rows dY[p][16] (channels 5..15 stay zero); the
// factor 2 / (5 N) of the mean goes into the gradient scale.
__global__ void k_lp_loss(LpPad P, const float* __restrict__ y, const float* __restrict__ t, bf16* __restrict__ dY,
                          double* acc) {
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
  if (threadIdx.x == 0) atomicAdd(acc, sh[0]);
}

// Held-out check of the network on a new sample, before it trains on it:
// per field f, acc[f] += sum y_f t_f, acc[5 + f] += sum y_f^2,
// acc[10 + f] += sum t_f^2 (y clipped to [-ymax, ymax] as in the guess).
__global__ void k_lp_dot(long N, const float* __restrict__ y, const float* __restrict__ t, float ymax, double* acc) {
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
  if (threadIdx.x < 15) atomicAdd(acc + threadIdx.x, sh[threadIdx.x][0]);
}

// Blend of each field's correction: automatic (fixed < 0): the least-squares
// factor alpha_f = <y, t> / <y, y> of the held-out check, limited to [0, 1]
// (0 when the network's output is zero or not finite), so that a network that
// does not help leaves the linear extrapolation; otherwise alpha_f = fixed.
__global__ void k_lp_blend(const double* __restrict__ acc, float fixed, float* __restrict__ alpha) {
  pdl_wait();
  const int f = threadIdx.x;
  if (f >= 5) return;
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
