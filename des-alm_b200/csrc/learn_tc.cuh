// learn_tc.cuh -- the learned guess's convolution on the 5th-generation
// tensor cores: tcgen05.mma with the accumulator in tensor memory, operands
// staged in shared memory by TMA.
//
// out[p][co] = act(bias[co] + sum_{ci, o} W[o][ci][co] in[p + off(o)][ci]) over
// tiles of 128 consecutive padded rows (the layout of learn.cuh).  For each of
// the 9 (dj, dk) pairs one TMA box per 8-channel chunk copies the window of
// 130 rows, t0 + off(0, dj, dk) - 1 .., into a shared-memory slab whose rows
// are 16 bytes apart.  That slab is the K-major, no-swizzle UMMA layout
// (8-row core matrices 128 bytes apart, channel chunks one slab apart), in
// which row r sits at start + 16 r: the operand for di = -1, 0, 1 is the same
// slab with its descriptor's start address moved by 0, 16 or 32 bytes.  One
// tcgen05.mma (M = 128 rows, N = COUT, K = 16 channels) per (di, 16-channel
// step) accumulates into tensor memory; 27 CIN / 16 of them make a tile.
//
// Roles: warp 0 (one lane) issues the TMA copies and the MMAs; warps 1-4 read
// the accumulator (tcgen05.ld, one TMEM lane per row) and run the epilogue.
// Windows cycle through LP_TC_STAGES stages ("full" mbarriers completed by TMA
// bytes, "empty" ones by tcgen05.commit); the accumulator is double-buffered
// in tensor memory, so one tile's epilogue overlaps the next tile's MMAs.
// Every mbarrier wait gives up after about two seconds: it sets *err, and the
// kernel finishes without further copies or MMAs and frees its tensor memory.
#pragma once
#include <cuda.h>
#include "learn.cuh"

namespace desalm {

constexpr int LP_TC_STAGES = 4;             // window stages
constexpr int LP_TC_SLAB = 2176;            // bytes between channel-chunk slabs (130 rows x 16 B, padded to 128 B)
constexpr int LP_TC_THREADS = 160;          // warp 0: TMA + MMA; warps 1-4: epilogue
constexpr unsigned long long LP_TC_WAIT_NS = 2000000000ull;

template <int CIN, int COUT>
struct LpTcSmem {
  static constexpr int KCH = CIN / 8;                                  // channel chunks of a row
  static constexpr size_t w = size_t(27) * CIN * COUT * sizeof(bf16);  // weights, UMMA B layout
  static constexpr size_t win = size_t(KCH) * LP_TC_SLAB;              // one window stage
  static constexpr size_t bars = 8 * (2 * LP_TC_STAGES + 6);           // full, empty, weights, accf x2, acce x2, drain
  static constexpr size_t total = w + LP_TC_STAGES * win + bars + 16;
  static_assert(w % 128 == 0 && win % 128 == 0, "TMA destinations stay 128-byte aligned");
};

// Weights of one layer in the UMMA B layout (K-major, no swizzle): for offset
// o and channel chunk c = ci / 8, a slab of COUT rows of 8 input channels,
// element ((o * CIN/8 + c) * COUT + co) * 8 + ci % 8.  Written by k_lp_pack_tc
// from the flat parameters: forward blocks W[o][ci][co] = W(co, ci, o), data-
// gradient blocks Wd[o][co][ci] = W(co, ci, 26 - o) (CIN and COUT swapped).
__global__ void k_lp_pack_tc(LpLayer ly, const float* __restrict__ theta, bf16* __restrict__ wf, bf16* __restrict__ wd) {
  pdl_wait();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = 27L * ly.cin_pad * ly.cout_pad;
  if (e >= total) return;
  // e enumerates (o, ci, co) of the forward block
  const int co = int(e % ly.cout_pad);
  const int ci = int((e / ly.cout_pad) % ly.cin_pad);
  const int o = int(e / ((long)ly.cout_pad * ly.cin_pad));
  float w = 0.0f;
  if (ci < ly.cin && co < ly.cout) w = theta[ly.woff + ((long)co * ly.cin + ci) * 27 + o];
  const bf16 b = __float2bfloat16(w);
  // forward: K = ci (CIN = cin_pad), N = co (COUT = cout_pad)
  wf[(((long)o * (ly.cin_pad / 8) + ci / 8) * ly.cout_pad + co) * 8 + ci % 8] = b;
  // data gradient at offset 26 - o: K = co (CIN = cout_pad), N = ci (COUT = cin_pad)
  const int od = 26 - o;
  wd[(((long)od * (ly.cout_pad / 8) + co / 8) * ly.cin_pad + ci) * 8 + co % 8] = b;
}

DESALM_DEV unsigned lp_smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

DESALM_DEV unsigned long long lp_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

DESALM_DEV void lp_bar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

DESALM_DEV void lp_bar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

DESALM_DEV void lp_bar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Wait for the phase of parity `parity` to complete; false after `limit_ns`
// (or, unless draining, when another thread already gave up), with *err set.
DESALM_DEV bool lp_bar_wait(unsigned bar, unsigned parity, int* err, bool drain = false,
                            unsigned long long limit_ns = LP_TC_WAIT_NS) {
  const unsigned long long t0 = lp_ns();
  for (unsigned n = 0;; ++n) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    if ((n & 255u) == 255u) {
      if (!drain && *(volatile int*)err) return false;
      if (lp_ns() - t0 > limit_ns) {
        atomicExch(err, 1);
        return false;
      }
    }
  }
}

DESALM_DEV void lp_tma_2d(unsigned dst, const CUtensorMap* map, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cta.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

DESALM_DEV void lp_bulk_copy(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// K-major, no-swizzle UMMA shared-memory descriptor: core matrices of 8 rows x
// 16 bytes, rows 16 bytes apart, 8-row groups sbo bytes apart, 16-byte K
// chunks lbo bytes apart.
DESALM_DEV unsigned long long lp_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3FFFu) | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
DESALM_HD constexpr unsigned lp_idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (unsigned(n >> 3) << 17) | (unsigned(128 >> 4) << 24);
}

DESALM_DEV void lp_mma(unsigned tmem, unsigned long long a, unsigned long long b, unsigned idesc, unsigned acc) {
  asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "setp.ne.b32 P, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, P;\n\t}" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

DESALM_DEV void lp_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

DESALM_DEV void lp_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
DESALM_DEV void lp_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 32 lanes x N columns of FP32 from tensor memory (N = 16 or 32)
template <int N>
DESALM_DEV void lp_tmem_ld(unsigned taddr, float* v);

template <>
DESALM_DEV void lp_tmem_ld<32>(unsigned taddr, float* v) {
  unsigned r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

template <>
DESALM_DEV void lp_tmem_ld<16>(unsigned taddr, float* v) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// The convolution (see the top of this file).  tmap: the input rows as a 2D
// BF16 tensor [np rows][CIN channels] with a box of 8 channels x 130 rows;
// wk: the weights in the UMMA B layout; the other arguments as k_lp_conv.
template <int CIN, int COUT>
__global__ void __launch_bounds__(LP_TC_THREADS) k_lp_conv_tc(const __grid_constant__ CUtensorMap tmap, LpPad P,
                                                           const bf16* __restrict__ wk, const float* __restrict__ bias,
                                                           int relu, const bf16* __restrict__ mask,
                                                           bf16* __restrict__ out, float* __restrict__ out32,
                                                           int cout32, int* err) {
  pdl_wait();
  using SM = LpTcSmem<CIN, COUT>;
  constexpr int KCH = SM::KCH, ST = LP_TC_STAGES;
  constexpr unsigned IDESC = lp_idesc(COUT);
  constexpr unsigned TMEM_COLS = 2 * COUT < 32 ? 32 : 2 * COUT;
  extern __shared__ __align__(128) unsigned char lp_tc_smem[];
  unsigned char* Wsm = lp_tc_smem;
  unsigned char* Win = lp_tc_smem + SM::w;
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(lp_tc_smem + SM::w + ST * SM::win);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(lp_tc_smem + SM::w + ST * SM::win + SM::bars);
  const unsigned full0 = lp_smem_u32(bars), empty0 = full0 + 8 * ST, wbar = empty0 + 8 * ST;
  const unsigned accf0 = wbar + 8, acce0 = accf0 + 16, dbar = acce0 + 16;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long ntiles = (P.p1 - P.p0 + LP_TM - 1) / LP_TM;
  const long my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long S = my_tiles * 9;  // (tile, pair) steps of this CTA

  if (tid == 0) {
    for (int s = 0; s < ST; ++s) {
      lp_bar_init(full0 + 8 * s, 1);
      lp_bar_init(empty0 + 8 * s, 1);
    }
    lp_bar_init(wbar, 1);
    lp_bar_init(accf0, 1);
    lp_bar_init(accf0 + 8, 1);
    lp_bar_init(acce0, 4);
    lp_bar_init(acce0 + 8, 4);
    lp_bar_init(dbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(lp_smem_u32(tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  lp_tc_fence_before();
  __syncthreads();
  lp_tc_fence_after();
  const unsigned tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0 && S > 0) {
      // ---- producer and MMA issuer
      auto issue_window = [&](long step) {
        const long tl = step / 9;
        const int g = int(step % 9);
        const int dj = g % 3 - 1, dk = g / 3 - 1;
        const long t0 = P.p0 + (blockIdx.x + tl * gridDim.x) * LP_TM;
        const int y = int(t0 + (long)P.ip * (dj + (long)P.jp * dk) - 1);
        const int s = int(step % ST);
        const unsigned dst = lp_smem_u32(Win + s * SM::win);
        lp_bar_expect_tx(full0 + 8 * s, KCH * LP_WROWS * 16);
        for (int c = 0; c < KCH; ++c) lp_tma_2d(dst + c * LP_TC_SLAB, &tmap, 8 * c, y, full0 + 8 * s);
      };
      lp_bar_expect_tx(wbar, unsigned(SM::w));
      lp_bulk_copy(lp_smem_u32(Wsm), wk, unsigned(SM::w), wbar);
      long issued = 0;  // windows whose copies were started
      for (; issued < ST && issued < S; ++issued) issue_window(issued);
      const bool wok = lp_bar_wait(wbar, 0, err);
      bool ok = wok;
      const unsigned wbase = lp_smem_u32(Wsm);
      long step = 0;
      for (; ok && step < S; ++step) {
        const int s = int(step % ST);
        const long tl = step / 9;
        const int g = int(step % 9);
        const int ab = int(tl & 1);
        if (!lp_bar_wait(full0 + 8 * s, unsigned((step / ST) & 1), err)) { ok = false; break; }
        if (g == 0 && tl >= 2 && !lp_bar_wait(acce0 + 8 * ab, unsigned(((tl >> 1) - 1) & 1), err)) {
          ok = false;
          break;
        }
        lp_tc_fence_after();
        const unsigned abase = lp_smem_u32(Win + s * SM::win);
#pragma unroll
        for (int di = 0; di < 3; ++di) {
          const int o = 3 * g + di;
#pragma unroll
          for (int kc = 0; kc < CIN / 16; ++kc) {
            const unsigned long long a = lp_desc(abase + 16 * di + 2 * kc * LP_TC_SLAB, LP_TC_SLAB, 128);
            const unsigned long long b =
                lp_desc(wbase + (o * KCH + 2 * kc) * COUT * 16, COUT * 16, 128);
            lp_mma(tmem + ab * COUT, a, b, IDESC, (g | di | kc) != 0);
          }
        }
        lp_commit(empty0 + 8 * s);
        if (g == 8) lp_commit(accf0 + 8 * ab);
        // refill the stage of the previous step once its MMAs are done
        if (step >= 1 && step - 1 + ST < S) {
          const long ps = step - 1;
          const int pst = int(ps % ST);
          if (!lp_bar_wait(empty0 + 8 * pst, unsigned((ps / ST) & 1), err)) {
            ++step;
            ok = false;
            break;
          }
          issue_window(ps + ST);
          ++issued;
        }
      }
      if (!ok) {
        // drain: every MMA issued so far, the weight copy, and the windows
        // started but not consumed, each with a bounded wait
        lp_commit(dbar);
        lp_bar_wait(dbar, 0, err, true);
        if (!wok) lp_bar_wait(wbar, 0, err, true);
        for (long w = wok ? step : 0; w < issued; ++w)
          lp_bar_wait(full0 + 8 * int(w % ST), unsigned((w / ST) & 1), err, true);
      }
    }
  } else {
    // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31, one row each
    const int q = warp & 3;
    const int row = 32 * q + lane;
    for (long tl = 0; tl < my_tiles; ++tl) {
      const int ab = int(tl & 1);
      if (!lp_bar_wait(accf0 + 8 * ab, unsigned((tl >> 1) & 1), err)) break;
      lp_tc_fence_after();
      float v[COUT];
      lp_tmem_ld<COUT>(tmem + (unsigned(32 * q) << 16) + ab * COUT, v);
      lp_tc_fence_before();
      __syncwarp();
      if (lane == 0) lp_bar_arrive(acce0 + 8 * ab);
      const long p = P.p0 + (blockIdx.x + tl * gridDim.x) * LP_TM + row;
      if (p >= P.p1) continue;
      const long l = lp_node(P, p);
      if (l < 0) continue;
#pragma unroll
      for (int c8 = 0; c8 < COUT / 8; ++c8) {
        float w8[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          w8[j] = v[8 * c8 + j] + (bias ? bias[8 * c8 + j] : 0.0f);
          if (relu) w8[j] = fmaxf(w8[j], 0.0f);
        }
        if (mask) {
          const uint4 mv = *reinterpret_cast<const uint4*>(mask + p * COUT + 8 * c8);
          const bf16* mb = reinterpret_cast<const bf16*>(&mv);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (!(__bfloat162float(mb[j]) > 0.0f)) w8[j] = 0.0f;
        }
        if (out) {
          uint4 ov;
          bf16* ob = reinterpret_cast<bf16*>(&ov);
#pragma unroll
          for (int j = 0; j < 8; ++j) ob[j] = __float2bfloat16(w8[j]);
          *reinterpret_cast<uint4*>(out + p * COUT + 8 * c8) = ov;
        }
        if (out32) {
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (8 * c8 + j < cout32) out32[(long)(8 * c8 + j) * P.N + l] = w8[j];
        }
      }
    }
  }
  lp_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    lp_tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}


// ---------------------------------------------------------------------------
// Weight and bias gradients of one layer on the tensor cores:
//   part[cta][o][ci][co] = sum_p X[p + off(o)][ci] D[p][co],
//   part[cta][27 CIN COUT + co] = sum_p D[p][co],
// p over a contiguous range of tiles per CTA (D is zero on halo rows; rows
// past the last interior row read as zero).  The contraction runs over rows,
// so both operands are MN-major: A = X windows, M = (window, channel); B = D,
// N = the output channels.  G = 128 / CIN windows of consecutive (dj, dk)
// pairs sit in consecutive buffers one window apart, so (window, 8-channel
// chunk) is a uniform core-matrix stride of one slab and one M = 128 MMA
// covers G offsets of the same di.  Groups of G windows: 3 (CIN 32) or 2
// (CIN 16) per tile, the last one partly used.  Each (group, di) owns an
// accumulator of COUT columns in tensor memory for the CTA's whole tile
// range; one CTA per SM.  Warp 0 (one lane) issues the copies and MMAs; warps
// 1-4 sum the bias gradient from each staged D tile and, at the end, move the
// accumulators to the partial slot.
// ---------------------------------------------------------------------------
template <int CIN, int COUT>
struct LpWgTc {
  static constexpr int G = 128 / CIN;                  // windows per group
  static constexpr int NG = (9 + G - 1) / G;           // groups per tile
  static constexpr int NACC = NG * 3;                  // accumulators
  static constexpr int COLS = NACC * COUT <= 256 ? 256 : 512;
  static constexpr int KCH = CIN / 8, DCH = COUT / 8;
  static constexpr size_t win = size_t(KCH) * LP_TC_SLAB;
  static constexpr size_t grp = G * win;               // one group buffer
  static constexpr size_t dt = size_t(DCH) * LP_TC_SLAB;
  static constexpr int NGS = 4;                        // group stages
  static constexpr size_t bars = 8 * (2 * NGS + 6);    // gfull, gempty, dfull x2, dempty x2, done, drain
  static constexpr size_t total = NGS * grp + 2 * dt + bars + 16 + 4 * 128 * COUT;
  static_assert(NACC * COUT <= 512, "accumulators fit tensor memory");
  static_assert(grp % 128 == 0 && dt % 128 == 0, "TMA destinations stay 128-byte aligned");
};

// MN-major instruction descriptor: FP32 accumulator, BF16 A and B, M = 128.
DESALM_HD constexpr unsigned lp_idesc_mn(int n) { return lp_idesc(n) | (1u << 15) | (1u << 16); }

template <int CIN, int COUT>
__global__ void __launch_bounds__(LP_TC_THREADS, 1)
    k_lp_wgrad_tc(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap dmap, LpPad P,
                  float* __restrict__ part, int* err) {
  pdl_wait();
  using C = LpWgTc<CIN, COUT>;
  constexpr int G = C::G, NG = C::NG, KCH = C::KCH, DCH = C::DCH, NGS = C::NGS;
  constexpr unsigned IDESC = lp_idesc_mn(COUT);
  constexpr unsigned COLS = C::COLS;
  constexpr long SLOT = 27L * CIN * COUT + COUT;
  extern __shared__ __align__(128) unsigned char lp_wg_smem[];
  unsigned char* Gb = lp_wg_smem;                      // NGS group buffers
  unsigned char* Db = lp_wg_smem + NGS * C::grp;       // two D tiles
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(lp_wg_smem + NGS * C::grp + 2 * C::dt);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(lp_wg_smem + NGS * C::grp + 2 * C::dt + C::bars);
  float* bred = reinterpret_cast<float*>(lp_wg_smem + NGS * C::grp + 2 * C::dt + C::bars + 16);  // [128][COUT]
  const unsigned gfull = lp_smem_u32(bars), gempty = gfull + 8 * NGS, dfull = gempty + 8 * NGS, dempty = dfull + 16;
  const unsigned done = dempty + 16, dbar = done + 8;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long ntiles = (P.p1 - P.p0 + LP_TM - 1) / LP_TM;
  const long per = (ntiles + gridDim.x - 1) / gridDim.x;
  const long ta = blockIdx.x * per, tb = min(ntiles, ta + per);
  const long my = tb > ta ? tb - ta : 0;
  const long S = my * NG;  // (tile, group) steps

  if (tid == 0) {
    for (int b = 0; b < NGS; ++b) {
      lp_bar_init(gfull + 8 * b, 1);
      lp_bar_init(gempty + 8 * b, 1);
    }
    for (int b = 0; b < 2; ++b) {
      lp_bar_init(dfull + 8 * b, 1);
      lp_bar_init(dempty + 8 * b, 1 + 4);  // the last group's MMAs and the four bias warps
    }
    lp_bar_init(done, 1);
    lp_bar_init(dbar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(lp_smem_u32(tmem_slot)),
                 "r"(COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  lp_tc_fence_before();
  __syncthreads();
  lp_tc_fence_after();
  const unsigned tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0 && S > 0) {
      auto t0_of = [&](long tl) { return P.p0 + (ta + tl) * LP_TM; };
      // copies of step (tile tl, group gr) into group buffer gr's stage; the
      // D tile with the first group
      auto issue = [&](long step) {
        const long tl = step / NG;
        const int gr = int(step % NG);
        const int b = int(step % NGS);
        const int nw = min(G, 9 - G * gr);
        const long t0 = t0_of(tl);
        const unsigned dst = lp_smem_u32(Gb + b * C::grp);
        lp_bar_expect_tx(gfull + 8 * b, nw * KCH * LP_WROWS * 16);
        for (int w = 0; w < nw; ++w) {
          const int g = G * gr + w;
          const int dj = g % 3 - 1, dk = g / 3 - 1;
          const int y = int(t0 + (long)P.ip * (dj + (long)P.jp * dk) - 1);
          for (int c = 0; c < KCH; ++c) lp_tma_2d(dst + w * C::win + c * LP_TC_SLAB, &xmap, 8 * c, y, gfull + 8 * b);
        }
      };
      auto issue_d = [&](long tl) {
        const int b = int(tl & 1);
        const unsigned dst = lp_smem_u32(Db + b * C::dt);
        lp_bar_expect_tx(dfull + 8 * b, DCH * LP_WROWS * 16);
        for (int c = 0; c < DCH; ++c) lp_tma_2d(dst + c * LP_TC_SLAB, &dmap, 8 * c, int(t0_of(tl)), dfull + 8 * b);
      };
      long issued = 0, dissued = 0;
      issue_d(0);
      dissued = 1;
      for (; issued < NGS && issued < S; ++issued) issue(issued);
      bool ok = true;
      long step = 0;
      for (; step < S; ++step) {
        const long tl = step / NG;
        const int gr = int(step % NG);
        const int b = int(step % NGS), db = int(tl & 1);
        if (gr == 0) {
          // the next D tile goes into the other buffer once the tile before has released it
          if (tl + 1 < my) {
            if (tl >= 1 && !lp_bar_wait(dempty + 8 * (db ^ 1), unsigned(((tl - 1) >> 1) & 1), err)) { ok = false; break; }
            issue_d(tl + 1);
            ++dissued;
          }
          if (!lp_bar_wait(dfull + 8 * db, unsigned((tl >> 1) & 1), err)) { ok = false; break; }
        }
        if (!lp_bar_wait(gfull + 8 * b, unsigned((step / NGS) & 1), err)) { ok = false; break; }
        lp_tc_fence_after();
        const unsigned abase = lp_smem_u32(Gb + b * C::grp), bbase = lp_smem_u32(Db + db * C::dt);
#pragma unroll
        for (int di = 0; di < 3; ++di) {
#pragma unroll
          for (int ks = 0; ks < LP_TM / 16; ++ks) {
            const unsigned long long a = lp_desc(abase + 16 * di + 256 * ks, 128, LP_TC_SLAB);
            const unsigned long long bd = lp_desc(bbase + 256 * ks, 128, LP_TC_SLAB);
            lp_mma(tmem + (gr * 3 + di) * COUT, a, bd, IDESC, (tl | ks) != 0);
          }
        }
        lp_commit(gempty + 8 * b);
        if (gr == NG - 1) lp_commit(dempty + 8 * db);
        // refill the previous step's group buffer once its MMAs are done
        if (step >= 1 && step - 1 + NGS < S) {
          const long ps = step - 1;
          if (!lp_bar_wait(gempty + 8 * int(ps % NGS), unsigned((ps / NGS) & 1), err)) { ++step; ok = false; break; }
          issue(ps + NGS);
          ++issued;
        }
      }
      lp_commit(done);
      if (!ok) {
        // drain: the MMAs issued so far, and the copies started but not consumed
        lp_commit(dbar);
        lp_bar_wait(dbar, 0, err, true);
        for (long w = step; w < issued; ++w) lp_bar_wait(gfull + 8 * int(w % NGS), unsigned((w / NGS) & 1), err, true);
        for (long t = (step + NG - 1) / NG; t < dissued; ++t)
          lp_bar_wait(dfull + 8 * int(t & 1), unsigned((t >> 1) & 1), err, true);
      }
    }
  } else {
    // ---- bias warps: row 32 (w % 4) + lane of every D tile
    const int q = warp & 3, row = 32 * q + lane;
    float bs[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) bs[c] = 0.0f;
    bool ok = true;
    for (long tl = 0; tl < my; ++tl) {
      const int db = int(tl & 1);
      if (!lp_bar_wait(dfull + 8 * db, unsigned((tl >> 1) & 1), err)) { ok = false; break; }
      const unsigned char* D0 = Db + db * C::dt + row * 16;
#pragma unroll
      for (int c = 0; c < DCH; ++c) {
        const uint4 v = *reinterpret_cast<const uint4*>(D0 + c * LP_TC_SLAB);
        const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
        for (int j = 0; j < 8; ++j) bs[8 * c + j] += __bfloat162float(e[j]);
      }
      __syncwarp();
      if (lane == 0) lp_bar_arrive(dempty + 8 * db);
    }
#pragma unroll
    for (int c = 0; c < COUT; ++c) bred[row * COUT + c] = bs[c];
    // ---- accumulators -> partial slot (after every MMA)
    if (ok && my > 0 && lp_bar_wait(done, 0, err)) {
      lp_tc_fence_after();
      float* slot = part + blockIdx.x * SLOT;
      for (int gr = 0; gr < NG; ++gr)
        for (int di = 0; di < 3; ++di) {
          float v[COUT];
          lp_tmem_ld<COUT>(tmem + (unsigned(32 * q) << 16) + (gr * 3 + di) * COUT, v);
          const int gi = row / CIN, ci = row % CIN, g = G * gr + gi;
          if (g < 9) {
            const int o = 3 * g + di;
            float4* dst = reinterpret_cast<float4*>(slot + ((long)o * CIN + ci) * COUT);
#pragma unroll
            for (int c = 0; c < COUT / 4; ++c) dst[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
          }
        }
      lp_tc_fence_before();
    } else if (my == 0) {
      float* slot = part + blockIdx.x * SLOT;
      for (long e = row; e < 27L * CIN * COUT; e += 128) slot[e] = 0.0f;
    }
  }
  __syncthreads();
  if (tid >= 32 && tid < 32 + COUT) {
    const int c = tid - 32;
    float t = 0.0f;
    for (int r = 0; r < 128; ++r) t += bred[r * COUT + c];
    part[blockIdx.x * SLOT + 27L * CIN * COUT + c] = t;
  }
  lp_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    lp_tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
  }
}

// Watchdog self-test: one thread waits on an mbarrier that nothing completes,
// with a limit of limit_ns, through the same bounded wait as the kernels
// above; it must give up and set *err.  Nothing else is in flight.
__global__ void k_wait_probe(unsigned long long limit_ns, int* err) {
  __shared__ unsigned long long bar;
  if (threadIdx.x != 0) return;
  const unsigned b = lp_smem_u32(&bar);
  lp_bar_init(b, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  lp_bar_wait(b, 0, err, false, limit_ns);
}

}  // namespace desalm
