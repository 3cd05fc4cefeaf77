// desalm.cu -- host runtime and C ABI of the B200 DES-ALM pseudo-time iteration.
//
// The context owns every device array (allocated once per level at init),
// the CUDA stream all work is ordered on, and the host-side mirror of the
// reference's mg_driver control flow (src/mg_driver.F90:2-323).  Each public
// function in include/desalm.h maps to one reference subroutine; kernels are
// in resid.cuh (K_R), sweep.cuh (K_I/K_J/K_K), mg.cuh (transfers, boundary
// conditions, norm, metrics) and sa.cuh (Spalart-Allmaras).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <utility>
#include <random>
#include <type_traits>

#include "desalm.h"
#include "common.cuh"
#include "resid.cuh"
#include "sweep.cuh"
#include "mg.cuh"
#include "sa.cuh"
#include "learn.cuh"
#include "learn_tc.cuh"
#include "alm.cuh"
#include "kw.cuh"
#include "outlet.cuh"
#include "wallfn.cuh"
#include "rfg.cuh"

using namespace desalm;

// Kernel launch through cudaLaunchKernelEx with programmatic stream
// serialisation: the launch of each kernel overlaps the completion of the
// one before it, and the kernel's pdl_wait() keeps its reads behind that
// grid's writes.  On the channel workload this measured 0.474 against 0.480
// s per MIXED physical step.  Failures are reported by the next
// cudaGetLastError().
constexpr int kProgrammaticLaunch = 1;
template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = kProgrammaticLaunch;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

namespace {

// Convergence state of the device-side pseudo-time loop.
struct DevConv {
  int itc, converged, pivots, nonfinite, zero_pivots, pivot_lines;
  double res[5], init[5];
};

struct ConvPar {
  int it_min, itmax;
  double er_min, eo_min, tnu;
};

// mg_residual + mg_ck_conver on the device (src/mg_residual.F90:77-84,
// src/mg_driver.F90:372-398): sums the norm partials, updates the loop
// state and sets the while-node condition of the graph.
__global__ void k_conv(const double* part, int nblk, DevConv* st, const int* flags, ConvPar cp,
                       cudaGraphConditionalHandle h) {
  pdl_wait();
  double sums[5];
  desalm::block_sum5(part, nblk, sums);   // every thread gets the sums
  if (threadIdx.x != 0) return;
  double res[5];
  for (int m = 0; m < 5; ++m) {
    res[m] = log10(sums[m] / cp.tnu);
    st->res[m] = res[m];
  }
  st->itc += 1;
  st->pivots += flags[0];
  st->zero_pivots += flags[1];
  st->pivot_lines += flags[2];
  if (st->itc == 1)
    for (int m = 0; m < 5; ++m) st->init[m] = res[m];
  double eomax = fmax(res[1], fmax(res[2], res[3]));
  double ermax = fmax(res[1] - st->init[1], fmax(res[2] - st->init[2], res[3] - st->init[3]));
  int conv = 0;
  if (st->itc > cp.it_min && ermax < cp.er_min) conv = 1;
  if (st->itc > cp.it_min && eomax < cp.eo_min) conv = 1;
  int finite = isfinite(res[1]) && isfinite(res[2]) && isfinite(res[3]);
  st->converged = conv;
  st->nonfinite = !finite;
  cudaGraphSetConditional(h, (!conv && finite && st->zero_pivots == 0 && st->itc < cp.itmax) ? 1u : 0u);
}

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

// One level: storage type chosen at runtime (FP64 or FP32 state, FP64 or
// FP32 sweep work); exactly one of the typed views is active.
struct Level {
  int im = 0, jm = 0, km = 0;
  long N = 0;
  double dc = 1, de = 1, dz = 1;
  int tbytes = 8, wbytes = 8;  // state / work element sizes
  std::vector<void*> allocs;
  Lv<double, double> dd{};
  Lv<double, float> df{};
  void* dq[4] = {nullptr, nullptr, nullptr, nullptr};  // prolongation correction
  double* fac[3] = {nullptr, nullptr, nullptr};         // rsmooth multipliers
  double* dpr[3] = {nullptr, nullptr, nullptr};         // rsmooth eliminated diagonal [n], then its reciprocals [n]
  bool dtau_valid = false;
};

// State of the learned initial guess (learn.cuh).
struct LpState {
  bool on = false;
  long N = 0;
  LpPad P{};                               // the fine level's zero-padded grid
  LpLayer ly[4];
  long nparam = 0;
  float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;  // flat parameters, gradient, Adam moments
  bf16 *wf[4] = {}, *wd[4] = {};           // forward / data-gradient weight blocks
  float *dW[4] = {}, *db[4] = {};          // per-layer weight and bias gradients (db inside dW's block)
  float* part = nullptr;                   // per-CTA partial gradients of k_lp_wgrad
  CUtensorMap tm_x0, tm_x1, tm_a[3], tm_dy4, tm_dya[2];  // TMA maps of the convolutions' inputs
  int* err = nullptr;                      // set by a tensor-core kernel whose wait timed out
  bf16 *x0 = nullptr, *a[3] = {}, *dy4 = nullptr, *dya[2] = {};  // features, activations, gradients
  bf16* x1 = nullptr;                      // features of the newest training sample
  float* yt = nullptr;                     // the training passes' output [5][N] (y keeps the guess's)
  // Training overlaps the physical step it precedes: its Adam steps run on
  // their own stream (ls while they are launched, the context's stream
  // otherwise) beside the pseudo-iterations, which touch none of the
  // network's buffers; the next use of the network waits for them (lp_join).
  cudaStream_t ls = nullptr, tstream = nullptr;
  cudaEvent_t ev_pred = nullptr, ev_train = nullptr;
  bool pending = false, inflight = false;
  double* h_loss = nullptr;                // pinned: the losses of the training in flight
  int h_loss_n = 0;
  float *y = nullptr, *t = nullptr;        // network output, training target [5][N]
  float *rs = nullptr, *rs5 = nullptr, *s5 = nullptr;  // feature scales (1/RMS), target scales, output scales
  double* acc = nullptr;                   // reductions
  double* red = nullptr;                   // their per-CTA partial sums [kLpRedBlocks][16]
  double* vacc = nullptr;                  // held-out check of the newest sample (k_lp_dot)
  float* alpha = nullptr;                  // blend of each field's correction
  float fixed_alpha = -1.0f;               // < 0: automatic blend
  // bit f: field f takes the correction.  Default none: the linear
  // extrapolation of converged time levels satisfies the discrete continuity
  // and momentum balance to second order in dt, and a pointwise correction
  // of any field breaks that consistency, which the artificial-compressibility
  // iteration then relaxes slowly.  Measured: velocity corrections cost 8.6
  // more pseudo-iterations per step on the cavity; on the turbine box a
  // pressure correction raised steps from 91-128 to 134-312 pseudo-iterations
  // (blend 0.25: 98-219), a turbulence-field correction to 103-190.  The
  // network still trains on every step and reports its held-out error.
  int field_mask = 0x00;
  double* qnm2[5] = {};                    // q^{n-2} of the fine level
  double* nut0 = nullptr;                  // nu_t at the start of a step begun from the network's guess
  double** tab = nullptr;                  // device table: q[5] qn[5] qnm1[5] qnm2[5]
  double* tab_h[20] = {};                  // the same pointers on the host
  int shifts = 0;                          // history shifts since the state was set
  bool predicted = false;                  // the current step began from the network's guess
  long samples = 0, steps = 0, predictions = 0, fallbacks = 0, adam_t = 0;
  long hold_until = 0;                     // no guesses before this many samples (after a fallback)
  double first_loss = -1, last_loss = -1;
  int train_steps = 8;                     // Adam steps per new sample
  int warm = 2;                            // samples before the network's guess is used
  float lr = 1e-3f;
  float ymax = LP_YMAX;                    // limit of |output| in the guess
};

}  // namespace

struct desalm_ctx {
  desalm_case c{};
  int ng = 0;
  std::vector<Level> L;
  cudaStream_t stream = nullptr;
  // a second stream for kernels that need not wait for the ones before them
  // (fork_side / join_side); forks and joins are captured as graph edges
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool alm_pending = false;  // this iteration's forcing runs on the side stream
  Par par{};
  std::string err;
  bool have_grid = false, have_state = false;
  bool have_wd = false;  // desalm_set_grid was given the wall distance
  // fine-level extras (always FP64)
  double *x = nullptr, *y = nullptr, *z = nullptr, *wd = nullptr, *dtev = nullptr;
  double* cov[9] = {};
  double** dcov = nullptr;    // device copy of cov[]
  double* rat = nullptr;
  int ratdim = 0;
  // lines per CTA of each level's DAF sweeps [level][direction], picked by
  // timing when the grid is set (autotune_sweeps): 16, 8 or 4 for the
  // shared-memory slab kernel, 1 for the lines-in-lanes kernel; 0: the
  // default (lines in lanes)
  int sweep_nl[4][3] = {};
  // the turbulence sweeps' kernel per direction: 1 lines in lanes, 16/8 the
  // slab's lines per CTA; 0: the default (lines in lanes)
  int sa_nl[3] = {};
  // CTA tile (i, j, k threads) of each level's residual kernels [level][0 =
  // K_R first pass, 1 = recalculation, 2 = turbulence residual], picked by
  // timing when the grid is set (autotune_tiles); the build's default shape
  // where the timing is off.  The tile changes the time only: every node is
  // computed by the same operations.
  unsigned tile[4][3][3] = {{{32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}},
                            {{32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}},
                            {{32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}},
                            {{32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}, {32, DESALM_KR_BY, DESALM_KR_BZ}}};
  double* pfix = nullptr;     // device scalar (type of the fine level: double)
  double* part = nullptr;     // norm partials
  int part_blocks = 0;
  double* norm = nullptr;     // device [5]
  double* h_norm = nullptr;   // pinned host [5]
  double* stage = nullptr;    // device staging of one host state array, 5 N (component-fastest)
  double** ftab = nullptr;    // device table of the fine level's q[5], qn[5], qnm1[5] field pointers
  LpState lp;                 // learned initial guess (predictor DESALM_PRED_LEARNED)
  struct {
    bool on = false;
    AlmDev dev{};
    std::vector<int> nker, elem0;     // per turbine
    double* falm = nullptr;           // [3][N] force added to rh(2:4) on the fine level
    std::vector<void*> allocs;        // this forcing's device tables
  } alm;                      // actuator-line forcing (rhs_lines)
  int* flags = nullptr;       // device [3]
  // scratch of the lines-in-lanes sweeps (k_gsweep, k_sa_gsweep): 16 arrays
  // of gss elements (rows x padded lines of the fine level's longest sweep)
  // in the sweep precision, shared by every level and sweep (they run one
  // after another on the stream)
  void* gsweep = nullptr;
  int gss = 0;
  SaWork sa{};
  KwWork kw{};                // k-omega work (turbulence = 2)
  struct {
    bool on = false;
    bool armed = false;               // desalm_rfg_inlet forced the plane since the last begin_step
    double time = 0.0;                // the time it was forced for
    RfgDev dev{};
    std::vector<void*> allocs;        // the generator's device tables
  } rfg;                      // synthetic inflow turbulence (rfg_inlet)
  int recalc = 0;             // decide_recalc_rh of the pseudo-iteration being enqueued
  double ckin = 1.0e-10, cein = 1.0e-6;  // k and omega floors on extrapolated faces
  // per-kernel CUDA-event timing (desalm_profile) and launch counter
  struct ProfRec { int cls, lvl; double nodes; cudaEvent_t a, b; };
  bool prof_on = false;
  std::vector<ProfRec> prof;
  size_t prof_used = 0;
  long launches = 0;
  // CUDA graph of a physical step's pseudo-time loop (use_graph = 1)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  long graph_kernels = 0;     // kernels per pseudo-iteration in the graph body
  DevConv* dconv = nullptr;   // device-side convergence state
  DevConv* hconv = nullptr;   // pinned host copy
  // driver state
  int itc = 0;
  double init_resd[5] = {0, 0, 0, 0, 0};
  std::vector<void*> allocs;
};

namespace {

#define CK(call)                                                                 \
  do {                                                                           \
    cudaError_t e__ = (call);                                                    \
    if (e__ != cudaSuccess) {                                                    \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e__);            \
      return DESALM_ECUDA;                                                       \
    }                                                                            \
  } while (0)

#define CKL()                                                                    \
  do {                                                                           \
    cudaError_t e__ = cudaGetLastError();                                        \
    if (e__ != cudaSuccess) {                                                    \
      ctx->err = std::string("kernel launch: ") + cudaGetErrorString(e__);       \
      return DESALM_ECUDA;                                                       \
    }                                                                            \
  } while (0)

#define RET(x)            \
  do {                    \
    int r__ = (x);        \
    if (r__) return r__;  \
  } while (0)

inline unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

// kernel classes for desalm_kernel_stats
enum KClass { KC_DTAU = 0, KC_RESID, KC_SWEEP_I, KC_SWEEP_J, KC_SWEEP_K, KC_RECALC, KC_BCOND, KC_PFIX,
              KC_NLEVEL, KC_PROLONG, KC_RSMOOTH, KC_NORM, KC_SA_RHS, KC_SA_SWEEP, KC_SA_BC,
              KC_XFORM_I, KC_XFORM_J, KC_XFORM_K, KC_SA_AUX, KC_LEARN, KC_ALM, KC_OUTLET, KC_WALLFN, KC_MISC, KC_COUNT };

struct ProfScope {
  desalm_ctx* ctx;
  size_t slot;
  bool on;
  ProfScope(desalm_ctx* c, int cls, int lvl, double nodes);
  ~ProfScope();
};

// Launch one kernel: count it and, when profiling, bracket it with events.
#define LAUNCH(CLS, LVL, NODES, ...)                 \
  do {                                               \
    ProfScope ps__(ctx, (CLS), (LVL), (NODES));      \
    __VA_ARGS__;                                     \
  } while (0)

int dalloc(desalm_ctx* ctx, std::vector<void*>& owner, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return DESALM_ENOMEM;
  }
  owner.push_back(*p);
  e = cudaMemsetAsync(*p, 0, bytes, ctx->stream);
  if (e != cudaSuccess) {
    ctx->err = std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
    return DESALM_ECUDA;
  }
  return 0;
}

template <class T, class W>
int alloc_level(desalm_ctx* ctx, Level& G, Lv<T, W>& L) {
  const long N = G.N;
  L.im = G.im; L.jm = G.jm; L.km = G.km;
  L.N = (int)N;
  L.sj = G.im; L.sk = G.im * G.jm;
  L.falm = nullptr;
  L.oute = 0;
  L.dc = T(G.dc); L.de = T(G.de); L.dz = T(G.dz);
  auto A = [&](T** p) { return dalloc(ctx, G.allocs, (void**)p, N * sizeof(T)); };
  auto AW = [&](W** p) { return dalloc(ctx, G.allocs, (void**)p, N * sizeof(W)); };
  for (int m = 0; m < 5; ++m) { RET(A(&L.q[m])); RET(A(&L.qn[m])); RET(A(&L.qnm1[m])); RET(A(&L.qold[m])); }
  for (int m = 0; m < 4; ++m) { RET(A(&L.rh[m])); RET(A(&L.pk[m])); }
  RET(A(&L.nut)); RET(A(&L.dtau)); RET(A(&L.diss1));
  RET(A(&L.dtc)); RET(A(&L.dtv));
  for (int d = 0; d < 3; ++d) {
    RET(A((T**)&L.csi[d])); RET(A((T**)&L.eta[d])); RET(A((T**)&L.zet[d]));
  }
  RET(A((T**)&L.aj));
  RET(A((T**)&L.rj));
  for (int t = 0; t < 9; ++t) {
    const T* m = t < 3 ? L.csi[t] : (t < 6 ? L.eta[t - 3] : L.zet[t - 6]);
    if (sizeof(W) == sizeof(T)) L.mw[t] = (const W*)m;
    else RET(AW((W**)&L.mw[t]));
  }
  for (int m = 0; m < 4; ++m) RET(AW(&L.wk[m]));
  RET(AW(&L.sig));
  for (int m = 0; m < 3; ++m) { RET(AW(&L.tc[m])); RET(AW(&L.hc[m])); }
  RET(dalloc(ctx, G.allocs, (void**)&L.bi, sizeof(W) * 8L * G.jm * G.km));
  RET(dalloc(ctx, G.allocs, (void**)&L.bj, sizeof(W) * 16L * G.im * G.km));
  RET(dalloc(ctx, G.allocs, (void**)&L.bk, sizeof(W) * 16L * G.im * G.jm));
  L.flags = ctx->flags;
  L.gs = (W*)ctx->gsweep;
  L.gss = ctx->gss;
  return 0;
}

// Shared memory of the slab kernels (line sweeps, SA sweeps, rsmooth): the
// widest slab that leaves room for two CTAs per SM is used, else the widest
// that fits one (below the 227 KB opt-in less the kernels' static shared
// memory).
constexpr size_t kSlabTwoPerSm = 110 * 1024;
constexpr size_t kSlabMax = 220 * 1024;

int check_case(desalm_ctx* ctx, const desalm_case& c) {
  auto bad = [&](const char* why) { ctx->err = why; return DESALM_EINVAL; };
  if (c.ng < 1 || c.ng > 4) return bad("ng must be 1..4");
  if (c.im < 5 || c.jm < 5 || c.km < 5) return bad("each extent must be >= 5");
  if ((c.icrs != 0 && c.icrs != 1) || (c.jcrs != 0 && c.jcrs != 1) || (c.kcrs != 0 && c.kcrs != 1))
    return bad("icrs/jcrs/kcrs must be 0 or 1");
  if (c.precision_mode != DESALM_FP64 && c.precision_mode != DESALM_MIXED) return bad("unknown precision_mode");
  if (c.wall_functions != 0 && c.wall_functions != 1) return bad("wall_functions must be 0 or 1");
  if (c.turbulence < 0 || c.turbulence > 2) return bad("turbulence must be 0 (laminar), 1 (Spalart-Allmaras) or 2 (k-omega)");
  if (c.predictor != DESALM_PRED_QN && c.predictor != DESALM_PRED_LINEAR && c.predictor != DESALM_PRED_LEARNED)
    return bad("unknown predictor");
  if (c.ifix < 1 || c.ifix > c.im || c.jfix < 1 || c.jfix > c.jm || c.kfix < 1 || c.kfix > c.km)
    return bad("pressure reference node outside the grid");
  // vertex-centred coarsening (ii = 2i - 1) needs odd extents on every level
  int im = c.im, jm = c.jm, km = c.km;
  for (int n = 1; n < c.ng; ++n) {
    if ((c.icrs && im % 2 == 0) || (c.jcrs && jm % 2 == 0) || (c.kcrs && km % 2 == 0))
      return bad("full coarsening needs odd extents on every level above the coarsest");
    im = (im + c.icrs) >> c.icrs; jm = (jm + c.jcrs) >> c.jcrs; km = (km + c.kcrs) >> c.kcrs;
    if (im < 5 || jm < 5 || km < 5) return bad("coarsest level must keep >= 5 nodes per direction");
  }
  if ((long)c.im * c.jm * c.km * 4 >= (1L << 31)) return bad("grid too large for 32-bit indexing");
  // the narrowest slab of every line solve must fit: DAF sweep 4 lines of
  // 10 W-fields, rsmooth 4 lines of 4 W-fields, SA sweep 8 lines of 4 W-fields
  const size_t wb = c.precision_mode == DESALM_FP64 ? 8 : 4;
  for (int n : {c.im - 2, c.jm - 2, c.km - 2})
    if ((size_t)10 * slab_fs(n + 2, 5) * wb > kSlabMax || (size_t)4 * slab_fs(n, 5) * wb > kSlabMax ||
        (size_t)4 * slab_fs(n, 9) * wb > kSlabMax)
      return bad("a grid line is too long for the shared-memory line solves (at most 554 interior nodes in "
                 "FP64 mode, 1118 in MIXED mode)");
  return 0;
}

void fill_par(desalm_ctx* ctx) {
  const desalm_case& c = ctx->c;
  Par& P = ctx->par;
  P.ren = c.ren; P.beta = c.beta; P.delti = c.delti; P.es = c.unsteady ? 1.0 : 0.0;
  P.cfl1 = c.cfl1; P.vnn1 = c.vnn1; P.pdiss = c.pdiss_coef;
  for (int d = 0; d < 3; ++d) { P.ep1[d] = c.ep[0][d]; P.ep2[d] = c.ep[1][d]; }
  // src/init.F90:482-509
  for (int m = 0; m < 4; ++m)
    for (int b = 0; b < 6; ++b) { P.sa[m][b] = 4.0 / 3.0; P.sb[m][b] = -(1.0 / 3.0); }
  for (int b = 0; b < 6; ++b) {
    P.btype[b] = c.btype[b];
    if (c.btype[b] == 1) for (int m = 1; m < 4; ++m) { P.sa[m][b] = 0; P.sb[m][b] = 0; }
    if (c.btype[b] == 2) {
      int m = c.bdir[b];
      if (m >= 1 && m <= 3) { P.sa[m][b] = 0; P.sb[m][b] = 0; }
    }
  }
  P.fine = 0;
}

// rsmooth factors for a line of n interior nodes: SGTSV's elimination of
// (-e, 1+2e, -e) in its own order (src/sgtsv.f:163-176).
void rs_factors(int n, double e, std::vector<double>& fac, std::vector<double>& dpr) {
  fac.assign(std::max(n - 1, 1), 0.0);
  dpr.assign(n, 0.0);
  const double dl = -e, du = -e, dg = 1.0 + 2.0 * e;
  dpr[0] = dg;
  for (int p = 0; p + 1 < n; ++p) {
    double f = dl / dpr[p];
    fac[p] = f;
    dpr[p + 1] = dg - f * du;
  }
}

// launch helpers --------------------------------------------------------------
dim3 blk3() { return dim3(32, 4, 1); }
template <class T, class W>
dim3 grid_interior(const Lv<T, W>& L) { return dim3(cdiv(L.im - 2, 32), cdiv(L.jm - 2, 4), L.km - 2); }
// the residual kernels' CTA shape (DESALM_KR_BY j rows x DESALM_KR_BZ k planes)
// the tuned tile of residual kernel `which` on level lvl, and its grid over the interior
dim3 blk_t(const desalm_ctx* ctx, int lvl, int which) {
  const unsigned* t = ctx->tile[lvl][which];
  return dim3(t[0], t[1], t[2]);
}
dim3 grid_t(const desalm_ctx* ctx, int lvl, int which, int im, int jm, int km) {
  const unsigned* t = ctx->tile[lvl][which];
  const int kl = which < 2 ? DESALM_KR_KLOOP : 1;   // a K_R thread takes DESALM_KR_KLOOP k planes
  return dim3(cdiv(im - 2, t[0]), cdiv(jm - 2, t[1]), cdiv(km - 2, t[2] * kl));
}
// K_R (MODE 0) or the recalculation (MODE 1) on level lvl: the tile
// KRF_TX x KRF_TY x KRF_TZ (31 x 4 x 2) is the face-shared k_resid_f, any
// other the one-node-per-thread k_resid with that CTA shape.  Both compute
// every node by the same operations.
template <class T, class W, int MODE>
cudaError_t launch_resid(const desalm_ctx* ctx, int lvl, cudaStream_t s, const Lv<T, W>& L, const Par& P, int upwind, int calc_pk,
                         int coarse, int bback) {
  const unsigned* t = ctx->tile[lvl][MODE];
  if (t[0] == KRF_TX && t[1] == KRF_TY && t[2] == KRF_TZ)
    return launch_k(k_resid_f<T, W, MODE>, dim3(cdiv(L.im - 2, KRF_TX), cdiv(L.jm - 2, KRF_TY), cdiv(L.km - 2, KRF_TZ)), 256, 0, s, L, P,
                    upwind, calc_pk, coarse, bback);
  return launch_k(k_resid<T, W, MODE>, grid_t(ctx, lvl, MODE, L.im, L.jm, L.km), blk_t(ctx, lvl, MODE), 0, s, L, P, upwind, calc_pk,
                  coarse, bback);
}

// One DAF line sweep as k_sweep4 with the widest slab (lines per CTA) whose
// shared memory leaves room for two CTAs per SM, else the widest that fits
// one CTA per SM.
template <class W>
size_t slab_bytes(int n, int nl) { return (size_t)10 * slab_fs(n + 2, nl + 1) * sizeof(W); }

// A slab of at most 48 KB (four or more CTAs per SM) runs with its 8 NL
// solver threads only; a larger one with kSlabThreads, the extra threads
// sharing the copies.  Both variants have the shared-memory opt-in, since the
// static arrays come on top of the slab.
constexpr size_t kSlabFourPerSm = 48 * 1024;
template <class T, class W, int DIR, int NL>
int sweep4_nl(desalm_ctx* ctx, Lv<T, W>& L, const Par& P, int lvl, int blo, int bhi, bool xform = true) {
  int amax, n, nb;
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; nb = L.km - 2; }
  else if (DIR == 1) { amax = L.im - 2 + L.oute; n = L.jm - 2; nb = L.km - 2; }
  else { amax = L.im - 2 + L.oute; n = L.km - 2; nb = L.jm - 2; }
  const size_t bytes = slab_bytes<W>(n, NL);
  const int cls = DIR == 0 ? KC_SWEEP_I : (DIR == 1 ? KC_SWEEP_J : KC_SWEEP_K);
  const double nin = double(amax) * n * nb;
  cudaStream_t s = ctx->stream;
  if (bytes <= kSlabFourPerSm)
    LAUNCH(cls, lvl, nin, launch_k(k_sweep4<T, W, DIR, NL, 8 * NL>, dim3(cdiv(amax, NL), nb), 8 * NL, bytes, s, L, P, blo, bhi));
  else
    LAUNCH(cls, lvl, nin, launch_k(k_sweep4<T, W, DIR, NL, kSlabThreads>, dim3(cdiv(amax, NL), nb), kSlabThreads, bytes, s, L, P, blo, bhi));
  CKL();
  if (!xform) return 0;
  const int xcls = DIR == 0 ? KC_XFORM_I : (DIR == 1 ? KC_XFORM_J : KC_XFORM_K);
  const dim3 gx(cdiv(L.im - 2 + L.oute, 32), cdiv(L.jm - 2, 4), L.km - 2);
  LAUNCH(xcls, lvl, nin, launch_k(k_xform<T, W, DIR>, gx, blk3(), 0, s, L));
  CKL();
  return 0;
}

// Shared-memory opt-in of every slab kernel (line sweeps, SA sweeps,
// rsmooth) on the current device (done when a context is created, outside any
// stream capture).
template <class T, class W>
cudaError_t slab_attrs() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  auto set = [&](const void* f) {
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return;
    const int mx = (int)std::min<size_t>(kSlabMax, (size_t)optin - fa.sharedSizeBytes);
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
  };
  set((const void*)k_sweep4<T, W, 0, 16, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 0, 8, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 0, 4, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 0, 16, 128>);
  set((const void*)k_sweep4<T, W, 0, 8, 64>);
  set((const void*)k_sweep4<T, W, 0, 4, 32>);
  set((const void*)k_sweep4<T, W, 1, 16, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 1, 8, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 1, 4, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 1, 16, 128>);
  set((const void*)k_sweep4<T, W, 1, 8, 64>);
  set((const void*)k_sweep4<T, W, 1, 4, 32>);
  set((const void*)k_sweep4<T, W, 2, 16, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 2, 8, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 2, 4, kSlabThreads>);
  set((const void*)k_sweep4<T, W, 2, 16, 128>);
  set((const void*)k_sweep4<T, W, 2, 8, 64>);
  set((const void*)k_sweep4<T, W, 2, 4, 32>);
  set((const void*)k_sa_sweep4<W, 0, 32>); set((const void*)k_sa_sweep4<W, 0, 16>); set((const void*)k_sa_sweep4<W, 0, 8>);
  set((const void*)k_sa_sweep4<W, 1, 32>); set((const void*)k_sa_sweep4<W, 1, 16>); set((const void*)k_sa_sweep4<W, 1, 8>);
  set((const void*)k_sa_sweep4<W, 2, 32>); set((const void*)k_sa_sweep4<W, 2, 16>); set((const void*)k_sa_sweep4<W, 2, 8>);
  set((const void*)k_rsmooth4<T, W, 0, 16>); set((const void*)k_rsmooth4<T, W, 0, 8>); set((const void*)k_rsmooth4<T, W, 0, 4>);
  set((const void*)k_rsmooth4<T, W, 1, 16>); set((const void*)k_rsmooth4<T, W, 1, 8>); set((const void*)k_rsmooth4<T, W, 1, 4>);
  set((const void*)k_rsmooth4<T, W, 2, 16>); set((const void*)k_rsmooth4<T, W, 2, 8>); set((const void*)k_rsmooth4<T, W, 2, 4>);
  return e;
}

// One DAF sweep (and its transform unless xform is false) with the lines per
// CTA that autotune_sweeps picked for this level and direction, else the
// widest slab that leaves room for two CTAs per SM, else the widest that fits
// one.  Every line is solved by the same operations whatever the width, so
// the choice changes the time only.
template <class T, class W, int DIR>
int gsweep(desalm_ctx* ctx, Lv<T, W>& L, const Par& P, int lvl, int blo, int bhi, bool xform) {
  int amax, nb;
  if (DIR == 0) { amax = L.jm - 2; nb = L.km - 2; }
  else if (DIR == 1) { amax = L.im - 2 + L.oute; nb = L.km - 2; }
  else { amax = L.im - 2 + L.oute; nb = L.jm - 2; }
  const int n = DIR == 0 ? L.im - 2 : (DIR == 1 ? L.jm - 2 : L.km - 2);
  const int cls = DIR == 0 ? KC_SWEEP_I : (DIR == 1 ? KC_SWEEP_J : KC_SWEEP_K);
  const double nin = double(amax) * n * nb;
  cudaStream_t s = ctx->stream;
  LAUNCH(cls, lvl, nin, launch_k(k_gsweep<T, W, DIR>, dim3(cdiv(amax, 32), nb), 256, 0, s, L, P, blo, bhi));
  CKL();
  if (!xform) return 0;
  const int xcls = DIR == 0 ? KC_XFORM_I : (DIR == 1 ? KC_XFORM_J : KC_XFORM_K);
  const dim3 gx(cdiv(L.im - 2 + L.oute, 32), cdiv(L.jm - 2, 4), L.km - 2);
  LAUNCH(xcls, lvl, nin, launch_k(k_xform<T, W, DIR>, gx, blk3(), 0, s, L));
  CKL();
  return 0;
}

// The warp-shuffle cyclic reduction of lines of at most 32 rows (k_psweep):
// one CTA per line, a warp per system.
template <class T, class W, int DIR>
int psweep(desalm_ctx* ctx, Lv<T, W>& L, const Par& P, int lvl, int blo, int bhi, bool xform) {
  int amax, nb;
  if (DIR == 0) { amax = L.jm - 2; nb = L.km - 2; }
  else if (DIR == 1) { amax = L.im - 2 + L.oute; nb = L.km - 2; }
  else { amax = L.im - 2 + L.oute; nb = L.jm - 2; }
  const int n = DIR == 0 ? L.im - 2 : (DIR == 1 ? L.jm - 2 : L.km - 2);
  const int cls = DIR == 0 ? KC_SWEEP_I : (DIR == 1 ? KC_SWEEP_J : KC_SWEEP_K);
  const double nin = double(amax) * n * nb;
  cudaStream_t s = ctx->stream;
  LAUNCH(cls, lvl, nin, launch_k(k_psweep<T, W, DIR>, dim3(amax, nb), 128, 0, s, L, P, blo, bhi));
  CKL();
  if (!xform) return 0;
  const int xcls = DIR == 0 ? KC_XFORM_I : (DIR == 1 ? KC_XFORM_J : KC_XFORM_K);
  const dim3 gx(cdiv(L.im - 2 + L.oute, 32), cdiv(L.jm - 2, 4), L.km - 2);
  LAUNCH(xcls, lvl, nin, launch_k(k_xform<T, W, DIR>, gx, blk3(), 0, s, L));
  CKL();
  return 0;
}

// Rows of the DAF line systems of a direction: the interior nodes, and on the
// i lines of the fine level the outlet row.
template <class T, class W, int DIR>
int sweep_rows(const Lv<T, W>& L) {
  return DIR == 0 ? L.im - 2 + L.oute : (DIR == 1 ? L.jm - 2 : L.km - 2);
}
constexpr int kPcrRows = 32;   // lines this short are solved by k_psweep

template <class T, class W, int DIR>
int launch_sweep(desalm_ctx* ctx, Lv<T, W>& L, const Par& P, int lvl, int blo, int bhi, bool xform = true) {
  const int n = DIR == 0 ? L.im - 2 : (DIR == 1 ? L.jm - 2 : L.km - 2);
  const int want = lvl < 4 ? ctx->sweep_nl[lvl][DIR] : 0;
  const bool short_lines = sweep_rows<T, W, DIR>(L) <= kPcrRows;
  if ((want == 0 || want == 2) && short_lines) return psweep<T, W, DIR>(ctx, L, P, lvl, blo, bhi, xform);
  if (want == 0 || want == 1 || want == 2) return gsweep<T, W, DIR>(ctx, L, P, lvl, blo, bhi, xform);
  if (want == 16 && slab_bytes<W>(n, 16) <= kSlabMax) return sweep4_nl<T, W, DIR, 16>(ctx, L, P, lvl, blo, bhi, xform);
  if (want == 8 && slab_bytes<W>(n, 8) <= kSlabMax) return sweep4_nl<T, W, DIR, 8>(ctx, L, P, lvl, blo, bhi, xform);
  if (want == 4 && slab_bytes<W>(n, 4) <= kSlabMax) return sweep4_nl<T, W, DIR, 4>(ctx, L, P, lvl, blo, bhi, xform);
  if (slab_bytes<W>(n, 16) <= kSlabTwoPerSm) return sweep4_nl<T, W, DIR, 16>(ctx, L, P, lvl, blo, bhi, xform);
  if (slab_bytes<W>(n, 8) <= kSlabTwoPerSm) return sweep4_nl<T, W, DIR, 8>(ctx, L, P, lvl, blo, bhi, xform);
  if (slab_bytes<W>(n, 4) <= kSlabMax) return sweep4_nl<T, W, DIR, 4>(ctx, L, P, lvl, blo, bhi, xform);
  ctx->err = "grid line too long for the shared-memory line sweep";
  return DESALM_EINVAL;
}

// Fork: the side stream waits for everything enqueued so far on the main
// stream.  Join: the main stream waits for everything enqueued so far on the
// side stream.
int fork_side(desalm_ctx* ctx) {
  CK(cudaEventRecord(ctx->ev_fork, ctx->stream));
  CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0));
  return 0;
}
int join_side(desalm_ctx* ctx) {
  CK(cudaEventRecord(ctx->ev_join, ctx->side));
  CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0));
  return 0;
}

// rhs_lines on the fine level (src/solver_daf.F90:378-381): element forces,
// then each turbine's projection into alm.falm, which K_R's first pass adds.
template <class T, class W>
int alm_run(desalm_ctx* ctx, Lv<T, W>& L, cudaStream_t s) {
  auto& A = ctx->alm;
  CK(cudaMemsetAsync(A.falm, 0, 3L * L.N * sizeof(double), s));
  LAUNCH(KC_ALM, 0, double(A.dev.E), launch_k(k_alm_forces<T, W>, 1, 256, 0, s, A.dev, L));
  if (A.dev.nker_all > 0)
    LAUNCH(KC_ALM, 0, double(A.dev.nker_all), launch_k(k_alm_project<T, W>, cdiv(A.dev.nker_all, 128), 128, 0, s, A.dev, L, A.falm));
  CKL();
  return 0;
}

template <class T, class W>
int launch_daf(desalm_ctx* ctx, Lv<T, W>& L, Level& G, int n, int recalc, int itr) {
  Par P = ctx->par;
  P.fine = (n == 0);
  const desalm_case& c = ctx->c;
  cudaStream_t s = ctx->stream;
  if (!G.dtau_valid) {
    LAUNCH(KC_DTAU, n, L.N, launch_k(k_dtau<T, W>, cdiv(L.N, 256), 256, 0, s, L, P));
    CKL();
    G.dtau_valid = true;
  }
  const int fine = (n == 0);
  const int upwind = fine ? 2 : 1;
  const int bback = fine && c.btype[0] != 5;
  const double nin = double(L.im - 2) * (L.jm - 2) * (L.km - 2);
  if (n == 0 && ctx->alm.on) {
    // the forcing was started beside the SA sub-iterations (enqueue_iteration)
    // or runs here
    if (ctx->alm_pending) {
      RET(join_side(ctx));
      ctx->alm_pending = false;
    } else {
      RET(alm_run(ctx, L, s));
    }
  }
  // the outlet plane's residual and its preparation for the sweeps
  // (src/solver_daf.F90:318-358) reads only q and dtau and writes only the
  // plane, so it runs beside k_resid on the side stream; the back face's
  // call writes a plane that nothing reads, so it is not made
  const bool out_side = L.oute && !ctx->prof_on;
  if (out_side) {
    RET(fork_side(ctx));
    LAUNCH(KC_OUTLET, n, double(L.jm - 2) * (L.km - 2),
           launch_k(k_outlet<T, W>, dim3(cdiv(L.jm - 2, 32), cdiv(L.km - 2, 4)), dim3(32, 4), 0, ctx->side, L, P));
    CKL();
  }
  LAUNCH(KC_RESID, n, nin, (launch_resid<T, W, 0>(ctx, n, s, L, P, upwind, itr == 1 ? 1 : 0, n > 0 ? 1 : 0, bback)));
  CKL();
  if (out_side) RET(join_side(ctx));
  if (L.oute && !out_side) {
    LAUNCH(KC_OUTLET, n, double(L.jm - 2) * (L.km - 2),
           launch_k(k_outlet<T, W>, dim3(cdiv(L.jm - 2, 32), cdiv(L.km - 2, 4)), dim3(32, 4), 0, s, L, P));
    CKL();
  }
  RET((launch_sweep<T, W, 0>(ctx, L, P, n, bback, 0)));
  RET((launch_sweep<T, W, 1>(ctx, L, P, n, fine && c.btype[2] != 5, fine && c.btype[3] != 5)));
  RET((launch_sweep<T, W, 2>(ctx, L, P, n, fine && c.btype[4] != 5, fine && c.btype[5] != 5 && c.btype[5] != 6)));
  return 0;
}

template <class T, class W>
int launch_recalc(desalm_ctx* ctx, Lv<T, W>& L, int n) {
  Par P = ctx->par;
  P.fine = (n == 0);
  LAUNCH(KC_RECALC, n, double(L.im - 2) * (L.jm - 2) * (L.km - 2), (launch_resid<T, W, 1>(ctx, n, ctx->stream, L, P, n == 0 ? 2 : 1, 0, n > 0 ? 1 : 0, 0)));
  CKL();
  return 0;
}

template <class T, class W>
int launch_bcond(desalm_ctx* ctx, Lv<T, W>& L) {
  Par P = ctx->par;
  P.fine = 1;
  cudaStream_t s = ctx->stream;
  const T* rat = (const T*)ctx->rat;
  const desalm_case& c = ctx->c;
  const int lfix = (c.ifix - 1) + L.sj * (c.jfix - 1) + L.sk * (c.kfix - 1);
  T* pfix = (T*)ctx->pfix;
  LAUNCH(KC_BCOND, 0, 2.0 * L.jm * L.km, launch_k(k_bcond<T, W, 0>, dim3(cdiv(L.jm, 64), L.km), 64, 0, s, L, P, rat, ctx->ratdim, -1, -1, lfix, pfix));
  CKL();
  LAUNCH(KC_BCOND, 0, 2.0 * L.im * L.km, launch_k(k_bcond<T, W, 1>, dim3(cdiv(L.im, 64), L.km), 64, 0, s, L, P, rat, ctx->ratdim, -1, -1, lfix, pfix));
  CKL();
  // the k faces, then p(ifix, jfix, kfix) into pfix
  LAUNCH(KC_BCOND, 0, 2.0 * L.im * L.jm, launch_k(k_bcond<T, W, 2>, dim3(cdiv(L.im, 64), L.jm), 64, 0, s, L, P, rat, ctx->ratdim, c.ifix - 1, c.jfix - 1, lfix, pfix));
  CKL();
  LAUNCH(KC_PFIX, 0, L.N, launch_k(k_pfix_sub<T, W>, cdiv(L.N, 256), 256, 0, s, L, (const T*)ctx->pfix));
  CKL();
  return 0;
}

template <class TF, class WF, class TC, class WC>
int launch_nlevel(desalm_ctx* ctx, Lv<TF, WF>& F, Lv<TC, WC>& C) {
  const desalm_case& c = ctx->c;
  LAUNCH(KC_NLEVEL, 0, double(C.N), launch_k(k_nlevel<TF, WF, TC, WC>, dim3(cdiv(C.im, 32), cdiv(C.jm, 4), C.km), dim3(32, 4, 1), 0, ctx->stream, F, C, c.icrs, c.jcrs, c.kcrs));
  CKL();
  return 0;
}

// One direction of rsmooth as k_rsmooth4 with the widest slab that leaves
// room for two CTAs per SM.
template <class WF>
size_t rs_slab_bytes(int n, int nl) { return (size_t)4 * slab_fs(n, nl + 1) * sizeof(WF); }
template <class TF, class WF, int DIR, int NL>
int rsmooth_nl(desalm_ctx* ctx, Lv<TF, WF>& F, WF* dq, Level& G, double e, int last, double nin) {
  const int amax = DIR == 0 ? F.jm - 2 : F.im - 2;
  const int n = DIR == 0 ? F.im - 2 : (DIR == 1 ? F.jm - 2 : F.km - 2);
  const int nb = DIR == 2 ? F.jm - 2 : F.km - 2;
  LAUNCH(KC_RSMOOTH, 0, nin, launch_k(k_rsmooth4<TF, WF, DIR, NL>, dim3(cdiv(amax, NL), nb), kSlabThreads, rs_slab_bytes<WF>(n, NL), ctx->stream, 
                                 F, dq, G.fac[DIR], G.dpr[DIR], e, last));
  CKL();
  return 0;
}
template <class TF, class WF, int DIR>
int rsmooth(desalm_ctx* ctx, Lv<TF, WF>& F, WF* dq, Level& G, double e, int last, double nin) {
  const int n = DIR == 0 ? F.im - 2 : (DIR == 1 ? F.jm - 2 : F.km - 2);
  if (rs_slab_bytes<WF>(n, 16) <= kSlabTwoPerSm) return rsmooth_nl<TF, WF, DIR, 16>(ctx, F, dq, G, e, last, nin);
  if (rs_slab_bytes<WF>(n, 8) <= kSlabTwoPerSm) return rsmooth_nl<TF, WF, DIR, 8>(ctx, F, dq, G, e, last, nin);
  if (rs_slab_bytes<WF>(n, 4) <= kSlabMax) return rsmooth_nl<TF, WF, DIR, 4>(ctx, F, dq, G, e, last, nin);
  ctx->err = "grid line too long for the shared-memory rsmooth";
  return DESALM_EINVAL;
}

template <class TF, class WF, class TC, class WC>
int launch_prolong(desalm_ctx* ctx, Lv<TF, WF>& F, Lv<TC, WC>& C, Level& G) {
  const desalm_case& c = ctx->c;
  cudaStream_t s = ctx->stream;
  WF* dq = (WF*)G.dq[0];  // the prolongation correction, in the sweep precision
  const double nin = double(F.im - 2) * (F.jm - 2) * (F.km - 2);
  LAUNCH(KC_PROLONG, 0, nin, launch_k(k_prolong_interp<TF, WF, TC, WC>, grid_interior(F), blk3(), 0, s, F, C, dq, c.icrs, c.jcrs, c.kcrs));
  CKL();
  RET((rsmooth<TF, WF, 0>(ctx, F, dq, G, c.ep[1][0], 0, nin)));
  RET((rsmooth<TF, WF, 1>(ctx, F, dq, G, c.ep[1][1], 0, nin)));
  RET((rsmooth<TF, WF, 2>(ctx, F, dq, G, c.ep[1][2], 1, nin)));
  return 0;
}

template <class T, class W>
int launch_norm(desalm_ctx* ctx, Lv<T, W>& L, int copy, double* out) {
  cudaStream_t s = ctx->stream;
  long total = (long)(L.im - 2) * (L.jm - 2) * (L.km - 2);
  int nb = (int)std::min<long>(ctx->part_blocks, std::max<long>(1, cdiv(total, 256)));
  LAUNCH(KC_NORM, 0, double(total), launch_k(k_norm_partial<T, W>, nb, 256, 0, s, L, ctx->part, 5, copy));
  CKL();
  LAUNCH(KC_NORM, 0, 0, launch_k(k_norm_final, 1, 256, 0, s, ctx->part, nb, ctx->norm));
  CKL();
  CK(cudaMemcpyAsync(ctx->h_norm, ctx->norm, 5 * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  double tnu = double((long)(L.im - 2) * (L.jm - 2) * (L.km - 2));
  for (int m = 0; m < 5; ++m) out[m] = std::log10(ctx->h_norm[m] / tnu);
  return 0;
}

// dispatch on the active view of a level ------------------------------------
// FP64 mode: FP64 state and sweeps on every level.  MIXED: FP64 state on
// every level (residual, metrics, update, restriction, coarse corrections
// q_c - qold_c, which FP32 storage would lose to cancellation) and FP32
// line-sweep work (LHS coefficients, eliminated rows, transformed residual).
enum Kind { K_DD, K_DF };
Kind kind_of(const desalm_ctx* ctx, int n) {
  (void)n;
  if (ctx->c.precision_mode == DESALM_FP64) return K_DD;
  return K_DF;
}

#define DISPATCH(ctx, n, FN, ...)                                   \
  ([&]() -> int {                                                   \
    Level& G__ = (ctx)->L[n];                                       \
    switch (kind_of(ctx, n)) {                                      \
      case K_DD: return FN((ctx), G__.dd, ##__VA_ARGS__);           \
      default: return FN((ctx), G__.df, ##__VA_ARGS__);             \
    }                                                               \
  }())

int do_daf(desalm_ctx* ctx, int n, int recalc, int itr) {
  Level& G = ctx->L[n];
  int rc;
  switch (kind_of(ctx, n)) {
    case K_DD: rc = launch_daf(ctx, G.dd, G, n, recalc, itr); break;
    default: rc = launch_daf(ctx, G.df, G, n, recalc, itr); break;
  }
  if (rc) return rc;
  if (n == 0) {
    // bcond_fm inside solver_daf (src/solver_daf.F90:421)
    rc = kind_of(ctx, 0) == K_DD ? launch_bcond(ctx, G.dd) : launch_bcond(ctx, G.df);
    if (rc) return rc;
  }
  if (recalc == 1) {
    switch (kind_of(ctx, n)) {
      case K_DD: rc = launch_recalc(ctx, G.dd, n); break;
      default: rc = launch_recalc(ctx, G.df, n); break;
    }
  }
  return rc;
}

int do_bcond(desalm_ctx* ctx) {
  Level& G = ctx->L[0];
  return kind_of(ctx, 0) == K_DD ? launch_bcond(ctx, G.dd) : launch_bcond(ctx, G.df);
}

// wf_eta(1) and wf_eta(2) on the fine level (src/mg_driver.F90:221-224)
template <class T, class W>
int launch_wallfn(desalm_ctx* ctx, Lv<T, W>& L) {
  Par P = ctx->par;
  P.fine = 1;
  LAUNCH(KC_WALLFN, 0, 2.0 * (L.im - 2) * (L.km - 2),
         launch_k(k_wallfn<T, W>, dim3(cdiv(L.im - 2, 32), cdiv(L.km - 2, 4), 2), dim3(32, 4), 0, ctx->stream, L, P,
                  (const double*)ctx->x, (const double*)ctx->y, (const double*)ctx->z, (const double*)ctx->wd));
  CKL();
  return 0;
}
int do_wallfn(desalm_ctx* ctx) {
  Level& G = ctx->L[0];
  return kind_of(ctx, 0) == K_DD ? launch_wallfn(ctx, G.dd) : launch_wallfn(ctx, G.df);
}

// ------------------------------------------------------------ autotuning
// The DAF sweeps of one level and direction timed at 16, 8 and 4 lines per
// CTA (each width whose slab fits): one warm-up launch, then five timed with
// CUDA events on the context's stream; the fastest width is kept.  Wide
// slabs copy longer contiguous runs; narrow ones give short coarse-level
// planes enough CTAs to fill the SMs.  Only the sweep runs (its transform,
// which for k updates q, does not): it solves the work arrays in place, and
// those are rewritten by k_resid before every use, so timing them changes
// no result.
template <class T, class W, int DIR>
int tune_sweep(desalm_ctx* ctx, Lv<T, W>& L, int lvl, cudaEvent_t e0, cudaEvent_t e1) {
  Par P = ctx->par;
  P.fine = (lvl == 0);
  const int n = DIR == 0 ? L.im - 2 : (DIR == 1 ? L.jm - 2 : L.km - 2);
  // short lines always take the cyclic reduction (a different elimination
  // order, so it is not one of the timed choices, which all give the same bits)
  if (sweep_rows<T, W, DIR>(L) <= kPcrRows) {
    ctx->sweep_nl[lvl][DIR] = 2;
    return 0;
  }
  float best = 0.f;
  int pick = 0;
  for (int nl : {1, 16, 8, 4}) {
    const size_t bytes = slab_bytes<W>(n, nl);
    if (nl != 1 && bytes > kSlabMax) continue;
    ctx->sweep_nl[lvl][DIR] = nl;
    RET((launch_sweep<T, W, DIR>(ctx, L, P, lvl, 0, 0, false)));
    CK(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < 5; ++r) RET((launch_sweep<T, W, DIR>(ctx, L, P, lvl, 0, 0, false)));
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (!pick || ms < best) { best = ms; pick = nl; }
  }
  ctx->sweep_nl[lvl][DIR] = pick;
  return 0;
}

template <class T, class W>
int tune_level(desalm_ctx* ctx, Lv<T, W>& L, int lvl, cudaEvent_t e0, cudaEvent_t e1) {
  RET((tune_sweep<T, W, 0>(ctx, L, lvl, e0, e1)));
  RET((tune_sweep<T, W, 1>(ctx, L, lvl, e0, e1)));
  return tune_sweep<T, W, 2>(ctx, L, lvl, e0, e1);
}

template <class SW, class W> SaT<SW> make_sa(desalm_ctx* ctx, Lv<double, W>& L);
template <class W> KwT<W> make_kw(desalm_ctx* ctx, Lv<double, W>& L);

// CTA tiles of 128 threads the residual kernels are timed with
// the last is the face-shared K_R tile (k_resid_f), tried for kernels 0 and 1 only
constexpr unsigned kTiles[9][3] = {{32, 4, 1}, {32, 2, 2}, {32, 1, 4}, {64, 2, 1}, {64, 1, 2}, {128, 1, 1}, {16, 8, 1}, {16, 4, 2},
                                   {KRF_TX, KRF_TY, KRF_TZ}};

// Times one residual kernel (which: 0 = K_R, 1 = recalculation, 2 =
// turbulence residual) on level lvl at every tile and keeps the fastest.
// The kernels run on the level's current arrays; what they write (the line
// sweeps' inputs, rh, the turbulence ADI rows) is rewritten before any use,
// and the FAS forcing pk is left alone (no pk update is asked for).
template <class T, class W>
int tune_tile(desalm_ctx* ctx, Lv<T, W>& L, int lvl, int which, cudaEvent_t e0, cudaEvent_t e1) {
  Par P = ctx->par;
  P.fine = (lvl == 0);
  cudaStream_t s = ctx->stream;
  auto run = [&]() -> cudaError_t {
    const dim3 g = grid_t(ctx, lvl, which, L.im, L.jm, L.km), b = blk_t(ctx, lvl, which);
    if (which == 0) return launch_resid<T, W, 0>(ctx, lvl, s, L, P, lvl > 0 ? 1 : 0, 0, lvl > 0 ? 1 : 0, 0);
    if (which == 1) return launch_resid<T, W, 1>(ctx, lvl, s, L, P, lvl == 0 ? 2 : 1, 0, lvl > 0 ? 1 : 0, 0);
    if constexpr (std::is_same<T, double>::value) return launch_k(k_sa_rhs<W>, g, b, 0, s, make_sa<W>(ctx, L));
    return cudaSuccess;
  };
  float best = 0.f;
  int pick = -1;
  for (int t = 0; t < (which < 2 ? 9 : 8); ++t) {
    for (int d = 0; d < 3; ++d) ctx->tile[lvl][which][d] = kTiles[t][d];
    CK(run());
    CK(cudaEventRecord(e0, s));
    for (int r = 0; r < 3; ++r) CK(run());
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (pick < 0 || ms < best) { best = ms; pick = t; }
  }
  for (int d = 0; d < 3; ++d) ctx->tile[lvl][which][d] = kTiles[pick][d];
  return 0;
}

template <class T, class W>
int tune_tiles_level(desalm_ctx* ctx, Lv<T, W>& L, int lvl, cudaEvent_t e0, cudaEvent_t e1) {
  RET((tune_tile<T, W>(ctx, L, lvl, 0, e0, e1)));
  RET((tune_tile<T, W>(ctx, L, lvl, 1, e0, e1)));
  // the SA residual's tile (k-omega's residual has its own fixed tile, KWF_*)
  if (lvl == 0 && ctx->c.turbulence == 1) RET((tune_tile<T, W>(ctx, L, lvl, 2, e0, e1)));
  return 0;
}

// Picks the sweep widths and the residual kernels' tiles of every level,
// unless DESALM_AUTOTUNE=0 in the environment (then the shared-memory rule
// and the build's default tile decide).
int tune_sa_fine(desalm_ctx* ctx, cudaEvent_t e0, cudaEvent_t e1);

int autotune_sweeps(desalm_ctx* ctx) {
  for (int d = 0; d < 3; ++d) ctx->sa_nl[d] = 0;
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) {
      ctx->sweep_nl[n][d] = 0;
      for (int w = 0; w < 3; ++w) {
        ctx->tile[n][w][0] = 32; ctx->tile[n][w][1] = DESALM_KR_BY; ctx->tile[n][w][2] = DESALM_KR_BZ;
      }
    }
  const char* env = std::getenv("DESALM_AUTOTUNE");
  if (env && std::string(env) == "0") return 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    ctx->err = std::string("cudaEventCreate: ") + cudaGetErrorString(ce);
    return DESALM_ECUDA;
  }
  int rc = 0;
  for (int n = 0; n < ctx->ng && n < 4 && !rc; ++n) {
    Level& G = ctx->L[n];
    rc = kind_of(ctx, n) == K_DD ? tune_level(ctx, G.dd, n, e0, e1) : tune_level(ctx, G.df, n, e0, e1);
    if (!rc) rc = kind_of(ctx, n) == K_DD ? tune_tiles_level(ctx, G.dd, n, e0, e1) : tune_tiles_level(ctx, G.df, n, e0, e1);
  }
  if (!rc) rc = tune_sa_fine(ctx, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

int do_nlevel(desalm_ctx* ctx, int n) {  // n = coarse level index (>= 1)
  Level& F = ctx->L[n - 1];
  Level& C = ctx->L[n];
  C.dtau_valid = false;
  if (kind_of(ctx, n - 1) == K_DD) return launch_nlevel(ctx, F.dd, C.dd);
  return launch_nlevel(ctx, F.df, C.df);
}

int do_prolong(desalm_ctx* ctx, int n) {  // fine level index n, coarse n+1
  Level& F = ctx->L[n];
  Level& C = ctx->L[n + 1];
  if (kind_of(ctx, n) == K_DD) return launch_prolong(ctx, F.dd, C.dd, F);
  return launch_prolong(ctx, F.df, C.df, F);
}

int do_norm(desalm_ctx* ctx, int n, int copy, double* out) {
  Level& G = ctx->L[n];
  switch (kind_of(ctx, n)) {
    case K_DD: return launch_norm(ctx, G.dd, copy, out);
    default: return launch_norm(ctx, G.df, copy, out);
  }
}

// 1/aj of level n, after aj has been set
int refresh_rj(desalm_ctx* ctx, int n) {
  Level& G = ctx->L[n];
  cudaStream_t s = ctx->stream;
  if (kind_of(ctx, n) == K_DD) launch_k(k_recip<double>, cdiv(G.N, 256), 256, 0, s, (double*)G.dd.rj, G.dd.aj, G.N);
  else launch_k(k_recip<double>, cdiv(G.N, 256), 256, 0, s, (double*)G.df.rj, G.df.aj, G.N);
  CKL();
  return 0;
}

// What depends on a level's metrics alone: the metric parts of dtau
// (k_dtau_pre), and the FP32 copies of a MIXED level's metrics that the
// sweeps' modal transforms read (the same rounding the transforms applied to
// the FP64 metrics before, so their results do not change).
int refresh_mw(desalm_ctx* ctx, int n) {
  Level& G = ctx->L[n];
  Par P = ctx->par;
  if (kind_of(ctx, n) == K_DD) launch_k(k_dtau_pre<double, double>, cdiv(G.N, 256), 256, 0, ctx->stream, G.dd, P);
  else launch_k(k_dtau_pre<double, float>, cdiv(G.N, 256), 256, 0, ctx->stream, G.df, P);
  CKL();
  if (kind_of(ctx, n) == K_DD) return 0;
  Lv<double, float>& L = G.df;
  for (int t = 0; t < 9; ++t) {
    const double* m = t < 3 ? L.csi[t] : (t < 6 ? L.eta[t - 3] : L.zet[t - 6]);
    launch_k(k_copy<float, double>, cdiv(G.N, 256), 256, 0, ctx->stream, (float*)L.mw[t], m, G.N);
  }
  CKL();
  return 0;
}

// pointer to one SoA field of a level and its element size
int field_ptr(desalm_ctx* ctx, int n, int f, void** p, int* esz) {
  Level& G = ctx->L[n];
  Kind k = kind_of(ctx, n);
  *esz = 8;
  auto pick = [&](auto& L) -> int {
    if (f >= DESALM_F_Q && f < DESALM_F_Q + 5) { *p = L.q[f - DESALM_F_Q]; return 0; }
    if (f >= DESALM_F_QN && f < DESALM_F_QN + 5) { *p = L.qn[f - DESALM_F_QN]; return 0; }
    if (f >= DESALM_F_QNM1 && f < DESALM_F_QNM1 + 5) { *p = L.qnm1[f - DESALM_F_QNM1]; return 0; }
    if (f >= DESALM_F_QOLD && f < DESALM_F_QOLD + 5) { *p = L.qold[f - DESALM_F_QOLD]; return 0; }
    if (f >= DESALM_F_RH && f < DESALM_F_RH + 4) { *p = L.rh[f - DESALM_F_RH]; return 0; }
    if (f >= DESALM_F_PK && f < DESALM_F_PK + 4) { *p = L.pk[f - DESALM_F_PK]; return 0; }
    if (f >= DESALM_F_CSI && f < DESALM_F_CSI + 3) { *p = (void*)L.csi[f - DESALM_F_CSI]; return 0; }
    if (f >= DESALM_F_ETA && f < DESALM_F_ETA + 3) { *p = (void*)L.eta[f - DESALM_F_ETA]; return 0; }
    if (f >= DESALM_F_ZET && f < DESALM_F_ZET + 3) { *p = (void*)L.zet[f - DESALM_F_ZET]; return 0; }
    if (f == DESALM_F_AJ) { *p = (void*)L.aj; return 0; }
    if (f == DESALM_F_NUT) { *p = L.nut; return 0; }
    if (f == DESALM_F_DTAU) { *p = L.dtau; return 0; }
    if (n == 0 && f == DESALM_F_DTEV) { *p = ctx->dtev; *esz = 8; return 0; }
    if (n == 0 && f == DESALM_F_WD) { *p = ctx->wd; *esz = 8; return 0; }
    if (n == 0 && f == DESALM_F_X) { *p = ctx->x; *esz = 8; return 0; }
    if (n == 0 && f == DESALM_F_Y) { *p = ctx->y; *esz = 8; return 0; }
    if (n == 0 && f == DESALM_F_Z) { *p = ctx->z; *esz = 8; return 0; }
    ctx->err = "unknown field id for this level";
    return DESALM_EINVAL;
  };
  if (k == K_DD) return pick(G.dd);
  return pick(G.df);
}

// Inflow extrapolation ratios on the host from the fine grid
// (src/init.F90:2750-2891).  The k faces' guard in the reference
// ('btype == 4 .and. btype == 5') is never true, so rat(:,:,5:6) are never
// assigned there; they stay zero here.
void outlet_ratios(const desalm_case& c, const double* x, const double* y, const double* z, std::vector<double>& rat, int rd) {
  rat.assign((size_t)6 * rd * rd, 0.0);
  const int im = c.im, jm = c.jm, km = c.km;
  auto id = [&](int i, int j, int k) { return (long)(i - 1) + (long)im * ((j - 1) + (long)jm * (k - 1)); };
  for (int b = 0; b < 4; ++b) {
    if (!(c.btype[b] == 4 || c.btype[b] == 5)) continue;
    int dir = c.bdir[b];
    if (dir < 1 || dir > 3) continue;
    const double* v = dir == 1 ? x : (dir == 2 ? y : z);
    if (b < 2) {
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
          double r;
          if (b == 0) r = (v[id(2, j, k)] - v[id(1, j, k)]) / (v[id(3, j, k)] - v[id(2, j, k)]);
          else r = (v[id(im, j, k)] - v[id(im - 1, j, k)]) / (v[id(im - 1, j, k)] - v[id(im - 2, j, k)]);
          rat[(size_t)b * rd * rd + (j - 1) + (size_t)rd * (k - 1)] = r;
        }
    } else {
      for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) {
          double r;
          if (b == 2) r = (v[id(i, 2, k)] - v[id(i, 1, k)]) / (v[id(i, 3, k)] - v[id(i, 2, k)]);
          else r = (v[id(i, jm, k)] - v[id(i, jm - 1, k)]) / (v[id(i, jm - 1, k)] - v[id(i, jm - 2, k)]);
          rat[(size_t)b * rd * rd + (i - 1) + (size_t)rd * (k - 1)] = r;
        }
    }
  }
}

int pseudo_iter(desalm_ctx* ctx, desalm_step_report* rep);
int enqueue_iteration(desalm_ctx* ctx);
int rfg_launch(desalm_ctx* ctx, double time);
int graph_step(desalm_ctx* ctx, desalm_step_report* rep);
int graph_launch(desalm_ctx* ctx);
int graph_finish(desalm_ctx* ctx, desalm_step_report* rep);
void drop_graph(desalm_ctx* ctx);
int autotune_sweeps(desalm_ctx* ctx);
int run_step(desalm_ctx* ctx, desalm_step_report* rep);
int sa_des_eddy(desalm_ctx* ctx);
int kw_eddy_run(desalm_ctx* ctx);
int sa_conservation(desalm_ctx* ctx);


// ----------------------------------------------------------- learned guess
constexpr int kLpWgradGrid = 148;  // partial slots of k_lp_wgrad_tc (one CTA per SM)
constexpr int kLpRedBlocks = 296;  // CTAs (and partial rows) of the learned guess's reductions

// cuTensorMapEncodeTiled, reached through the runtime's driver entry point
typedef CUresult (*LpEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// TMA map of channel-last rows [np][C] (BF16): boxes of 8 channels x 130 rows,
// no swizzle, rows past the ends read as zero.
int lp_tmap(desalm_ctx* ctx, CUtensorMap* m, const bf16* rows, int C, long np) {
  static LpEncodeTiled enc = nullptr;
  if (!enc) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess) {
      ctx->err = "cuTensorMapEncodeTiled is not available";
      return DESALM_ECUDA;
    }
    enc = (LpEncodeTiled)fn;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)C, (cuuint64_t)np};
  const cuuint64_t strides[1] = {(cuuint64_t)C * sizeof(bf16)};
  const cuuint32_t box[2] = {8, (cuuint32_t)LP_WROWS};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)rows, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    ctx->err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return DESALM_ECUDA;
  }
  return 0;
}

// One convolution on the tensor cores (k_lp_conv_tc); map describes `in`.
template <int CIN, int COUT>
int lp_conv(desalm_ctx* ctx, const CUtensorMap& map, const bf16* w, const float* bias, int relu, const bf16* mask,
            bf16* out, float* out32, int cout32) {
  LpState& lp = ctx->lp;
  const long tiles = (lp.P.p1 - lp.P.p0 + LP_TM - 1) / LP_TM;
  const unsigned grid = (unsigned)std::min<long>(tiles, 148L * 2);
  LAUNCH(KC_LEARN, 0, (double)lp.N, launch_k(k_lp_conv_tc<CIN, COUT>, grid, LP_TC_THREADS, LpTcSmem<CIN, COUT>::total,
                                             lp.ls, map, lp.P, w, bias, relu, mask, out, out32, cout32, lp.err));
  CKL();
  return 0;
}

// The tensor-core kernels' error flag (read after a synchronisation): a wait
// that timed out leaves DESALM_ETIMEOUT and clears the flag.
int lp_check(desalm_ctx* ctx) {
  int e = 0;
  CK(cudaMemcpy(&e, ctx->lp.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(ctx->lp.err, 0, sizeof(int)));
    ctx->err = "learned guess: a tensor-core kernel gave up waiting for its copies or MMAs";
    return DESALM_ETIMEOUT;
  }
  return 0;
}

// Weight and bias gradient of one layer into dW ([27][CIN][COUT] then [COUT])
// on the tensor cores: per-CTA partials (k_lp_wgrad_tc, one CTA per SM),
// then their sum.  xmap describes X, dmap D.
template <int CIN, int COUT>
int lp_wgrad(desalm_ctx* ctx, const CUtensorMap& xmap, const CUtensorMap& dmap, float* dW) {
  LpState& lp = ctx->lp;
  constexpr long SLOT = 27L * CIN * COUT + COUT;
  constexpr int grid = 148;
  static_assert(grid <= kLpWgradGrid, "partial slots");
  LAUNCH(KC_LEARN, 0, (double)lp.N, launch_k(k_lp_wgrad_tc<CIN, COUT>, grid, LP_TC_THREADS, LpWgTc<CIN, COUT>::total,
                                             lp.ls, xmap, dmap, lp.P, lp.part, lp.err));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_reduce, cdiv(SLOT, 256), 256, 0, lp.ls, grid, SLOT,
                                    (const float*)lp.part, dW));
  CKL();
  return 0;
}

template <class K>
cudaError_t lp_optin(K* k, size_t bytes) {
  return cudaFuncSetAttribute((const void*)k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t lp_attrs() {
  cudaError_t e = lp_optin(k_lp_conv_tc<16, 32>, LpTcSmem<16, 32>::total);
  if (e == cudaSuccess) e = lp_optin(k_lp_conv_tc<32, 32>, LpTcSmem<32, 32>::total);
  if (e == cudaSuccess) e = lp_optin(k_lp_conv_tc<32, 16>, LpTcSmem<32, 16>::total);
  if (e == cudaSuccess) e = lp_optin(k_lp_wgrad_tc<16, 32>, LpWgTc<16, 32>::total);
  if (e == cudaSuccess) e = lp_optin(k_lp_wgrad_tc<32, 32>, LpWgTc<32, 32>::total);
  if (e == cudaSuccess) e = lp_optin(k_lp_wgrad_tc<32, 16>, LpWgTc<32, 16>::total);
  return e;
}

// Buffers and initial weights (He normal, seeded; the last layer scaled by
// 0.1 so that the first guesses stay close to the linear extrapolation).
int lp_alloc(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  const Level& F = ctx->L[0];
  lp.N = F.N;
  lp.P = lp_pad(F.im, F.jm, F.km);
  const int cin[4] = {15, 32, 32, 32}, cout[4] = {32, 32, 32, 5};
  const int cinp[4] = {16, 32, 32, 32}, coutp[4] = {32, 32, 32, 16};
  long off = 0;
  for (int l = 0; l < 4; ++l) {
    LpLayer& y = lp.ly[l];
    y.cin = cin[l]; y.cout = cout[l]; y.cin_pad = cinp[l]; y.cout_pad = coutp[l];
    y.woff = off; off += (long)y.cout * y.cin * 27;
    y.boff = off; off += y.cout;
  }
  lp.nparam = off;
  auto A = [&](void** p, size_t bytes) { return dalloc(ctx, ctx->allocs, p, bytes); };
  const long N = lp.N;
  RET(A((void**)&lp.theta, off * sizeof(float))); RET(A((void**)&lp.grad, off * sizeof(float)));
  RET(A((void**)&lp.m, off * sizeof(float))); RET(A((void**)&lp.v, off * sizeof(float)));
  for (int l = 0; l < 4; ++l) {
    const size_t wb = 27L * cinp[l] * coutp[l];
    RET(A((void**)&lp.wf[l], wb * sizeof(bf16))); RET(A((void**)&lp.wd[l], wb * sizeof(bf16)));
    RET(A((void**)&lp.dW[l], (wb + coutp[l]) * sizeof(float)));
    lp.db[l] = lp.dW[l] + wb;
  }
  RET(A((void**)&lp.part, (size_t)kLpWgradGrid * (27L * 32 * 32 + 32) * sizeof(float)));
  // channel-last rows of the padded grid; the halo rows stay zero
  const long NP = lp.P.np;
  RET(A((void**)&lp.x0, 16L * NP * sizeof(bf16)));
  RET(A((void**)&lp.x1, 16L * NP * sizeof(bf16)));
  for (int l = 0; l < 3; ++l) RET(A((void**)&lp.a[l], 32L * NP * sizeof(bf16)));
  RET(A((void**)&lp.dy4, 16L * NP * sizeof(bf16)));
  for (int l = 0; l < 2; ++l) RET(A((void**)&lp.dya[l], 32L * NP * sizeof(bf16)));
  RET(A((void**)&lp.err, sizeof(int)));
  RET(lp_tmap(ctx, &lp.tm_x0, lp.x0, 16, NP));
  RET(lp_tmap(ctx, &lp.tm_x1, lp.x1, 16, NP));
  CK(cudaStreamCreateWithFlags(&lp.tstream, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&lp.ev_pred, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&lp.ev_train, cudaEventDisableTiming));
  if (cudaMallocHost((void**)&lp.h_loss, 256 * sizeof(double)) != cudaSuccess) {
    ctx->err = "cudaMallocHost failed";
    return DESALM_ENOMEM;
  }
  lp.ls = ctx->stream;
  for (int l = 0; l < 3; ++l) RET(lp_tmap(ctx, &lp.tm_a[l], lp.a[l], 32, NP));
  RET(lp_tmap(ctx, &lp.tm_dy4, lp.dy4, 16, NP));
  for (int l = 0; l < 2; ++l) RET(lp_tmap(ctx, &lp.tm_dya[l], lp.dya[l], 32, NP));
  RET(A((void**)&lp.y, 5L * N * sizeof(float))); RET(A((void**)&lp.t, 5L * N * sizeof(float)));
  RET(A((void**)&lp.yt, 5L * N * sizeof(float)));
  RET(A((void**)&lp.rs, 16 * sizeof(float))); RET(A((void**)&lp.rs5, 8 * sizeof(float)));
  RET(A((void**)&lp.s5, 8 * sizeof(float))); RET(A((void**)&lp.acc, 16 * sizeof(double)));
  RET(A((void**)&lp.red, kLpRedBlocks * 16 * sizeof(double)));
  RET(A((void**)&lp.vacc, 16 * sizeof(double))); RET(A((void**)&lp.alpha, 8 * sizeof(float)));
  for (int f = 0; f < 5; ++f) RET(A((void**)&lp.qnm2[f], N * sizeof(double)));
  RET(A((void**)&lp.nut0, N * sizeof(double)));
  RET(A((void**)&lp.tab, 20 * sizeof(double*)));
  cudaStream_t s = ctx->stream;
  double* tab[20];
  int esz = 8;
  for (int f = 0; f < 5; ++f) {
    RET(field_ptr(ctx, 0, DESALM_F_Q + f, (void**)&tab[f], &esz));
    RET(field_ptr(ctx, 0, DESALM_F_QN + f, (void**)&tab[5 + f], &esz));
    RET(field_ptr(ctx, 0, DESALM_F_QNM1 + f, (void**)&tab[10 + f], &esz));
    tab[15 + f] = lp.qnm2[f];
  }
  for (int e = 0; e < 20; ++e) lp.tab_h[e] = tab[e];
  CK(cudaMemcpyAsync(lp.tab, tab, sizeof(tab), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(lp.m, 0, off * sizeof(float), s));
  CK(cudaMemsetAsync(lp.v, 0, off * sizeof(float), s));
  std::vector<float> th(off, 0.0f);
  std::mt19937 rng(20241203u);
  for (int l = 0; l < 4; ++l) {
    const LpLayer& y = lp.ly[l];
    std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (27.0f * y.cin)) * (l == 3 ? 0.1f : 1.0f));
    for (long e = 0; e < (long)y.cout * y.cin * 27; ++e) th[y.woff + e] = nd(rng);
  }
  CK(cudaMemcpyAsync(lp.theta, th.data(), off * sizeof(float), cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  lp.on = true;
  return 0;
}

int lp_pack(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  for (int l = 0; l < 4; ++l) {
    const long total = 27L * lp.ly[l].cin_pad * lp.ly[l].cout_pad;
    LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_pack_tc, cdiv(total, 256), 256, 0, lp.ls, lp.ly[l], (const float*)lp.theta, lp.wf[l], lp.wd[l]));
  }
  CKL();
  return 0;
}

// Forward pass on the features xin describes (lp.x0 or lp.x1): activations
// a[0..2], output yout (FP32: lp.y, or lp.yt for training).
int lp_forward(desalm_ctx* ctx, const CUtensorMap& xin, float* yout) {
  LpState& lp = ctx->lp;
  const float* b[4];
  for (int l = 0; l < 4; ++l) b[l] = lp.theta + lp.ly[l].boff;
  // the bias pointers index the flat vector: each layer's bias is contiguous there
  RET((lp_conv<16, 32>(ctx, xin, lp.wf[0], b[0], 1, nullptr, lp.a[0], nullptr, 0)));
  RET((lp_conv<32, 32>(ctx, lp.tm_a[0], lp.wf[1], b[1], 1, nullptr, lp.a[1], nullptr, 0)));
  RET((lp_conv<32, 32>(ctx, lp.tm_a[1], lp.wf[2], b[2], 1, nullptr, lp.a[2], nullptr, 0)));
  RET((lp_conv<32, 16>(ctx, lp.tm_a[2], lp.wf[3], b[3], 0, nullptr, nullptr, yout, 5)));
  return 0;
}

// Loss against lp.t and the gradient of the mean squared error in lp.grad
// for the features xin describes.  On the context's stream the loss goes to
// *loss (host, after a synchronize); on the training stream its sum goes to
// the pinned slot *hsum without waiting (read by lp_join).
int lp_backward(desalm_ctx* ctx, const CUtensorMap& xin, const float* yin, double* loss, double* hsum = nullptr) {
  LpState& lp = ctx->lp;
  cudaStream_t s = lp.ls;
  const long N = lp.N;
  LAUNCH(KC_LEARN, 0, (double)N, launch_k(k_lp_loss, kLpRedBlocks, 256, 0, s, lp.P, yin, (const float*)lp.t, lp.dy4, lp.red));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_fold, 1, 32, 0, s, (const double*)lp.red, kLpRedBlocks, 1, lp.acc));
  CKL();
  // layer 4 (a[2] -> y)
  RET((lp_wgrad<32, 16>(ctx, lp.tm_a[2], lp.tm_dy4, lp.dW[3])));
  RET((lp_conv<16, 32>(ctx, lp.tm_dy4, lp.wd[3], nullptr, 0, lp.a[2], lp.dya[0], nullptr, 0)));
  // layer 3 (a[1] -> a[2])
  RET((lp_wgrad<32, 32>(ctx, lp.tm_a[1], lp.tm_dya[0], lp.dW[2])));
  RET((lp_conv<32, 32>(ctx, lp.tm_dya[0], lp.wd[2], nullptr, 0, lp.a[1], lp.dya[1], nullptr, 0)));
  // layer 2 (a[0] -> a[1])
  RET((lp_wgrad<32, 32>(ctx, lp.tm_a[0], lp.tm_dya[1], lp.dW[1])));
  RET((lp_conv<32, 32>(ctx, lp.tm_dya[1], lp.wd[1], nullptr, 0, lp.a[0], lp.dya[0], nullptr, 0)));
  // layer 1 (x0 -> a[0])
  RET((lp_wgrad<16, 32>(ctx, xin, lp.tm_dya[0], lp.dW[0])));
  const float gscale = float(2.0 / (5.0 * double(N)));
  for (int l = 0; l < 4; ++l) {
    const long n = (long)lp.ly[l].cout * lp.ly[l].cin * 27 + lp.ly[l].cout;
    LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_gather_grad, cdiv(n, 256), 256, 0, s, lp.ly[l], (const float*)lp.dW[l],
                                      (const float*)lp.db[l], gscale, lp.grad));
  }
  CKL();
  if (hsum) {
    CK(cudaMemcpyAsync(hsum, lp.acc, sizeof(double), cudaMemcpyDeviceToHost, s));
    return 0;
  }
  double sum = 0;
  CK(cudaMemcpyAsync(&sum, lp.acc, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  RET(lp_check(ctx));
  if (loss) *loss = sum / (5.0 * double(N));
  return 0;
}

// Features of (qn, qnm1, qnm2) at table offsets (a, b, c) into x (lp.x0 or
// lp.x1), with the scales of these three levels (computed on the device).
int lp_features(desalm_ctx* ctx, int a, int b, int c, bf16* x) {
  LpState& lp = ctx->lp;
  cudaStream_t s = ctx->stream;
  const long N = lp.N;
  const double* const* A = (const double* const*)(lp.tab + a);
  const double* const* B = (const double* const*)(lp.tab + b);
  const double* const* C = (const double* const*)(lp.tab + c);
  LAUNCH(KC_LEARN, 0, (double)N, launch_k(k_lp_sumsq, kLpRedBlocks, 128, 0, s, N, A, B, C, lp.red));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_fold, 1, 32, 0, s, (const double*)lp.red, kLpRedBlocks, 15, lp.acc));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_scales, 1, 32, 0, s, N, (const double*)lp.acc, lp.rs, lp.rs5, lp.s5));
  LAUNCH(KC_LEARN, 0, (double)N, launch_k(k_lp_features, cdiv(N, 256), 256, 0, s, lp.P, A, B, C, (const float*)lp.rs, x));
  CKL();
  return 0;
}

// One Adam step on the sample whose features xin describes and target lp.t
// (on lp.ls); hsum: see lp_backward.
int lp_train_step(desalm_ctx* ctx, const CUtensorMap& xin, double* loss, double* hsum = nullptr) {
  LpState& lp = ctx->lp;
  RET(lp_pack(ctx));
  RET(lp_forward(ctx, xin, lp.yt));
  RET(lp_backward(ctx, xin, lp.yt, loss, hsum));
  lp.adam_t += 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = float(1.0 / (1.0 - std::pow(double(b1), double(lp.adam_t))));
  const float c2 = float(1.0 / (1.0 - std::pow(double(b2), double(lp.adam_t))));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_adam, cdiv(lp.nparam, 256), 256, 0, lp.ls, lp.nparam, lp.theta,
                                    (const float*)lp.grad, lp.m, lp.v, lp.lr, b1, b2, 1e-8f, c1, c2));
  CKL();
  lp.steps += 1;
  return 0;
}

// At the start of a physical step, before the history shift: the newest
// converged level q is the target of a sample whose features come from
// (qn, qnm1, qnm2); train on it.
int lp_learn(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  if (lp.shifts < 1) return 0;  // q^{n-2} not known yet
  RET(lp_features(ctx, 5, 10, 15, lp.x1));
  LAUNCH(KC_LEARN, 0, (double)lp.N, launch_k(k_lp_target, cdiv(lp.N, 256), 256, 0, ctx->stream, lp.N,
                                             (const double* const*)(lp.tab + 0), (const double* const*)(lp.tab + 5),
                                             (const double* const*)(lp.tab + 10), (const float*)lp.rs5, lp.t));
  CKL();
  // held-out check: the current network on the new sample, before training on it
  RET(lp_pack(ctx));
  RET(lp_forward(ctx, lp.tm_x1, lp.y));
  LAUNCH(KC_LEARN, 0, (double)lp.N, launch_k(k_lp_dot, kLpRedBlocks, 128, 0, ctx->stream, lp.N, (const float*)lp.y,
                                             (const float*)lp.t, lp.ymax, lp.red));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_fold, 1, 32, 0, ctx->stream, (const double*)lp.red, kLpRedBlocks, 15, lp.vacc));
  LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_blend, 1, 32, 0, ctx->stream, (const double*)lp.vacc, lp.fixed_alpha, lp.field_mask, lp.alpha));
  CKL();
  lp.samples += 1;
  if (!ctx->prof_on) {  // trained after the prediction, beside the step (lp_train_launch)
    lp.pending = true;
    return 0;
  }
  for (int it = 0; it < lp.train_steps; ++it) {  // profiling: in line, on the context's stream
    double loss = 0;
    RET(lp_train_step(ctx, lp.tm_x1, &loss));
    if (lp.first_loss < 0) lp.first_loss = loss;
    lp.last_loss = loss;
  }
  return 0;
}

// The pending Adam steps on the training stream, after everything the
// context's stream has queued (the prediction's forward pass included).
int lp_train_launch(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  if (!lp.pending) return 0;
  lp.pending = false;
  CK(cudaEventRecord(lp.ev_pred, ctx->stream));
  CK(cudaStreamWaitEvent(lp.tstream, lp.ev_pred, 0));
  lp.ls = lp.tstream;
  const int n = std::min(lp.train_steps, 256);
  int rc = 0;
  for (int it = 0; it < n && !rc; ++it) rc = lp_train_step(ctx, lp.tm_x1, nullptr, lp.h_loss + it);
  lp.ls = ctx->stream;
  RET(rc);
  CK(cudaEventRecord(lp.ev_train, lp.tstream));
  lp.h_loss_n = n;
  lp.inflight = true;
  return 0;
}

// Wait for the training in flight: the context's stream waits for it, and
// its losses and error flag are read.
int lp_join(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  if (!lp.inflight) return 0;
  lp.inflight = false;
  CK(cudaStreamWaitEvent(ctx->stream, lp.ev_train, 0));
  CK(cudaEventSynchronize(lp.ev_train));
  const double scale = 1.0 / (5.0 * double(lp.N));
  for (int it = 0; it < lp.h_loss_n; ++it) {
    const double loss = lp.h_loss[it] * scale;
    if (lp.first_loss < 0) lp.first_loss = loss;
    lp.last_loss = loss;
  }
  return lp_check(ctx);
}

// After the shift and the linear extrapolation: q <- 2 q^n - q^{n-1} + the
// network's correction, once it has seen lp.warm samples (and, after a
// fallback, lp.warm more).
int lp_predict(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  lp.predicted = false;
  if (lp.samples < lp.warm || lp.samples < lp.hold_until || lp.shifts < 1) return 0;
  RET(lp_features(ctx, 5, 10, 15, lp.x0));
  RET(lp_pack(ctx));
  RET(lp_forward(ctx, lp.tm_x0, lp.y));
  if (lp.fixed_alpha >= 0.0f || lp.field_mask != 0x1f)
    LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_blend, 1, 32, 0, ctx->stream, (const double*)lp.vacc, lp.fixed_alpha, lp.field_mask, lp.alpha));
  LAUNCH(KC_LEARN, 0, (double)lp.N, launch_k(k_lp_apply, cdiv(lp.N, 256), 256, 0, ctx->stream, lp.N, lp.tab + 0,
                                             (const double* const*)(lp.tab + 5), (const double* const*)(lp.tab + 10),
                                             (const float*)lp.s5, (const float*)lp.alpha, (const float*)lp.y, lp.ymax));
  CKL();
  void* nut;
  int esz;
  RET(field_ptr(ctx, 0, DESALM_F_NUT, &nut, &esz));
  CK(cudaMemcpyAsync(lp.nut0, nut, lp.N * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  lp.predictions += 1;
  lp.predicted = true;
  return 0;
}

// A step begun from the network's guess that ended with a non-finite norm or
// a zero pivot starts again from the linear extrapolation: q and nu_t as the
// linear guess would have left them, then the rest of desalm_begin_step.
int lp_fallback(desalm_ctx* ctx) {
  LpState& lp = ctx->lp;
  cudaStream_t s = ctx->stream;
  const Level& F = ctx->L[0];
  for (int m = 0; m < 5; ++m)
    LAUNCH(KC_MISC, 0, F.N, launch_k(k_extrapolate<double>, cdiv(F.N, 256), 256, 0, s, lp.tab_h[m],
                                     (const double*)lp.tab_h[5 + m], (const double*)lp.tab_h[10 + m], F.N));
  if (ctx->c.turbulence == 2)
    LAUNCH(KC_MISC, 0, F.N, launch_k(k_extrapolate<double>, cdiv(F.N, 256), 256, 0, s, ctx->kw.a[0],
                                     (const double*)ctx->kw.a[1], (const double*)ctx->kw.a[2], F.N));
  CKL();
  void* nut;
  int esz;
  RET(field_ptr(ctx, 0, DESALM_F_NUT, &nut, &esz));
  CK(cudaMemcpyAsync(nut, lp.nut0, lp.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
  if (ctx->c.conservation) RET(sa_conservation(ctx));
  for (auto& L : ctx->L) L.dtau_valid = false;
  lp.fallbacks += 1;
  lp.predicted = false;
  lp.hold_until = lp.samples + std::max(1, lp.warm);
  return 0;
}

}  // namespace

// =============================================================== C ABI
extern "C" {

const char* desalm_last_error(const desalm_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void desalm_destroy(desalm_ctx* ctx) {
  if (!ctx) return;
  if (ctx->lp.tstream) cudaStreamSynchronize(ctx->lp.tstream);  // training in flight
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& G : ctx->L)
    for (void* p : G.allocs) cudaFree(p);
  for (void* p : ctx->allocs) cudaFree(p);
  for (void* p : ctx->alm.allocs) cudaFree(p);
  for (void* p : ctx->rfg.allocs) cudaFree(p);
  for (auto& r : ctx->prof) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  if (ctx->hconv) cudaFreeHost(ctx->hconv);
  if (ctx->h_norm) cudaFreeHost(ctx->h_norm);
  if (ctx->side) cudaStreamSynchronize(ctx->side);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->lp.tstream) cudaStreamDestroy(ctx->lp.tstream);
  if (ctx->lp.ev_pred) cudaEventDestroy(ctx->lp.ev_pred);
  if (ctx->lp.ev_train) cudaEventDestroy(ctx->lp.ev_train);
  if (ctx->lp.h_loss) cudaFreeHost(ctx->lp.h_loss);
  delete ctx;
}

int desalm_init(const desalm_case* c, desalm_ctx** out) {
  if (!c || !out) return DESALM_EINVAL;
  *out = nullptr;
  desalm_ctx* ctx = new desalm_ctx();
  int rc = check_case(ctx, *c);
  if (rc) {
    // keep the message reachable: return the context so desalm_last_error works
    *out = ctx;
    return rc;
  }
  ctx->c = *c;
  ctx->ng = c->ng;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    ctx->err = std::string("no CUDA device: ") + cudaGetErrorString(e);
    *out = ctx;
    return DESALM_ECUDA;
  }
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    ctx->err = std::string("cudaStreamCreate: ") + cudaGetErrorString(e);
    *out = ctx;
    return DESALM_ECUDA;
  }
  fill_par(ctx);
  ctx->L.resize(ctx->ng);
  ctx->L[0].im = c->im; ctx->L[0].jm = c->jm; ctx->L[0].km = c->km;
  for (int n = 1; n < ctx->ng; ++n) {
    ctx->L[n].im = (ctx->L[n - 1].im + c->icrs) >> c->icrs;
    ctx->L[n].jm = (ctx->L[n - 1].jm + c->jcrs) >> c->jcrs;
    ctx->L[n].km = (ctx->L[n - 1].km + c->kcrs) >> c->kcrs;
  }
  rc = dalloc(ctx, ctx->allocs, (void**)&ctx->flags, 3 * sizeof(int));
  if (rc) { *out = ctx; return rc; }
  {
    // rows x lines of the longest sweep, the lines of a plane padded to a
    // multiple of 32 (each warp's row is whole 128-byte lines); the coarse
    // levels and the turbulence sweeps need less
    auto rup = [](long v) { return (v + 31) / 32 * 32; };
    const long e = c->btype[1] == 5 ? 1 : 0;   // the outlet row and line of the fine level
    const long im2 = c->im - 2, jm2 = c->jm - 2, km2 = c->km - 2;
    const long g = std::max((im2 + e) * rup(jm2) * km2, std::max(jm2 * rup(im2 + e) * km2, km2 * rup(im2 + e) * jm2));
    const size_t wb = c->precision_mode == DESALM_FP64 ? 8 : 4;
    ctx->gss = (int)rup(g);
    rc = dalloc(ctx, ctx->allocs, &ctx->gsweep, 16 * (size_t)ctx->gss * wb);
    if (rc) { *out = ctx; return rc; }
  }
  for (int n = 0; n < ctx->ng; ++n) {
    Level& G = ctx->L[n];
    G.N = (long)G.im * G.jm * G.km;
    G.dc = 1.0 / std::pow(2.0, double(n * c->icrs));
    G.de = 1.0 / std::pow(2.0, double(n * c->jcrs));
    G.dz = 1.0 / std::pow(2.0, double(n * c->kcrs));
    Kind k = kind_of(ctx, n);
    if (k == K_DD) rc = alloc_level(ctx, G, G.dd);
    else rc = alloc_level(ctx, G, G.df);
    if (rc) { *out = ctx; return rc; }
    // the characteristics outlet plane is solved on the fine level only
    // (src/solver_daf.F90:371-373)
    G.dd.oute = G.df.oute = (n == 0 && c->btype[1] == 5) ? 1 : 0;
    G.tbytes = 8;
    G.wbytes = k == K_DD ? 8 : 4;
    if (n + 1 < ctx->ng) {
      rc = dalloc(ctx, G.allocs, &G.dq[0], (size_t)4 * G.N * G.wbytes);
      if (rc) { *out = ctx; return rc; }
      const int ext[3] = {G.im, G.jm, G.km};
      for (int d = 0; d < 3; ++d) {
        std::vector<double> fac, dpr;
        rs_factors(ext[d] - 2, c->ep[1][d], fac, dpr);
        const size_t nd = dpr.size();
        dpr.resize(2 * nd);
        for (size_t p = 0; p < nd; ++p) dpr[nd + p] = 1.0 / dpr[p];
        rc = dalloc(ctx, G.allocs, (void**)&G.fac[d], fac.size() * sizeof(double));
        if (!rc) rc = dalloc(ctx, G.allocs, (void**)&G.dpr[d], dpr.size() * sizeof(double));
        if (rc) { *out = ctx; return rc; }
        cudaMemcpyAsync(G.fac[d], fac.data(), fac.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
        cudaMemcpyAsync(G.dpr[d], dpr.data(), dpr.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
      }
    }
  }
  const long NF = ctx->L[0].N;
  auto A = [&](double** p, long n) { return dalloc(ctx, ctx->allocs, (void**)p, n * sizeof(double)); };
  rc = A(&ctx->x, NF); if (!rc) rc = A(&ctx->y, NF); if (!rc) rc = A(&ctx->z, NF);
  if (!rc) rc = A(&ctx->wd, NF);
  if (!rc) rc = A(&ctx->dtev, NF);
  for (int t = 0; t < 9 && !rc; ++t) rc = A(&ctx->cov[t], NF);
  if (!rc) rc = dalloc(ctx, ctx->allocs, (void**)&ctx->dcov, 9 * sizeof(double*));
  if (!rc) cudaMemcpyAsync(ctx->dcov, ctx->cov, 9 * sizeof(double*), cudaMemcpyHostToDevice, ctx->stream);
  ctx->ratdim = std::max(c->im, std::max(c->jm, c->km));
  if (!rc) rc = A(&ctx->rat, 6L * ctx->ratdim * ctx->ratdim);
  if (!rc) rc = A(&ctx->pfix, 1);
  ctx->part_blocks = 148 * 8;
  if (!rc) rc = A(&ctx->part, 5L * ctx->part_blocks);
  if (!rc) rc = A(&ctx->norm, 5);
  if (!rc && c->turbulence)
    for (int t = 0; t < SaWork::NARR && !rc; ++t) rc = A(&ctx->sa.a[t], NF);
  if (!rc && c->turbulence == 2)
    for (int t = 0; t < KwWork::NARR && !rc; ++t) rc = A(&ctx->kw.a[t], NF);
  if (rc) { *out = ctx; return rc; }
  if (cudaMallocHost((void**)&ctx->h_norm, 5 * sizeof(double)) != cudaSuccess) {
    ctx->err = "cudaMallocHost failed";
    *out = ctx;
    return DESALM_ENOMEM;
  }
  // state transfers: one staging array and the fine level's field table
  rc = A(&ctx->stage, 5 * NF);
  if (!rc) rc = dalloc(ctx, ctx->allocs, (void**)&ctx->ftab, 15 * sizeof(double*));
  if (rc) { *out = ctx; return rc; }
  {
    double* tab[15];
    const int fb[3] = {DESALM_F_Q, DESALM_F_QN, DESALM_F_QNM1};
    int esz = 8;
    for (int a = 0; a < 3; ++a)
      for (int m = 0; m < 5; ++m) field_ptr(ctx, 0, fb[a] + m, (void**)&tab[5 * a + m], &esz);
    cudaMemcpyAsync(ctx->ftab, tab, sizeof(tab), cudaMemcpyHostToDevice, ctx->stream);
  }
  e = kind_of(ctx, 0) == K_DD ? slab_attrs<double, double>() : slab_attrs<double, float>();
  if (e == cudaSuccess && c->predictor == DESALM_PRED_LEARNED) e = lp_attrs();
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    ctx->err = std::string("init: ") + cudaGetErrorString(e);
    *out = ctx;
    return DESALM_ECUDA;
  }
  *out = ctx;
  if (c->predictor == DESALM_PRED_LEARNED) return lp_alloc(ctx);
  return 0;
}

int desalm_level_dims(const desalm_ctx* ctx, int n, int dims[3]) {
  if (!ctx || n < 1 || n > ctx->ng) return DESALM_EINVAL;
  dims[0] = ctx->L[n - 1].im; dims[1] = ctx->L[n - 1].jm; dims[2] = ctx->L[n - 1].km;
  return 0;
}

int desalm_set_grid(desalm_ctx* ctx, const double* x, const double* y, const double* z, const double* wd) {
  if (!ctx || !x || !y || !z) return DESALM_EINVAL;
  if (ctx->L.empty()) return DESALM_ENOTREADY;
  const desalm_case& c = ctx->c;
  cudaStream_t s = ctx->stream;
  const long NF = ctx->L[0].N;
  CK(cudaMemcpyAsync(ctx->x, x, NF * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->y, y, NF * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->z, z, NF * sizeof(double), cudaMemcpyHostToDevice, s));
  if (wd) CK(cudaMemcpyAsync(ctx->wd, wd, NF * sizeof(double), cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(ctx->wd, 0, NF * sizeof(double), s));
  ctx->have_wd = wd != nullptr;
  // coordinates of every level (injection), metrics per level in FP64
  double* xs[3] = {ctx->x, ctx->y, ctx->z};
  std::vector<double*> lvl_xyz(3 * ctx->ng, nullptr);
  for (int t = 0; t < 3; ++t) lvl_xyz[t] = xs[t];
  std::vector<void*> tmp;
  auto cleanup = [&]() { for (void* p : tmp) cudaFree(p); };
  for (int n = 1; n < ctx->ng; ++n) {
    Level& C = ctx->L[n];
    Level& F = ctx->L[n - 1];
    for (int t = 0; t < 3; ++t) {
      double* p = nullptr;
      if (cudaMalloc((void**)&p, C.N * sizeof(double)) != cudaSuccess) { cleanup(); ctx->err = "cudaMalloc"; return DESALM_ENOMEM; }
      tmp.push_back(p);
      launch_k(k_inject<double, double>, dim3(cdiv(C.im, 64), C.jm, C.km), 64, 0, s, p, lvl_xyz[3 * (n - 1) + t], C.im, C.jm, C.km, F.im, F.jm,
                                                                              c.icrs, c.jcrs, c.kcrs);
      lvl_xyz[3 * n + t] = p;
    }
  }
  for (int n = 0; n < ctx->ng; ++n) {
    Level& G = ctx->L[n];
    double* cov[9];
    double* met[9];
    double* aj = nullptr;
    for (int t = 0; t < 9; ++t) {
      if (n == 0) cov[t] = ctx->cov[t];
      else {
        if (cudaMalloc((void**)&cov[t], G.N * sizeof(double)) != cudaSuccess) { cleanup(); ctx->err = "cudaMalloc"; return DESALM_ENOMEM; }
        tmp.push_back(cov[t]);
      }
    }
    // metrics are computed in FP64; FP32 levels receive a converted copy
    for (int t = 0; t < 10; ++t) {
      double* p = nullptr;
      if (cudaMalloc((void**)&p, G.N * sizeof(double)) != cudaSuccess) { cleanup(); ctx->err = "cudaMalloc"; return DESALM_ENOMEM; }
      tmp.push_back(p);
      if (t < 9) met[t] = p; else aj = p;
    }
    double** dcov = nullptr;
    double** dmet = nullptr;
    if (cudaMalloc((void**)&dcov, 9 * sizeof(double*)) != cudaSuccess || cudaMalloc((void**)&dmet, 9 * sizeof(double*)) != cudaSuccess) {
      cleanup(); ctx->err = "cudaMalloc"; return DESALM_ENOMEM;
    }
    tmp.push_back(dcov); tmp.push_back(dmet);
    CK(cudaMemcpyAsync(dcov, cov, 9 * sizeof(double*), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dmet, met, 9 * sizeof(double*), cudaMemcpyHostToDevice, s));
    launch_k(k_metrics, dim3(cdiv(G.im, 64), G.jm, G.km), 64, 0, s, lvl_xyz[3 * n], lvl_xyz[3 * n + 1], lvl_xyz[3 * n + 2], G.im, G.jm, G.km,
                                                             G.dc, G.de, G.dz, dcov, dmet, aj);
    CKL();
    // copy into the level's typed arrays
    void* dst[10];
    int esz;
    for (int d = 0; d < 3; ++d) {
      RET(field_ptr(ctx, n, DESALM_F_CSI + d, &dst[d], &esz));
      RET(field_ptr(ctx, n, DESALM_F_ETA + d, &dst[3 + d], &esz));
      RET(field_ptr(ctx, n, DESALM_F_ZET + d, &dst[6 + d], &esz));
    }
    RET(field_ptr(ctx, n, DESALM_F_AJ, &dst[9], &esz));
    for (int t = 0; t < 10; ++t) {
      const double* src = t < 9 ? met[t] : aj;
      if (esz == 8) CK(cudaMemcpyAsync(dst[t], src, G.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
      else launch_k(k_copy<float, double>, cdiv(G.N, 256), 256, 0, s, (float*)dst[t], src, G.N);
    }
    CKL();
    RET(refresh_rj(ctx, n));
    RET(refresh_mw(ctx, n));
    if (n == 0)
      launch_k(k_dtev, cdiv(G.N, 256), 256, 0, s, dcov, ctx->dtev, G.N, c.cfl2, c.vnn2, c.ren, c.delti, c.unsteady);
    CKL();
    G.dtau_valid = false;
    // the temporaries above are freed after the stream drains
  }
  std::vector<double> rat;
  outlet_ratios(c, x, y, z, rat, ctx->ratdim);
  CK(cudaMemcpyAsync(ctx->rat, rat.data(), rat.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  cudaError_t e = cudaStreamSynchronize(s);
  cleanup();
  if (e != cudaSuccess) {
    ctx->err = std::string("set_grid: ") + cudaGetErrorString(e);
    return DESALM_ECUDA;
  }
  // the sweep widths for this grid; a captured step uses the old ones
  RET(autotune_sweeps(ctx));
  drop_graph(ctx);
  // the inflow generator's node tables hold the old grid's coordinates:
  // it is off until desalm_rfg_set is called again
  ctx->rfg.on = false;
  ctx->rfg.armed = false;
  ctx->have_grid = true;
  return 0;
}

int desalm_set_state(desalm_ctx* ctx, const double* q, const double* qn, const double* qnm1, const double* nut) {
  if (!ctx || !q) return DESALM_EINVAL;
  cudaStream_t s = ctx->stream;
  const long N = ctx->L[0].N;
  const double* srcs[3] = {q, qn, qnm1};
  for (int a = 0; a < 3; ++a) {
    double** dst = ctx->ftab + 5 * a;
    if (!srcs[a]) {
      for (int m = 0; m < 5; ++m) {
        void* p;
        int esz;
        RET(field_ptr(ctx, 0, DESALM_F_Q + 8 * a + m, &p, &esz));
        CK(cudaMemsetAsync(p, 0, N * sizeof(double), s));
      }
      continue;
    }
    // stream order keeps the next copy into the staging array behind this conversion
    CK(cudaMemcpyAsync(ctx->stage, srcs[a], 5 * N * sizeof(double), cudaMemcpyHostToDevice, s));
    LAUNCH(KC_MISC, 0, N, launch_k(k_aos_to_soa<double>, cdiv(N, 256), 256, 0, s, dst, ctx->stage, 5, N));
    CKL();
  }
  void* dn;
  int esz;
  RET(field_ptr(ctx, 0, DESALM_F_NUT, &dn, &esz));
  if (nut) CK(cudaMemcpyAsync(dn, nut, N * sizeof(double), cudaMemcpyHostToDevice, s));
  else CK(cudaMemsetAsync(dn, 0, N * sizeof(double), s));
  // the caller may reuse its arrays when this returns
  CK(cudaStreamSynchronize(s));
  for (auto& L : ctx->L) L.dtau_valid = false;
  ctx->have_state = true;
  // q^{n-2} of the learned guess is known after one shift when both older
  // levels were given, after two or three otherwise
  ctx->lp.shifts = qnm1 ? 0 : (qn ? -1 : -2);
  return 0;
}

int desalm_get_state(desalm_ctx* ctx, double* q, double* qn, double* qnm1, double* nut) {
  if (!ctx) return DESALM_EINVAL;
  cudaStream_t s = ctx->stream;
  const long N = ctx->L[0].N;
  double* dsts[3] = {q, qn, qnm1};
  for (int a = 0; a < 3; ++a) {
    if (!dsts[a]) continue;
    LAUNCH(KC_MISC, 0, N, launch_k(k_soa_to_aos<double>, cdiv(N, 256), 256, 0, s, ctx->stage, ctx->ftab + 5 * a, 5, N));
    CKL();
    CK(cudaMemcpyAsync(dsts[a], ctx->stage, 5 * N * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  if (nut) {
    void* dn;
    int esz;
    RET(field_ptr(ctx, 0, DESALM_F_NUT, &dn, &esz));
    CK(cudaMemcpyAsync(nut, dn, N * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  return 0;
}

// The reference's own arrays are real(rdf) = FP32 (src/precision.F90:11):
// these variants take them as they are.  The state goes through the device
// staging array as FP32 (5 N floats fit in its 5 N doubles) and is widened
// on the device; the grid, read once, is widened on the host.
int desalm_set_state_f32(desalm_ctx* ctx, const float* q, const float* qn, const float* qnm1, const float* nut) {
  if (!ctx || !q) return DESALM_EINVAL;
  cudaStream_t s = ctx->stream;
  const long N = ctx->L[0].N;
  float* st = (float*)ctx->stage;
  const float* srcs[3] = {q, qn, qnm1};
  for (int a = 0; a < 3; ++a) {
    double** dst = ctx->ftab + 5 * a;
    if (!srcs[a]) {
      for (int m = 0; m < 5; ++m) {
        void* p;
        int esz;
        RET(field_ptr(ctx, 0, DESALM_F_Q + 8 * a + m, &p, &esz));
        CK(cudaMemsetAsync(p, 0, N * sizeof(double), s));
      }
      continue;
    }
    CK(cudaMemcpyAsync(st, srcs[a], 5 * N * sizeof(float), cudaMemcpyHostToDevice, s));
    LAUNCH(KC_MISC, 0, N, launch_k(k_aos_to_soa<double, float>, cdiv(N, 256), 256, 0, s, dst, (const float*)st, 5, N));
    CKL();
  }
  void* dn;
  int esz;
  RET(field_ptr(ctx, 0, DESALM_F_NUT, &dn, &esz));
  if (nut) {
    CK(cudaMemcpyAsync(st, nut, N * sizeof(float), cudaMemcpyHostToDevice, s));
    LAUNCH(KC_MISC, 0, N, launch_k(k_copy<double, float>, cdiv(N, 256), 256, 0, s, (double*)dn, (const float*)st, N));
    CKL();
  } else {
    CK(cudaMemsetAsync(dn, 0, N * sizeof(double), s));
  }
  CK(cudaStreamSynchronize(s));
  for (auto& L : ctx->L) L.dtau_valid = false;
  ctx->have_state = true;
  ctx->lp.shifts = qnm1 ? 0 : (qn ? -1 : -2);
  return 0;
}

int desalm_get_state_f32(desalm_ctx* ctx, float* q, float* qn, float* qnm1, float* nut) {
  if (!ctx) return DESALM_EINVAL;
  cudaStream_t s = ctx->stream;
  const long N = ctx->L[0].N;
  float* st = (float*)ctx->stage;
  float* dsts[3] = {q, qn, qnm1};
  for (int a = 0; a < 3; ++a) {
    if (!dsts[a]) continue;
    LAUNCH(KC_MISC, 0, N, launch_k(k_soa_to_aos<double, float>, cdiv(N, 256), 256, 0, s, st, ctx->ftab + 5 * a, 5, N));
    CKL();
    CK(cudaMemcpyAsync(dsts[a], st, 5 * N * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  if (nut) {
    void* dn;
    int esz;
    RET(field_ptr(ctx, 0, DESALM_F_NUT, &dn, &esz));
    LAUNCH(KC_MISC, 0, N, launch_k(k_copy<float, double>, cdiv(N, 256), 256, 0, s, st, (const double*)dn, N));
    CKL();
    CK(cudaMemcpyAsync(nut, st, N * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  return 0;
}

int desalm_set_grid_f32(desalm_ctx* ctx, const float* x, const float* y, const float* z, const float* wd) {
  if (!ctx || !x || !y || !z) return DESALM_EINVAL;
  if (ctx->L.empty()) return DESALM_ENOTREADY;
  const long N = ctx->L[0].N;
  std::vector<double> X(x, x + N), Y(y, y + N), Z(z, z + N), D;
  if (wd) D.assign(wd, wd + N);
  return desalm_set_grid(ctx, X.data(), Y.data(), Z.data(), wd ? D.data() : nullptr);
}

int desalm_get_field(desalm_ctx* ctx, int n, int f, double* out) {
  if (!ctx || !out || n < 1 || n > ctx->ng) return DESALM_EINVAL;
  void* p;
  int esz;
  RET(field_ptr(ctx, n - 1, f, &p, &esz));
  const long N = ctx->L[n - 1].N;
  cudaStream_t s = ctx->stream;
  if (esz == 8) {
    CK(cudaMemcpyAsync(out, p, N * sizeof(double), cudaMemcpyDeviceToHost, s));
  } else {
    double* d = nullptr;
    CK(cudaMalloc((void**)&d, N * sizeof(double)));
    launch_k(k_copy<double, float>, cdiv(N, 256), 256, 0, s, d, (const float*)p, N);
    cudaMemcpyAsync(out, d, N * sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    cudaFree(d);
  }
  CK(cudaStreamSynchronize(s));
  return 0;
}

int desalm_set_field(desalm_ctx* ctx, int n, int f, const double* in) {
  if (!ctx || !in || n < 1 || n > ctx->ng) return DESALM_EINVAL;
  void* p;
  int esz;
  RET(field_ptr(ctx, n - 1, f, &p, &esz));
  const long N = ctx->L[n - 1].N;
  cudaStream_t s = ctx->stream;
  if (esz == 8) {
    CK(cudaMemcpyAsync(p, in, N * sizeof(double), cudaMemcpyHostToDevice, s));
  } else {
    double* d = nullptr;
    CK(cudaMalloc((void**)&d, N * sizeof(double)));
    cudaMemcpyAsync(d, in, N * sizeof(double), cudaMemcpyHostToDevice, s);
    launch_k(k_copy<float, double>, cdiv(N, 256), 256, 0, s, (float*)p, d, N);
    cudaStreamSynchronize(s);
    cudaFree(d);
  }
  if (f == DESALM_F_AJ) RET(refresh_rj(ctx, n - 1));
  if (f >= DESALM_F_CSI && f < DESALM_F_ZET + 3) RET(refresh_mw(ctx, n - 1));
  CK(cudaStreamSynchronize(s));
  if (f == DESALM_F_NUT || (f >= DESALM_F_CSI && f <= DESALM_F_AJ)) ctx->L[n - 1].dtau_valid = false;
  return 0;
}

int desalm_solver_daf(desalm_ctx* ctx, int n, int recalc, int itr) {
  if (!ctx || n < 1 || n > ctx->ng) return DESALM_EINVAL;
  if (!ctx->have_grid) { ctx->err = "grid not set"; return DESALM_ENOTREADY; }
  RET(do_daf(ctx, n - 1, recalc, itr));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_mg_nlevel(desalm_ctx* ctx, int n) {
  if (!ctx || n < 2 || n > ctx->ng) return DESALM_EINVAL;
  RET(do_nlevel(ctx, n - 1));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_mg_prolong(desalm_ctx* ctx, int n) {
  if (!ctx || n < 1 || n >= ctx->ng) return DESALM_EINVAL;
  RET(do_prolong(ctx, n - 1));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_mg_residual(desalm_ctx* ctx, int n, double res[5]) {
  if (!ctx || !res || n < 1 || n > ctx->ng) return DESALM_EINVAL;
  return do_norm(ctx, n - 1, 0, res);
}

int desalm_bcond_fm(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  RET(do_bcond(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_des_eddy(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  if (ctx->c.turbulence != 1) { ctx->err = "des_eddy needs turbulence = 1"; return DESALM_EINVAL; }
  RET(sa_des_eddy(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_kw_eddy(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  if (ctx->c.turbulence != 2) { ctx->err = "kw_eddy needs turbulence = 2"; return DESALM_EINVAL; }
  if (!ctx->have_grid || !ctx->have_state) { ctx->err = "grid or state not set"; return DESALM_ENOTREADY; }
  RET(kw_eddy_run(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_set_omega(desalm_ctx* ctx, const double* omega, const double* omega_n, const double* omega_nm1) {
  if (!ctx) return DESALM_EINVAL;
  if (ctx->c.turbulence != 2) { ctx->err = "omega needs turbulence = 2"; return DESALM_EINVAL; }
  if (!omega) { ctx->err = "null omega"; return DESALM_EINVAL; }
  const size_t b = ctx->L[0].N * sizeof(double);
  const double* src[3] = {omega, omega_n, omega_nm1};
  for (int t = 0; t < 3; ++t) {
    if (src[t]) CK(cudaMemcpyAsync(ctx->kw.a[t], src[t], b, cudaMemcpyHostToDevice, ctx->stream));
    else CK(cudaMemsetAsync(ctx->kw.a[t], 0, b, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_get_omega(desalm_ctx* ctx, double* omega, double* omega_n, double* omega_nm1) {
  if (!ctx) return DESALM_EINVAL;
  if (ctx->c.turbulence != 2) { ctx->err = "omega needs turbulence = 2"; return DESALM_EINVAL; }
  const size_t b = ctx->L[0].N * sizeof(double);
  double* dst[3] = {omega, omega_n, omega_nm1};
  for (int t = 0; t < 3; ++t)
    if (dst[t]) CK(cudaMemcpyAsync(dst[t], ctx->kw.a[t], b, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_kw_config(desalm_ctx* ctx, double ckin, double cein) {
  if (!ctx) return DESALM_EINVAL;
  if (!(ckin >= 0.0) || !(cein > 0.0)) { ctx->err = "kw_config: ckin >= 0 and cein > 0"; return DESALM_EINVAL; }
  ctx->ckin = ckin;
  ctx->cein = cein;
  drop_graph(ctx);  // the captured step holds the old floors
  return 0;
}

int desalm_wall_functions(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  if (!ctx->have_grid || !ctx->have_state) { ctx->err = "grid or state not set"; return DESALM_ENOTREADY; }
  if (!ctx->have_wd) { ctx->err = "the wall functions need the wall distance (desalm_set_grid wd)"; return DESALM_EINVAL; }
  RET(do_wallfn(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_conservation(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  RET(sa_conservation(ctx));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_save_qold(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  Level& G = ctx->L[0];
  for (int m = 0; m < 5; ++m) {
    void *src, *dst;
    int esz;
    RET(field_ptr(ctx, 0, DESALM_F_Q + m, &src, &esz));
    RET(field_ptr(ctx, 0, DESALM_F_QOLD + m, &dst, &esz));
    CK(cudaMemcpyAsync(dst, src, G.N * esz, cudaMemcpyDeviceToDevice, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_begin_step(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  if (!ctx->have_grid || !ctx->have_state) { ctx->err = "grid or state not set"; return DESALM_ENOTREADY; }
  if (ctx->c.wall_functions && !ctx->have_wd) {
    ctx->err = "the wall functions need the wall distance (desalm_set_grid wd)";
    return DESALM_EINVAL;
  }
  const desalm_case& c = ctx->c;
  cudaStream_t s = ctx->stream;
  Level& F = ctx->L[0];
  const bool learned = c.predictor == DESALM_PRED_LEARNED;
  // the learned guess trains on the step just converged before the shift
  if (learned) {
    RET(lp_join(ctx));
    RET(lp_learn(ctx));
  }
  // qnm1 <- qn; qn <- q (src/mg_driver.F90:48-51)
  for (int m = 0; m < 5; ++m) {
    void *q, *qn, *qnm1;
    int esz;
    RET(field_ptr(ctx, 0, DESALM_F_Q + m, &q, &esz));
    RET(field_ptr(ctx, 0, DESALM_F_QN + m, &qn, &esz));
    RET(field_ptr(ctx, 0, DESALM_F_QNM1 + m, &qnm1, &esz));
    if (learned) CK(cudaMemcpyAsync(ctx->lp.qnm2[m], qnm1, F.N * esz, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(qnm1, qn, F.N * esz, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(qn, q, F.N * esz, cudaMemcpyDeviceToDevice, s));
    if (c.predictor == DESALM_PRED_LINEAR || learned)
      LAUNCH(KC_MISC, 0, F.N, launch_k(k_extrapolate<double>, cdiv(F.N, 256), 256, 0, s, (double*)q, (const double*)qn, (const double*)qnm1, F.N));
  }
  CKL();
  if (c.turbulence == 2) {  // omega: qnm1(2) <- qn(2) <- q(6), then the same guess without the network
    double* const* w = ctx->kw.a;
    CK(cudaMemcpyAsync(w[2], w[1], F.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(w[1], w[0], F.N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (c.predictor == DESALM_PRED_LINEAR || learned)
      LAUNCH(KC_MISC, 0, F.N, launch_k(k_extrapolate<double>, cdiv(F.N, 256), 256, 0, s, w[0], (const double*)w[1], (const double*)w[2], F.N));
    CKL();
  }
  if (learned) {
    ctx->lp.shifts += 1;
    RET(lp_predict(ctx));
    RET(lp_train_launch(ctx));
  }
  // The inflow plane that desalm_rfg_inlet forced for this step is an
  // inflow boundary (velocity held through the step): an extrapolated or
  // learned guess has overwritten it, so it is forced again for the same time
  // (the same values, bit for bit).  Under the q^n guess it is untouched.
  if (ctx->rfg.armed && (c.predictor == DESALM_PRED_LINEAR || learned)) RET(rfg_launch(ctx, ctx->rfg.time));
  ctx->rfg.armed = false;
  // inject qn, qnm1 to the coarse levels (src/mg_driver.F90:55-58)
  for (int n = 1; n < ctx->ng; ++n) {
    Level& C = ctx->L[n];
    Level& P = ctx->L[n - 1];
    for (int a = 0; a < 2; ++a)
      for (int m = 0; m < 5; ++m) {
        int f = (a == 0 ? DESALM_F_QN : DESALM_F_QNM1) + m;
        void *pf, *pc;
        int ef, ec;
        RET(field_ptr(ctx, n - 1, f, &pf, &ef));
        RET(field_ptr(ctx, n, f, &pc, &ec));
        dim3 g(cdiv(C.im, 64), C.jm, C.km);
        if (ef == 8 && ec == 8)
          LAUNCH(KC_MISC, n, C.N, launch_k(k_inject<double, double>, g, 64, 0, s, (double*)pc, (const double*)pf, C.im, C.jm, C.km, P.im, P.jm, c.icrs, c.jcrs, c.kcrs));
        else if (ef == 8)
          LAUNCH(KC_MISC, n, C.N, launch_k(k_inject<double, float>, g, 64, 0, s, (float*)pc, (const double*)pf, C.im, C.jm, C.km, P.im, P.jm, c.icrs, c.jcrs, c.kcrs));
        else
          LAUNCH(KC_MISC, n, C.N, launch_k(k_inject<float, float>, g, 64, 0, s, (float*)pc, (const float*)pf, C.im, C.jm, C.km, P.im, P.jm, c.icrs, c.jcrs, c.kcrs));
      }
  }
  CKL();
  if (c.conservation) RET(sa_conservation(ctx));
  ctx->itc = 0;
  RET(desalm_save_qold(ctx));
  return 0;
}

int desalm_pseudo_iteration(desalm_ctx* ctx, desalm_step_report* rep) {
  if (!ctx) return DESALM_EINVAL;
  return pseudo_iter(ctx, rep);
}

int desalm_mg_driver(desalm_ctx* ctx, desalm_step_report* rep) {
  if (!ctx) return DESALM_EINVAL;
  RET(desalm_begin_step(ctx));
  int rc = run_step(ctx, rep);
  if ((rc == DESALM_ENONFINITE || rc == DESALM_ESINGULAR) && ctx->lp.predicted) {
    RET(lp_fallback(ctx));
    ctx->itc = 0;
    RET(desalm_save_qold(ctx));
    rc = run_step(ctx, rep);
  }
  return rc;
}

int desalm_mg_driver_batch(desalm_ctx* const* ctxs, int n, desalm_step_report* reps) {
  if (!ctxs || n < 0) return DESALM_EINVAL;
  for (int b = 0; b < n; ++b)
    if (!ctxs[b]) return DESALM_EINVAL;
  // contexts on the graph path (not the learned guess, which trains and
  // falls back on the host) have their steps in flight together; the others
  // step one after another in between
  std::vector<char> inflight(n, 0);
  int first = 0;
  for (int b = 0; b < n && !first; ++b) {
    desalm_ctx* ctx = ctxs[b];
    desalm_step_report* rep = reps ? reps + b : nullptr;
    const bool batched = ctx->c.use_graph && !ctx->prof_on && ctx->c.predictor != DESALM_PRED_LEARNED;
    if (!batched) {
      first = desalm_mg_driver(ctx, rep);
      continue;
    }
    first = desalm_begin_step(ctx);
    if (!first) first = graph_launch(ctx);
    if (!first) inflight[b] = 1;
  }
  // every step in flight is finished, also after an error
  for (int b = 0; b < n; ++b) {
    if (!inflight[b]) continue;
    const int rc = graph_finish(ctxs[b], reps ? reps + b : nullptr);
    if (!first) first = rc;
  }
  return first;
}

int desalm_sweep_widths(desalm_ctx* ctx, int nl[12]) {
  if (!ctx || !nl) return DESALM_EINVAL;
  for (int n = 0; n < 4; ++n)
    for (int d = 0; d < 3; ++d) nl[3 * n + d] = n < ctx->ng ? ctx->sweep_nl[n][d] : 0;
  return 0;
}

int desalm_turb_sweep_widths(desalm_ctx* ctx, int nl[3]) {
  if (!ctx || !nl) return DESALM_EINVAL;
  for (int d = 0; d < 3; ++d) nl[d] = ctx->sa_nl[d];
  return 0;
}

int desalm_set_sweep_widths(desalm_ctx* ctx, const int nl[12], const int turb[3]) {
  if (!ctx) return DESALM_EINVAL;
  const size_t wb = ctx->c.precision_mode == DESALM_FP64 ? 8 : 4;
  if (nl) {
    for (int n = 0; n < 4; ++n)
      for (int d = 0; d < 3; ++d) {
        const int v = nl[3 * n + d];
        if (n >= ctx->ng) {
          if (v) { ctx->err = "sweep width given for a level the case does not have"; return DESALM_EINVAL; }
          continue;
        }
        const Level& G = ctx->L[n];
        const int len = d == 0 ? G.im - 2 : (d == 1 ? G.jm - 2 : G.km - 2);
        const int rows = len + ((d == 0 && n == 0 && ctx->c.btype[1] == 5) ? 1 : 0);
        const bool ok = v == 0 || v == 1 || (v == 2 && rows <= kPcrRows) ||
                        ((v == 4 || v == 8 || v == 16) && (size_t)10 * slab_fs(len + 2, v + 1) * wb <= kSlabMax);
        if (!ok) {
          ctx->err = "DAF sweep width must be 0, 1, 2 (lines of at most 32 rows), or 4, 8, 16 with a slab that fits";
          return DESALM_EINVAL;
        }
      }
  }
  if (turb) {
    for (int d = 0; d < 3; ++d) {
      const int v = turb[d];
      const int len = d == 0 ? ctx->c.im - 2 : (d == 1 ? ctx->c.jm - 2 : ctx->c.km - 2);
      const bool ok = v == 0 || v == 1 || ((v == 8 || v == 16 || v == 32) && (size_t)4 * slab_fs(len, v + 1) * wb <= kSlabMax);
      if (!ok) { ctx->err = "turbulence sweep width must be 0, 1, or 8, 16, 32 with a slab that fits"; return DESALM_EINVAL; }
    }
  }
  if (nl)
    for (int n = 0; n < ctx->ng; ++n)
      for (int d = 0; d < 3; ++d) ctx->sweep_nl[n][d] = nl[3 * n + d];
  if (turb)
    for (int d = 0; d < 3; ++d) ctx->sa_nl[d] = turb[d];
  drop_graph(ctx);
  return 0;
}

int desalm_kernel_tiles(desalm_ctx* ctx, int tiles[36]) {
  if (!ctx || !tiles) return DESALM_EINVAL;
  for (int n = 0; n < 4; ++n)
    for (int w = 0; w < 3; ++w)
      for (int d = 0; d < 3; ++d) tiles[9 * n + 3 * w + d] = n < ctx->ng ? (int)ctx->tile[n][w][d] : 0;
  return 0;
}

int desalm_sync(desalm_ctx* ctx) {
  if (!ctx) return DESALM_EINVAL;
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

}  // extern "C"

namespace {

// One pseudo-time iteration (src/mg_driver.F90:81-316).  qold_mg of the fine
// level holds q at the start of the iteration (set by desalm_begin_step for
// the first one and by the norm kernel of the previous one).
// The kernels of one pseudo-time iteration up to bcond_fm
// (src/mg_driver.F90:98-304), enqueued on the context stream; used eagerly
// and under stream capture.  It is split where the reference exchanges
// overset donor data between blocks (desalm_overset_mg_driver): each
// fine-level smoothing iteration itr is the turbulence sub-iterations
// (part 0; mg_bintp_tur follows, src/mg_driver.F90:164-183) and the DAF step
// with the wall functions (part 1; mg_bintp_mom follows, :237-244); then the
// coarse levels, the prolongation and bcond_fm.
int enqueue_fine(desalm_ctx* ctx, int itr, int part) {
  const desalm_case& c = ctx->c;
  const int n = 0;
  if (part == 0) {
    if (itr == 1) {
      ctx->alm_pending = false;
      CK(cudaMemsetAsync(ctx->flags, 0, 3 * sizeof(int), ctx->stream));
      ctx->recalc = 0;
    }
    // decide_recalc_rh keeps its last value on the coarsest level (Q5)
    if (n != ctx->ng - 1) ctx->recalc = (itr != c.iter[n]) ? 0 : 1;
    // the forcing reads the velocities, which the turbulence sub-iterations
    // leave alone: it runs beside them and joins before k_resid
    if (ctx->alm.on && c.turbulence && !ctx->prof_on) {
      RET(fork_side(ctx));
      Level& G0 = ctx->L[0];
      RET(kind_of(ctx, 0) == K_DD ? alm_run(ctx, G0.dd, ctx->side) : alm_run(ctx, G0.df, ctx->side));
      ctx->alm_pending = true;
    }
    if (c.turbulence == 1) RET(sa_des_eddy(ctx));
    if (c.turbulence == 2) RET(kw_eddy_run(ctx));
    return 0;
  }
  // the recalculated residual on the coarsest level feeds nothing
  const int rc_eff = (n == ctx->ng - 1) ? 0 : ctx->recalc;
  RET(do_daf(ctx, n, rc_eff, itr));
  if (c.wall_functions) RET(do_wallfn(ctx));
  return 0;
}

int enqueue_coarse(desalm_ctx* ctx) {
  const desalm_case& c = ctx->c;
  for (int n = 1; n < ctx->ng; ++n) {
    RET(do_nlevel(ctx, n));
    for (int itr = 1; itr <= c.iter[n]; ++itr) {
      if (n != ctx->ng - 1) ctx->recalc = (itr != c.iter[n]) ? 0 : 1;
      const int rc_eff = (n == ctx->ng - 1) ? 0 : ctx->recalc;
      RET(do_daf(ctx, n, rc_eff, itr));
    }
  }
  for (int n = ctx->ng - 2; n >= 0; --n) RET(do_prolong(ctx, n));
  RET(do_bcond(ctx));
  return 0;
}

int enqueue_iteration(desalm_ctx* ctx) {
  for (int itr = 1; itr <= ctx->c.iter[0]; ++itr) {
    RET(enqueue_fine(ctx, itr, 0));
    RET(enqueue_fine(ctx, itr, 1));
  }
  return enqueue_coarse(ctx);
}

int pseudo_iter(desalm_ctx* ctx, desalm_step_report* rep) {
  const desalm_case& c = ctx->c;
  ctx->itc++;
  RET(enqueue_iteration(ctx));
  double res[5];
  RET(do_norm(ctx, 0, 1, res));
  int hflags[3] = {0, 0, 0};
  CK(cudaMemcpy(hflags, ctx->flags, 3 * sizeof(int), cudaMemcpyDeviceToHost));
  if (ctx->itc == 1)
    for (int m = 0; m < 5; ++m) ctx->init_resd[m] = res[m];
  // mg_ck_conver (src/mg_driver.F90:372-398)
  double eomax = std::max(res[1], std::max(res[2], res[3]));
  double ermax = std::max(res[1] - ctx->init_resd[1], std::max(res[2] - ctx->init_resd[2], res[3] - ctx->init_resd[3]));
  bool conv = false;
  if (ctx->itc > c.it_min && ermax < c.er_min) conv = true;
  if (ctx->itc > c.it_min && eomax < c.eo_min) conv = true;
  if (rep) {
    rep->iterations = ctx->itc;
    rep->converged = conv ? 1 : 0;
    for (int m = 0; m < 5; ++m) { rep->residual[m] = res[m]; rep->init_residual[m] = ctx->init_resd[m]; }
    rep->pivots = hflags[0];
    rep->pivot_lines = hflags[2];
  }
  if (hflags[1]) { ctx->err = "zero pivot in a line solve"; return DESALM_ESINGULAR; }
  for (int m = 1; m < 4; ++m)
    if (!std::isfinite(res[m])) { ctx->err = "non-finite convergence norm"; return DESALM_ENONFINITE; }
  return 0;
}

}  // namespace

namespace {
ProfScope::ProfScope(desalm_ctx* c, int cls, int lvl, double nodes) : ctx(c), slot(0), on(c->prof_on) {
  ctx->launches++;
  if (!on) return;
  if (ctx->prof_used == ctx->prof.size()) {
    desalm_ctx::ProfRec r{};
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    ctx->prof.push_back(r);
  }
  slot = ctx->prof_used++;
  desalm_ctx::ProfRec& r = ctx->prof[slot];
  r.cls = cls; r.lvl = lvl; r.nodes = nodes;
  cudaEventRecord(r.a, ctx->stream);
}
ProfScope::~ProfScope() {
  if (on) cudaEventRecord(ctx->prof[slot].b, ctx->stream);
}
}  // namespace

extern "C" {
// Enable/disable per-kernel event timing; resets the statistics and the
// launch counter.
int desalm_profile(desalm_ctx* ctx, int enable) {
  if (!ctx) return DESALM_EINVAL;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->prof_on = enable != 0;
  ctx->prof_used = 0;
  ctx->launches = 0;
  return 0;
}
// Per kernel class and level (KC_COUNT x 4 entries, index cls*4 + level):
// total milliseconds, launches and nodes processed since desalm_profile.
int desalm_kernel_stats(desalm_ctx* ctx, double* ms, long* launches, double* nodes, long* total_launches) {
  if (!ctx) return DESALM_EINVAL;
  CK(cudaStreamSynchronize(ctx->stream));
  for (int t = 0; t < KC_COUNT * 4; ++t) { ms[t] = 0; launches[t] = 0; nodes[t] = 0; }
  for (size_t i = 0; i < ctx->prof_used; ++i) {
    desalm_ctx::ProfRec& r = ctx->prof[i];
    float e = 0.f;
    cudaEventElapsedTime(&e, r.a, r.b);
    int t = r.cls * 4 + std::min(r.lvl, 3);
    ms[t] += e; launches[t] += 1; nodes[t] += r.nodes;
  }
  if (total_launches) *total_launches = ctx->launches;
  return 0;
}
int desalm_kernel_class_count(void) { return KC_COUNT; }
// The CUDA stream of the context (cudaStream_t), for callers that order
// their own work or events with the library's.
void* desalm_stream(desalm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }
}  // extern "C"

namespace {

// SA view of the fine level: nu_tilde, nu_t and the residual terms in FP64;
// the ADI work in W (FP32 in MIXED mode).
template <class SW, class W>
SaT<SW> make_sa(desalm_ctx* ctx, Lv<double, W>& L) {
  SaT<SW> S{};
  S.im = L.im; S.jm = L.jm; S.km = L.km; S.N = L.N; S.sj = L.sj; S.sk = L.sk;
  for (int m = 0; m < 5; ++m) S.q[m] = L.q[m];
  S.qn5 = L.qn[4]; S.qnm1_5 = L.qnm1[4];
  for (int d = 0; d < 3; ++d) { S.csi[d] = L.csi[d]; S.eta[d] = L.eta[d]; S.zet[d] = L.zet[d]; }
  S.aj = L.aj; S.rj = L.rj; S.wd = ctx->wd; S.dtev = ctx->dtev; S.nut = L.nut;
  S.wo = ctx->sa.a[0];
  S.rh = (SW*)ctx->sa.a[1];
  for (int t = 0; t < 9; ++t) S.co[t] = (SW*)ctx->sa.a[2 + t];
  for (int d = 0; d < 3; ++d) S.uc[d] = ctx->sa.a[11 + d];
  S.flags = ctx->flags;
  S.gs = (SW*)ctx->gsweep;
  S.gss = ctx->gss;
  S.ren = ctx->c.ren; S.delti = ctx->c.delti; S.es = ctx->c.unsteady ? 1.0 : 0.0;
  for (int b = 0; b < 6; ++b) { S.sa1[b] = ctx->par.sa[0][b]; S.sb1[b] = ctx->par.sb[0][b]; S.btype[b] = ctx->c.btype[b]; }
  S.rat = (const double*)ctx->rat;
  S.ratdim = ctx->ratdim;
  S.upd = L.q[4];
  return S;
}

// One SA ADI sweep as k_sa_sweep4 with the widest slab whose shared memory
// leaves room for two CTAs per SM (amax lines of n nodes in each of nb planes).
template <class SW>
size_t sa_slab_bytes(int n, int nl) { return (size_t)4 * slab_fs(n, nl + 1) * sizeof(SW); }
template <class SW, int DIR, int NL>
int sa_sweep_nl(desalm_ctx* ctx, SaT<SW>& S, int amax, int n, int nb, double nin) {
  cudaStream_t s = ctx->stream;
  LAUNCH(KC_SA_SWEEP, 0, nin, launch_k(k_sa_sweep4<SW, DIR, NL>, dim3(cdiv(amax, NL), nb), kSlabThreads, sa_slab_bytes<SW>(n, NL), s, S));
  CKL();
  return 0;
}
template <class SW, int DIR>
int sa_sweep(desalm_ctx* ctx, SaT<SW>& S, int amax, int n, int nb, double nin) {
  const int want = ctx->sa_nl[DIR];
  if (want == 0 || want == 1) {
    LAUNCH(KC_SA_SWEEP, 0, nin, launch_k(k_sa_gsweep<SW, DIR>, dim3(cdiv(amax, 64), nb, 1), 128, 0, ctx->stream, S, SaPair<SW>{}));
    CKL();
    return 0;
  }
  if (want == 32 && sa_slab_bytes<SW>(n, 32) <= kSlabMax) return sa_sweep_nl<SW, DIR, 32>(ctx, S, amax, n, nb, nin);
  if (want == 16 && sa_slab_bytes<SW>(n, 16) <= kSlabMax) return sa_sweep_nl<SW, DIR, 16>(ctx, S, amax, n, nb, nin);
  if (want == 8 && sa_slab_bytes<SW>(n, 8) <= kSlabMax) return sa_sweep_nl<SW, DIR, 8>(ctx, S, amax, n, nb, nin);
  if (sa_slab_bytes<SW>(n, 32) <= kSlabTwoPerSm) return sa_sweep_nl<SW, DIR, 32>(ctx, S, amax, n, nb, nin);
  if (sa_slab_bytes<SW>(n, 16) <= kSlabTwoPerSm) return sa_sweep_nl<SW, DIR, 16>(ctx, S, amax, n, nb, nin);
  if (sa_slab_bytes<SW>(n, 8) <= kSlabMax) return sa_sweep_nl<SW, DIR, 8>(ctx, S, amax, n, nb, nin);
  ctx->err = "grid line too long for the shared-memory SA sweep";
  return DESALM_EINVAL;
}

// The turbulence line sweep of one direction timed with the lines-in-lanes
// kernel and with each slab width that fits (one warm-up launch, five timed
// with CUDA events); the fastest is kept.  The sweeps of i and j write only
// the model's right-hand-side work array, which the residual rewrites before
// any use, so timing them changes no result.
template <class W, int DIR>
int tune_sa_dir(desalm_ctx* ctx, SaT<W>& S, cudaEvent_t e0, cudaEvent_t e1) {
  const int amax = DIR == 0 ? S.jm - 2 : S.im - 2;
  const int n = DIR == 0 ? S.im - 2 : (DIR == 1 ? S.jm - 2 : S.km - 2);
  const int nb = DIR == 2 ? S.jm - 2 : S.km - 2;
  const double nin = double(amax) * n * nb;
  float best = 0.f;
  int pick = 0;
  for (int nl : {1, 32, 16, 8}) {
    if (nl != 1 && sa_slab_bytes<W>(n, nl) > kSlabMax) continue;
    ctx->sa_nl[DIR] = nl;
    RET((sa_sweep<W, DIR>(ctx, S, amax, n, nb, nin)));
    CK(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < 5; ++r) RET((sa_sweep<W, DIR>(ctx, S, amax, n, nb, nin)));
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (!pick || ms < best) { best = ms; pick = nl; }
  }
  ctx->sa_nl[DIR] = pick;
  return 0;
}

// The i and j turbulence sweeps are timed; the k sweep, which also updates
// the model's scalar, takes the j sweep's choice (both read their rows
// coalesced across the lanes, with a stride along the line).
template <class W>
int tune_sa(desalm_ctx* ctx, Lv<double, W>& L, cudaEvent_t e0, cudaEvent_t e1) {
  SaT<W> S = make_sa<W>(ctx, L);
  RET((tune_sa_dir<W, 0>(ctx, S, e0, e1)));
  RET((tune_sa_dir<W, 1>(ctx, S, e0, e1)));
  ctx->sa_nl[2] = ctx->sa_nl[1];
  return 0;
}
int tune_sa_fine(desalm_ctx* ctx, cudaEvent_t e0, cudaEvent_t e1) {
  if (!ctx->c.turbulence) return 0;
  return kind_of(ctx, 0) == K_DD ? tune_sa(ctx, ctx->L[0].dd, e0, e1) : tune_sa(ctx, ctx->L[0].df, e0, e1);
}

template <class W>
int sa_run(desalm_ctx* ctx, Lv<double, W>& L) {
  SaT<W> S = make_sa<W>(ctx, L);
  cudaStream_t s = ctx->stream;
  const double nin = double(L.im - 2) * (L.jm - 2) * (L.km - 2);
  const dim3 gi(cdiv(L.im - 2, 32), cdiv(L.jm - 2, 4), L.km - 2);
  LAUNCH(KC_SA_AUX, 0, nin, launch_k(k_sa_source<W>, gi, blk3(), 0, s, S));
  LAUNCH(KC_SA_AUX, 0, L.N, launch_k(k_sa_ucn<W>, cdiv(L.N, 256), 256, 0, s, S));
  for (int it = 0; it < ctx->c.itk; ++it) {
    LAUNCH(KC_SA_RHS, 0, nin, launch_k(k_sa_rhs<W>, grid_t(ctx, 0, 2, L.im, L.jm, L.km), blk_t(ctx, 0, 2), 0, s, S));
    RET((sa_sweep<W, 0>(ctx, S, L.jm - 2, L.im - 2, L.km - 2, nin)));
    RET((sa_sweep<W, 1>(ctx, S, L.im - 2, L.jm - 2, L.km - 2, nin)));
    RET((sa_sweep<W, 2>(ctx, S, L.im - 2, L.km - 2, L.jm - 2, nin)));
    LAUNCH(KC_SA_BC, 0, 2.0 * L.jm * L.km, launch_k(k_sa_bc<W, 0>, dim3(cdiv(L.jm, 64), L.km), 64, 0, s, S));
    LAUNCH(KC_SA_BC, 0, 2.0 * L.im * L.km, launch_k(k_sa_bc<W, 1>, dim3(cdiv(L.im, 64), L.km), 64, 0, s, S));
    LAUNCH(KC_SA_BC, 0, 2.0 * L.im * L.jm, launch_k(k_sa_bc<W, 2>, dim3(cdiv(L.im, 64), L.jm), 64, 0, s, S));
    LAUNCH(KC_SA_BC, 0, L.N, launch_k(k_sa_clamp<W>, cdiv(L.N, 256), 256, 0, s, S));
  }
  CKL();
  ctx->L[0].dtau_valid = false;  // nu_t changed
  return 0;
}

template <class W>
int cons_run(desalm_ctx* ctx, Lv<double, W>& L) {
  Sa S = make_sa<double>(ctx, L);
  cudaStream_t s = ctx->stream;
  double* acc = ctx->part;
  LAUNCH(KC_MISC, 0, 2.0 * L.jm * L.km, launch_k(k_cons_sum, 1, 256, 0, s, S, acc));
  LAUNCH(KC_MISC, 0, 1.0 * L.jm * L.km, launch_k(k_cons_apply, cdiv(L.jm * L.km, 128), 128, 0, s, S, acc, ctx->dcov));
  CKL();
  return 0;
}

int sa_des_eddy(desalm_ctx* ctx) {
  if (ctx->c.turbulence != 1) return 0;
  return kind_of(ctx, 0) == K_DD ? sa_run(ctx, ctx->L[0].dd) : sa_run(ctx, ctx->L[0].df);
}

// k-omega view of the fine level: k's rows and right-hand side in the SA
// work arrays, omega and the model's FP64 arrays in KwWork.
template <class W>
KwT<W> make_kw(desalm_ctx* ctx, Lv<double, W>& L) {
  KwT<W> K{};
  K.S = make_sa<W>(ctx, L);
  double* const* a = ctx->kw.a;
  K.om = a[0]; K.omn = a[1]; K.omnm1 = a[2];
  K.As = a[3]; K.Ac = a[4]; K.Bs = a[5]; K.ptke = a[6];
  for (int t = 0; t < 9; ++t) K.cow[t] = (W*)a[9 + t];
  K.rhw = (W*)a[18];
  K.ckin = ctx->ckin; K.cein = ctx->cein;
  const int* bt = ctx->c.btype;
  K.ista = bt[0] != 1 ? 0 : 1; K.iend = bt[1] != 1 ? L.im - 1 : L.im - 2;
  K.jsta = bt[2] != 1 ? 0 : 1; K.jend = bt[3] != 1 ? L.jm - 1 : L.jm - 2;
  K.ksta = bt[4] != 1 ? 0 : 1; K.kend = bt[5] != 1 ? L.km - 1 : L.km - 2;
  return K;
}

// kw_eddy (src/kw_eddy.F90:109-289): the model's coefficients and
// production once, then itk sub-iterations of the fused residual, the line
// solves of k and of omega (each updating its scalar after its k sweep), the
// boundary values, nu_t and the wall edges.
// The line solves of two independent scalars along one direction: one
// launch of the lines-in-lanes kernel for both where that kernel is chosen,
// else the two in turn.
template <class SW, int DIR>
int sa_sweep_pair(desalm_ctx* ctx, SaT<SW>& S, SaT<SW>& S2, int amax, int n, int nb, double nin) {
  const int want = ctx->sa_nl[DIR];
  if (want == 0 || want == 1) {
    SaPair<SW> B{{S2.co[3 * DIR + 0], S2.co[3 * DIR + 1], S2.co[3 * DIR + 2]}, S2.rh, S2.upd};
    LAUNCH(KC_SA_SWEEP, 0, 2 * nin, launch_k(k_sa_gsweep<SW, DIR>, dim3(cdiv(amax, 64), nb, 2), 128, 0, ctx->stream, S, B));
    CKL();
    return 0;
  }
  RET((sa_sweep<SW, DIR>(ctx, S, amax, n, nb, nin)));
  return sa_sweep<SW, DIR>(ctx, S2, amax, n, nb, nin);
}

template <class W>
int kw_run(desalm_ctx* ctx, Lv<double, W>& L) {
  KwT<W> K = make_kw<W>(ctx, L);
  SaT<W> Sw = K.S;           // the omega line solves: omega's rows, right-hand side and field
  for (int t = 0; t < 9; ++t) Sw.co[t] = K.cow[t];
  Sw.rh = K.rhw;
  Sw.upd = K.om;
  cudaStream_t s = ctx->stream;
  const double nin = double(L.im - 2) * (L.jm - 2) * (L.km - 2);
  LAUNCH(KC_SA_AUX, 0, L.N, launch_k(k_sa_ucn<W>, cdiv(L.N, 256), 256, 0, s, K.S));
  LAUNCH(KC_SA_AUX, 0, L.N, launch_k(k_kw_pre<W>, cdiv(L.N, 256), 256, 0, s, K));
  for (int it = 0; it < ctx->c.itk; ++it) {
    LAUNCH(KC_SA_RHS, 0, nin, launch_k(k_kw_rhs<W>, dim3(cdiv(L.im - 2, KWF_TX), cdiv(L.jm - 2, KWF_TY), cdiv(L.km - 2, KWF_TZ)), 256, 0, s, K));
    // k's and omega's line solves are independent (each has its own rows and
    // right-hand side from k_kw_rhs and updates its own field in its k
    // sweep), so they run together direction by direction
    RET((sa_sweep_pair<W, 0>(ctx, K.S, Sw, L.jm - 2, L.im - 2, L.km - 2, nin)));
    RET((sa_sweep_pair<W, 1>(ctx, K.S, Sw, L.im - 2, L.jm - 2, L.km - 2, nin)));
    RET((sa_sweep_pair<W, 2>(ctx, K.S, Sw, L.im - 2, L.km - 2, L.jm - 2, nin)));
    const int nj = K.jend - K.jsta + 1, ni = K.iend - K.ista + 1, nk = K.kend - K.ksta + 1;
    LAUNCH(KC_SA_BC, 0, 2.0 * nj * nk, launch_k(k_kw_bc<W, 0>, dim3(cdiv(nj, 64), nk), 64, 0, s, K));
    LAUNCH(KC_SA_BC, 0, 2.0 * ni * nk, launch_k(k_kw_bc<W, 1>, dim3(cdiv(ni, 64), nk), 64, 0, s, K));
    LAUNCH(KC_SA_BC, 0, 2.0 * ni * nj, launch_k(k_kw_bc<W, 2>, dim3(cdiv(ni, 64), nj), 64, 0, s, K));
    LAUNCH(KC_SA_BC, 0, L.N, launch_k(k_kw_nut<W>, cdiv(L.N, 256), 256, 0, s, K));
    LAUNCH(KC_SA_BC, 0, 0.0, launch_k(k_kw_edges<W>, 1, 256, 0, s, K));
  }
  CKL();
  ctx->L[0].dtau_valid = false;  // nu_t changed
  return 0;
}

int kw_eddy_run(desalm_ctx* ctx) {
  if (ctx->c.turbulence != 2) return 0;
  return kind_of(ctx, 0) == K_DD ? kw_run(ctx, ctx->L[0].dd) : kw_run(ctx, ctx->L[0].df);
}

int sa_conservation(desalm_ctx* ctx) {
  return kind_of(ctx, 0) == K_DD ? cons_run(ctx, ctx->L[0].dd) : cons_run(ctx, ctx->L[0].df);
}

}  // namespace

namespace {

// Build (once) the graph of a physical step's pseudo-time loop: a while
// conditional node whose body is one pseudo-iteration followed by the norm
// and k_conv, which decides on the device whether to run another iteration
// (no host round trip per pseudo-iteration).
int build_graph(desalm_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  // laminar fine-level dtau never changes: make it valid outside the graph
  if (!ctx->c.turbulence && !ctx->L[0].dtau_valid) {
    Level& G = ctx->L[0];
    Par P = ctx->par;
    P.fine = 1;
    if (kind_of(ctx, 0) == K_DD) LAUNCH(KC_DTAU, 0, G.N, launch_k(k_dtau<double, double>, cdiv(G.N, 256), 256, 0, s, G.dd, P));
    else LAUNCH(KC_DTAU, 0, G.N, launch_k(k_dtau<double, float>, cdiv(G.N, 256), 256, 0, s, G.df, P));
    CKL();
    G.dtau_valid = true;
  }
  if (!ctx->dconv) {
    RET(dalloc(ctx, ctx->allocs, (void**)&ctx->dconv, sizeof(DevConv)));
    if (cudaMallocHost((void**)&ctx->hconv, sizeof(DevConv)) != cudaSuccess) { ctx->err = "cudaMallocHost"; return DESALM_ENOMEM; }
  }
  CK(cudaStreamSynchronize(s));
  cudaGraph_t g = nullptr;
  CK(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  CK(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  CK(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  long l0 = ctx->launches;
  CK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_iteration(ctx);
  Level& G = ctx->L[0];
  const int nb = ctx->part_blocks;
  const long total = (long)(G.im - 2) * (G.jm - 2) * (G.km - 2);
  ConvPar cv{ctx->c.it_min, ctx->c.itmax, ctx->c.er_min, ctx->c.eo_min, double(total)};
  if (!rc) {
    int nbu = (int)std::min<long>(nb, std::max<long>(1, cdiv(total, 256)));
    if (kind_of(ctx, 0) == K_DD) LAUNCH(KC_NORM, 0, double(total), launch_k(k_norm_partial<double, double>, nbu, 256, 0, s, G.dd, ctx->part, 5, 1));
    else LAUNCH(KC_NORM, 0, double(total), launch_k(k_norm_partial<double, float>, nbu, 256, 0, s, G.df, ctx->part, 5, 1));
    LAUNCH(KC_NORM, 0, 0, launch_k(k_conv, 1, 256, 0, s, ctx->part, nbu, ctx->dconv, ctx->flags, cv, h));
  }
  cudaGraph_t out = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &out);
  if (rc || e != cudaSuccess) {
    cudaGraphDestroy(g);
    if (!rc) ctx->err = std::string("graph capture: ") + cudaGetErrorString(e);
    return rc ? rc : DESALM_ECUDA;
  }
  ctx->graph_kernels = ctx->launches - l0;
  ctx->launches = l0;
  e = cudaGraphInstantiate(&ctx->gexec, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    ctx->err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e);
    return DESALM_ECUDA;
  }
  ctx->graph = g;
  return 0;
}

// The pseudo-time loop of one physical step: the CUDA graph, or eagerly
// (while profiling, or when use_graph is off).
int run_step(desalm_ctx* ctx, desalm_step_report* rep) {
  if (ctx->c.use_graph && !ctx->prof_on) return graph_step(ctx, rep);
  desalm_step_report r{};
  int piv = 0, plines = 0;
  for (int it = 1; it <= ctx->c.itmax; ++it) {
    RET(pseudo_iter(ctx, &r));
    piv += r.pivots;
    plines += r.pivot_lines;
    if (r.converged) break;
  }
  r.pivots = piv;
  r.pivot_lines = plines;
  if (rep) *rep = r;
  return 0;
}

// The captured physical step in two halves, so that several contexts can
// have theirs in flight at once (desalm_mg_driver_batch): graph_launch
// enqueues the graph and the read-back of its convergence state on the
// context's stream; graph_finish waits for that stream alone.
int graph_launch(desalm_ctx* ctx) {
  if (!ctx->gexec) RET(build_graph(ctx));
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(ctx->dconv, 0, sizeof(DevConv), s));
  CK(cudaGraphLaunch(ctx->gexec, s));
  CK(cudaMemcpyAsync(ctx->hconv, ctx->dconv, sizeof(DevConv), cudaMemcpyDeviceToHost, s));
  return 0;
}

int graph_finish(desalm_ctx* ctx, desalm_step_report* rep) {
  CK(cudaStreamSynchronize(ctx->stream));
  const DevConv& st = *ctx->hconv;
  ctx->itc = st.itc;
  for (int m = 0; m < 5; ++m) ctx->init_resd[m] = st.init[m];
  ctx->launches += ctx->graph_kernels * st.itc;
  if (rep) {
    rep->iterations = st.itc;
    rep->converged = st.converged;
    for (int m = 0; m < 5; ++m) { rep->residual[m] = st.res[m]; rep->init_residual[m] = st.init[m]; }
    rep->pivots = st.pivots;
    rep->pivot_lines = st.pivot_lines;
  }
  if (st.zero_pivots) { ctx->err = "zero pivot in a line solve"; return DESALM_ESINGULAR; }
  if (st.nonfinite) { ctx->err = "non-finite convergence norm"; return DESALM_ENONFINITE; }
  return 0;
}

int graph_step(desalm_ctx* ctx, desalm_step_report* rep) {
  RET(graph_launch(ctx));
  return graph_finish(ctx, rep);
}

}  // namespace

// ------------------------------------------------------ learned guess ABI
extern "C" {

int desalm_lp_blend(desalm_ctx* ctx, float alpha) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx) return DESALM_EINVAL;
  if (!ctx->lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  if (std::isnan(alpha) || alpha > 1.0f) { ctx->err = "lp_blend: alpha must be <= 1"; return DESALM_EINVAL; }
  ctx->lp.fixed_alpha = alpha < 0.0f ? -1.0f : alpha;
  return 0;
}

int desalm_lp_fields(desalm_ctx* ctx, int mask) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx) return DESALM_EINVAL;
  if (!ctx->lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  if (mask < 0 || mask > 0x1f) { ctx->err = "lp_fields: mask must be within 0..31"; return DESALM_EINVAL; }
  ctx->lp.field_mask = mask;
  return 0;
}

int desalm_lp_config(desalm_ctx* ctx, int train_steps, int warm, float lr, float ymax) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx) return DESALM_EINVAL;
  if (!ctx->lp.on) { ctx->err = "the learned guess is off (predictor is not DESALM_PRED_LEARNED)"; return DESALM_EINVAL; }
  if (train_steps > 1000 || warm > 1000000 || !(lr < 1.0f) || std::isnan(ymax)) {
    ctx->err = "lp_config: value out of range";
    return DESALM_EINVAL;
  }
  if (train_steps >= 0) ctx->lp.train_steps = train_steps;
  if (warm >= 0) ctx->lp.warm = warm;
  if (lr >= 0.0f) ctx->lp.lr = lr;
  if (ymax >= 0.0f) ctx->lp.ymax = ymax;
  return 0;
}

int desalm_lp_report_get(desalm_ctx* ctx, desalm_lp_report* r) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !r) return DESALM_EINVAL;
  const LpState& lp = ctx->lp;
  r->nparam = lp.nparam;
  r->samples = lp.samples;
  r->train_steps = lp.steps;
  r->predictions = lp.predictions;
  r->fallbacks = lp.fallbacks;
  r->first_loss = lp.first_loss;
  r->last_loss = lp.last_loss;
  r->heldout_ratio = -1.0;
  for (int f = 0; f < 5; ++f) r->alpha[f] = 0.0;
  if (lp.on && lp.samples > 0) {
    double v[16];
    float a[8];
    CK(cudaMemcpyAsync(v, lp.vacc, sizeof(v), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(a, lp.alpha, sizeof(a), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    double num = 0.0, den = 0.0;
    for (int f = 0; f < 5; ++f) {
      num += v[10 + f] - 2.0 * a[f] * v[f] + double(a[f]) * a[f] * v[5 + f];
      den += v[10 + f];
      r->alpha[f] = a[f];
    }
    r->heldout_ratio = den > 0.0 ? num / den : -1.0;
  }
  return 0;
}

int desalm_lp_get_params(desalm_ctx* ctx, float* theta) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !theta) return DESALM_EINVAL;
  if (!ctx->lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  CK(cudaMemcpyAsync(theta, ctx->lp.theta, ctx->lp.nparam * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_lp_set_params(desalm_ctx* ctx, const float* theta) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !theta) return DESALM_EINVAL;
  LpState& lp = ctx->lp;
  if (!lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  CK(cudaMemcpyAsync(lp.theta, theta, lp.nparam * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  // a new parameter vector restarts Adam
  CK(cudaMemsetAsync(lp.m, 0, lp.nparam * sizeof(float), ctx->stream));
  CK(cudaMemsetAsync(lp.v, 0, lp.nparam * sizeof(float), ctx->stream));
  lp.adam_t = 0;
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_lp_eval(desalm_ctx* ctx, const float* x, const float* t, float* y, double* loss, float* grad) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !x) return DESALM_EINVAL;
  LpState& lp = ctx->lp;
  if (!lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  cudaStream_t s = ctx->stream;
  const long N = lp.N;
  // the FP32 features pass through the state staging array (5 N doubles =
  // 10 N floats), 8 channels at a time
  float* xf = reinterpret_cast<float*>(ctx->stage);
  for (long c0 = 0; c0 < 16; c0 += 8) {
    const long nc = std::min<long>(8, 16 - c0);
    CK(cudaMemcpyAsync(xf, x + c0 * N, nc * N * sizeof(float), cudaMemcpyHostToDevice, s));
    LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_rows_in, cdiv(N, 256), 256, 0, s, lp.P, 16, (int)c0, (int)nc, (const float*)xf, lp.x0));
    CKL();
  }
  RET(lp_pack(ctx));
  RET(lp_forward(ctx, lp.tm_x0, lp.y));
  if (y) CK(cudaMemcpyAsync(y, lp.y, 5 * N * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (t) {
    CK(cudaMemcpyAsync(lp.t, t, 5 * N * sizeof(float), cudaMemcpyHostToDevice, s));
    double l = 0;
    RET(lp_backward(ctx, lp.tm_x0, lp.y, &l));
    if (loss) *loss = l;
    if (grad) CK(cudaMemcpyAsync(grad, lp.grad, lp.nparam * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  CK(cudaStreamSynchronize(s));
  RET(lp_check(ctx));
  return 0;
}

int desalm_lp_get_buffer(desalm_ctx* ctx, int which, float* out) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !out) return DESALM_EINVAL;
  LpState& lp = ctx->lp;
  if (!lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  cudaStream_t s = ctx->stream;
  const long N = lp.N;
  switch (which) {
    case DESALM_LP_FEATURES: {
      float* xf = reinterpret_cast<float*>(ctx->stage);
      for (long c0 = 0; c0 < 16; c0 += 8) {
        const long nc = std::min<long>(8, 16 - c0);
        LAUNCH(KC_LEARN, 0, 0.0, launch_k(k_lp_rows_out, cdiv(N, 256), 256, 0, s, lp.P, 16, (int)c0, (int)nc, (const bf16*)lp.x0, xf));
        CKL();
        CK(cudaMemcpyAsync(out + c0 * N, xf, nc * N * sizeof(float), cudaMemcpyDeviceToHost, s));
      }
      break;
    }
    case DESALM_LP_TARGET: CK(cudaMemcpyAsync(out, lp.t, 5 * N * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    case DESALM_LP_OUTPUT: CK(cudaMemcpyAsync(out, lp.y, 5 * N * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    case DESALM_LP_SCALES: CK(cudaMemcpyAsync(out, lp.rs, 16 * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    case DESALM_LP_ALPHA: CK(cudaMemcpyAsync(out, lp.alpha, 5 * sizeof(float), cudaMemcpyDeviceToHost, s)); break;
    default: ctx->err = "lp_get_buffer: unknown buffer"; return DESALM_EINVAL;
  }
  CK(cudaStreamSynchronize(s));
  return 0;
}

}  // extern "C"

// ------------------------------------------------------ watchdog self-test
extern "C" {

int desalm_watchdog_selftest(desalm_ctx* ctx, double seconds) {
  if (!ctx || !(seconds > 0.0) || seconds > 10.0) return DESALM_EINVAL;
  int* e = nullptr;
  CK(cudaMalloc(&e, sizeof(int)));
  cudaError_t r = cudaMemsetAsync(e, 0, sizeof(int), ctx->stream);
  if (r == cudaSuccess) {
    k_wait_probe<<<1, 32, 0, ctx->stream>>>((unsigned long long)(seconds * 1e9), e);
    r = cudaGetLastError();
  }
  int h = 0;
  if (r == cudaSuccess) r = cudaMemcpyAsync(&h, e, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream);
  if (r == cudaSuccess) r = cudaStreamSynchronize(ctx->stream);
  cudaFree(e);
  if (r != cudaSuccess) {
    ctx->err = std::string("watchdog self-test: ") + cudaGetErrorString(r);
    return DESALM_ECUDA;
  }
  if (h) {
    ctx->err = "watchdog self-test: the bounded wait gave up as it should";
    return DESALM_ETIMEOUT;
  }
  return 0;
}

}  // extern "C"

// ------------------------------------------------------ checkpoint / restart
extern "C" {

// The reference's restart file from the device state (output_restart,
// src/main.F90:315-393): q(1..me), nu_t when turbulent, qn(1..me), FP32.
int desalm_checkpoint_write(desalm_ctx* ctx, const char* path) {
  if (!ctx || !path) return DESALM_EINVAL;
  if (!ctx->have_state) { ctx->err = "no state to write"; return DESALM_ENOTREADY; }
  const desalm_case& c = ctx->c;
  const size_t N = size_t(c.im) * c.jm * c.km;
  std::vector<double> q(5 * N), qn(5 * N), nut(N);
  RET(desalm_get_state(ctx, q.data(), qn.data(), nullptr, nut.data()));
  const int r = desalm_solu_write(path, c.im, c.jm, c.km, c.turbulence, q.data(), qn.data(), nut.data());
  if (r) ctx->err = desalm_io_error();
  return r;
}

// The device state from a restart file (init_solu, src/init.F90:2324-2475).
// q^{n-1} is not in the file: the reference starts it at zero
// (src/init.F90:1089) and the first step's history shift refills it.
int desalm_checkpoint_read(desalm_ctx* ctx, const char* path) {
  if (!ctx || !path) return DESALM_EINVAL;
  const desalm_case& c = ctx->c;
  const size_t N = size_t(c.im) * c.jm * c.km;
  std::vector<double> q(5 * N), qn(5 * N), nut(N, 0.0);
  const int r = desalm_solu_read(path, c.im, c.jm, c.km, c.turbulence, q.data(), qn.data(), nut.data());
  if (r) {
    ctx->err = desalm_io_error();
    return r;
  }
  return desalm_set_state(ctx, q.data(), qn.data(), nullptr, nut.data());
}

// The learned guess's training state: parameters, Adam moments and counters.
// Layout (little-endian): "DESALMLP", int32 version 1, int64 nparam, int64
// adam steps, int64 samples, then nparam FP32 each of theta, m, v.
int desalm_lp_checkpoint_write(desalm_ctx* ctx, const char* path) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !path) return DESALM_EINVAL;
  LpState& lp = ctx->lp;
  if (!lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  const size_t n = size_t(lp.nparam);
  std::vector<float> buf(3 * n);
  CK(cudaMemcpyAsync(buf.data(), lp.theta, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(buf.data() + n, lp.m, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(buf.data() + 2 * n, lp.v, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  FILE* f = fopen(path, "wb");
  if (!f) { ctx->err = std::string("cannot open ") + path; return DESALM_EIO; }
  const int32_t ver = 1;
  const int64_t hdr[3] = {int64_t(n), int64_t(lp.adam_t), int64_t(lp.samples)};
  bool ok = fwrite("DESALMLP", 1, 8, f) == 8 && fwrite(&ver, 4, 1, f) == 1 && fwrite(hdr, 8, 3, f) == 3 &&
            fwrite(buf.data(), 4, 3 * n, f) == 3 * n;
  ok = (fclose(f) == 0) && ok;
  if (!ok) { ctx->err = std::string("write to ") + path + " failed"; return DESALM_EIO; }
  return 0;
}

int desalm_lp_checkpoint_read(desalm_ctx* ctx, const char* path) {
  if (ctx && ctx->lp.inflight) RET(lp_join(ctx));  // the training in flight first
  if (!ctx || !path) return DESALM_EINVAL;
  LpState& lp = ctx->lp;
  if (!lp.on) { ctx->err = "the learned guess is off"; return DESALM_EINVAL; }
  FILE* f = fopen(path, "rb");
  if (!f) { ctx->err = std::string("cannot open ") + path; return DESALM_EIO; }
  char magic[8];
  int32_t ver = 0;
  int64_t hdr[3] = {0, 0, 0};
  const size_t n = size_t(lp.nparam);
  std::vector<float> buf(3 * n);
  bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, "DESALMLP", 8) == 0 && fread(&ver, 4, 1, f) == 1 && ver == 1 &&
            fread(hdr, 8, 3, f) == 3 && hdr[0] == int64_t(n) && fread(buf.data(), 4, 3 * n, f) == 3 * n;
  fclose(f);
  if (!ok) { ctx->err = std::string(path) + ": not a learned-guess checkpoint of this network"; return DESALM_EIO; }
  CK(cudaMemcpyAsync(lp.theta, buf.data(), n * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(lp.m, buf.data() + n, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaMemcpyAsync(lp.v, buf.data() + 2 * n, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  lp.adam_t = long(hdr[1]);
  lp.samples = long(hdr[2]);
  return 0;
}

}  // extern "C"

// ------------------------------------------------------ actuator-line forcing
namespace {

// Drop the captured physical step so that the next one is captured again
// with the current kernels and parameters.
void drop_graph(desalm_ctx* ctx) {
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  ctx->gexec = nullptr;
  ctx->graph = nullptr;
}

template <class V>
int alm_copy(desalm_ctx* ctx, const std::vector<V>& h, const V** out) {
  void* p = nullptr;
  const size_t bytes = std::max<size_t>(1, h.size()) * sizeof(V);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) { ctx->err = std::string("cudaMalloc: ") + cudaGetErrorString(e); return DESALM_ENOMEM; }
  ctx->alm.allocs.push_back(p);
  if (!h.empty()) CK(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice, ctx->stream));
  *out = (const V*)p;
  return 0;
}

}  // namespace

extern "C" {

int desalm_alm_set(desalm_ctx* ctx, const desalm_alm* a) {
  if (!ctx) return DESALM_EINVAL;
  auto& A = ctx->alm;
  auto bad = [&](const std::string& why) { ctx->err = "alm_set: " + why; return DESALM_EINVAL; };
  const Level& F = ctx->L[0];
  const int im = F.im, jm = F.jm, km = F.km;
  if (a && a->n_tur > 0) {
    if (!a->tur || a->npolar < 1 || !a->polar_offset || !a->polar_count || !a->polar_rows)
      return bad("missing turbine or polar tables");
    if (!(a->length_scale > 0.0) || !(a->vel_infty >= 0.0)) return bad("length_scale must be > 0");
    for (int p = 0; p < a->npolar; ++p) {
      const int o = a->polar_offset[p], n = a->polar_count[p];
      if (o < 0 || n < 2) return bad("polar " + std::to_string(p) + " needs two rows or more");
      if (a->polar_rows[3L * (o + n - 1)] != -999.0) return bad("polar " + std::to_string(p) + " must end with angle -999");
    }
    for (int t = 0; t < a->n_tur; ++t) {
      const desalm_alm_turbine& T = a->tur[t];
      if (T.nblades < 1 || T.nelems < 1 || T.nangles < 1 || T.nker < 0 || !(T.tur_rad > 0.0))
        return bad("turbine " + std::to_string(t + 1) + ": bad sizes or radius");
      if (!T.node_index || !T.node_pos || !T.disk_dat || !T.polar_b || !T.polar_a ||
          (T.nker > 0 && (!T.ker_index || !T.ker_pos || !T.ker_dat)))
        return bad("turbine " + std::to_string(t + 1) + ": missing table");
      const long ne = long(T.nangles) * T.nelems;
      for (long e = 0; e < ne; ++e) {
        const int i = T.node_index[3 * e], j = T.node_index[3 * e + 1], k = T.node_index[3 * e + 2];
        // cells whose lower corner is not interior are skipped on the device; any
        // cell that is used must lie inside the grid
        const bool inner = i >= 2 && i <= im - 1 && j >= 2 && j <= jm - 1 && k >= 2 && k <= km - 1;
        if (!inner && (i < 1 || i > im || j < 1 || j > jm || k < 1 || k > km))
          return bad("turbine " + std::to_string(t + 1) + ": element cell outside the grid");
        if (inner) {
          const long jk = long(j - 1) + long(jm) * (k - 1);
          if (T.polar_b[jk] < 0 || T.polar_b[jk] >= a->npolar || T.polar_a[jk] < 0 || T.polar_a[jk] >= a->npolar)
            return bad("turbine " + std::to_string(t + 1) + ": polar index out of range");
        }
      }
      for (int n = 0; n < T.nker; ++n) {
        const int* I = T.ker_index + 3 * n;
        if (I[0] < 1 || I[0] > im || I[1] < 1 || I[1] > jm || I[2] < 1 || I[2] > km)
          return bad("turbine " + std::to_string(t + 1) + ": kernel node outside the grid");
      }
    }
  }
  // the previous tables are released once the stream has finished with them
  CK(cudaStreamSynchronize(ctx->stream));
  for (void* p : A.allocs) cudaFree(p);
  A.allocs.clear();
  A.on = false;
  A.nker.clear();
  A.elem0.clear();
  drop_graph(ctx);
  auto set_falm = [&](double* f) {
    if (kind_of(ctx, 0) == K_DD) ctx->L[0].dd.falm = f;
    else ctx->L[0].df.falm = f;
  };
  set_falm(nullptr);
  if (!a || a->n_tur <= 0) return 0;

  std::vector<int> tur_of, ker_tur, meta, node_index, polar_b, polar_a, ker_index, polar_off(a->polar_offset, a->polar_offset + a->npolar);
  std::vector<double> par, angle, node_pos, disk_dat, ker_pos, ker_dat;
  long nrows = 0;
  for (int p = 0; p < a->npolar; ++p) nrows = std::max<long>(nrows, a->polar_offset[p] + a->polar_count[p]);
  std::vector<double> polar_rows(a->polar_rows, a->polar_rows + 3 * nrows);
  int E = 0;
  long nodeoff = 0, keroff = 0;
  const long JK = long(jm) * km;
  for (int t = 0; t < a->n_tur; ++t) {
    const desalm_alm_turbine& T = a->tur[t];
    const int ne = T.nblades * T.nelems;
    const int m[ALM_META] = {T.nblades, T.nelems, T.nangles, T.nker, E, int(nodeoff), int(t * JK), int(keroff)};
    meta.insert(meta.end(), m, m + ALM_META);
    par.push_back(T.tsr); par.push_back(T.tur_rad); par.push_back(T.hub_rad);
    angle.push_back(T.angle);
    for (int g = 0; g < ne; ++g) tur_of.push_back(t);
    const long nn = long(T.nangles) * T.nelems;
    node_index.insert(node_index.end(), T.node_index, T.node_index + 3 * nn);
    node_pos.insert(node_pos.end(), T.node_pos, T.node_pos + 27 * nn);
    disk_dat.insert(disk_dat.end(), T.disk_dat, T.disk_dat + 8 * JK);
    polar_b.insert(polar_b.end(), T.polar_b, T.polar_b + JK);
    polar_a.insert(polar_a.end(), T.polar_a, T.polar_a + JK);
    for (int n = 0; n < T.nker; ++n) ker_tur.push_back(t);
    if (T.nker > 0) {
      ker_index.insert(ker_index.end(), T.ker_index, T.ker_index + 3L * T.nker);
      ker_pos.insert(ker_pos.end(), T.ker_pos, T.ker_pos + 3L * T.nker);
      ker_dat.insert(ker_dat.end(), T.ker_dat, T.ker_dat + 4L * T.nker);
    }
    A.nker.push_back(T.nker);
    A.elem0.push_back(E);
    E += ne;
    nodeoff += nn;
    keroff += T.nker;
  }
  AlmDev& D = A.dev;
  D.n_tur = a->n_tur;
  D.E = E;
  D.im = im; D.jm = jm; D.km = km;
  D.length_scale = a->length_scale;
  D.vel_scale = ctx->c.ren * 10E-7 / a->length_scale;
  D.vel_infty = a->vel_infty;
  D.nker_all = int(keroff);
  D.nrows = int(nrows);
  RET(alm_copy(ctx, tur_of, &D.tur_of));
  RET(alm_copy(ctx, ker_tur, &D.ker_tur));
  RET(alm_copy(ctx, meta, &D.meta));
  RET(alm_copy(ctx, par, &D.par));
  RET(alm_copy(ctx, angle, &D.angle));
  RET(alm_copy(ctx, node_index, &D.node_index));
  RET(alm_copy(ctx, node_pos, &D.node_pos));
  RET(alm_copy(ctx, disk_dat, &D.disk_dat));
  RET(alm_copy(ctx, polar_b, &D.polar_b));
  RET(alm_copy(ctx, polar_a, &D.polar_a));
  RET(alm_copy(ctx, ker_index, &D.ker_index));
  RET(alm_copy(ctx, ker_pos, &D.ker_pos));
  RET(alm_copy(ctx, ker_dat, &D.ker_dat));
  RET(alm_copy(ctx, polar_off, &D.polar_off));
  RET(alm_copy(ctx, polar_rows, &D.polar_rows));
  std::vector<double> zero_scr(size_t(E) * ALM_SCR, 0.0), zero_f(size_t(E) * 6, 0.0), zero_field(3 * size_t(F.N), 0.0);
  const double* p = nullptr;
  RET(alm_copy(ctx, zero_scr, &p)); D.scr = const_cast<double*>(p);
  RET(alm_copy(ctx, zero_f, &p)); D.forces = const_cast<double*>(p);
  RET(alm_copy(ctx, zero_field, &p)); A.falm = const_cast<double*>(p);
  CK(cudaStreamSynchronize(ctx->stream));
  set_falm(A.falm);
  A.on = true;
  return 0;
}

int desalm_alm_set_angle(desalm_ctx* ctx, int n_t, double angle) {
  if (!ctx) return DESALM_EINVAL;
  auto& A = ctx->alm;
  if (!A.on || n_t < 1 || n_t > A.dev.n_tur) { ctx->err = "alm_set_angle: no such turbine"; return DESALM_EINVAL; }
  CK(cudaMemcpyAsync(const_cast<double*>(A.dev.angle) + (n_t - 1), &angle, sizeof(double), cudaMemcpyHostToDevice,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

int desalm_alm_get(desalm_ctx* ctx, int what, double* out) {
  if (!ctx || !out) return DESALM_EINVAL;
  auto& A = ctx->alm;
  if (!A.on) { ctx->err = "alm_get: the forcing is off"; return DESALM_EINVAL; }
  if (what == DESALM_ALM_FORCES)
    CK(cudaMemcpyAsync(out, A.dev.forces, 6 * size_t(A.dev.E) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  else if (what == DESALM_ALM_FIELD)
    CK(cudaMemcpyAsync(out, A.falm, 3 * size_t(ctx->L[0].N) * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  else { ctx->err = "alm_get: unknown item"; return DESALM_EINVAL; }
  CK(cudaStreamSynchronize(ctx->stream));
  return 0;
}

}  // extern "C"

// --------------------------------------------- synthetic inflow turbulence
// The random flow generator (rfg.cuh): desalm_rfg_modes draws the spectrum's
// modes on the host (initialize_rfg), desalm_rfg_set moves them and the inflow
// tables to the device and decomposes every node's correlation tensor once
// (rfg_init), desalm_rfg_inlet sets the inflow plane's velocities for a time
// (rfg_mpi_inlet_forcing).
namespace {

// Normal deviates for the mode tables: a splitmix64 stream (Steele, Lea &
// Flood 2014) of uniform doubles in (0, 1), turned into pairs of normal
// deviates by the polar method (Marsaglia & Bray 1964), the second of each
// pair kept for the next call.  The reference draws from its own generator
// (src/rfg.F90:126-236) with the same polar method and call order.
struct RfgGauss {
  uint64_t s;
  bool have = false;
  double kept = 0.0;
  double uniform() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return ((double)(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  }
  double next(double mean, double stdev) {
    double g;
    if (have) {
      g = kept;
      have = false;
    } else {
      double v1, v2, rsq;
      do {
        v1 = 2.0 * uniform() - 1.0;
        v2 = 2.0 * uniform() - 1.0;
        rsq = v1 * v1 + v2 * v2;
      } while (rsq >= 1.0 || rsq == 0.0);
      const double fac = std::sqrt(-2.0 * std::log(rsq) / rsq);
      kept = v1 * fac;
      have = true;
      g = v2 * fac;
    }
    return mean + stdev * g;
  }
};

constexpr int kRfgMaxModes = 1 << 20;

void rfg_free(desalm_ctx* ctx) {
  for (void* p : ctx->rfg.allocs) cudaFree(p);
  ctx->rfg.allocs.clear();
  ctx->rfg.on = false;
  ctx->rfg.armed = false;
  ctx->rfg.dev = RfgDev{};
}

int rfg_launch(desalm_ctx* ctx, double time) {
  const Level& F = ctx->L[0];
  void* qp[3];
  int esz;
  for (int d = 0; d < 3; ++d) RET(field_ptr(ctx, 0, DESALM_F_Q + 1 + d, &qp[d], &esz));
  const long nn = (long)(F.jm - 2) * (F.km - 2);
  LAUNCH(KC_MISC, 0, double(nn), launch_k(k_rfg_inlet, cdiv(nn, RFG_THREADS), RFG_THREADS, 0, ctx->stream, ctx->rfg.dev, time,
                                          (double*)qp[0], (double*)qp[1], (double*)qp[2]));
  CKL();
  return 0;
}

}  // namespace

extern "C" {

int desalm_rfg_modes(int nmodes, long long seed, double* p, double* q, double* k, double* omega) {
  if (nmodes < 1 || nmodes > kRfgMaxModes || !p || !q || !k || !omega) return DESALM_EINVAL;
  RfgGauss g{(uint64_t)seed};
  const size_t N = (size_t)nmodes;
  std::vector<double> zet(3 * N), csi(3 * N);
  // the draws in the order of initialize_rfg (src/rfg.F90:75-84): zet(1..3,:),
  // csi(1..3,:) ~ N(0, 1), k(1..3,:) ~ N(0, 0.5^2), omega ~ N(0, 1)
  for (int d = 0; d < 3; ++d)
    for (size_t i = 0; i < N; ++i) zet[3 * i + d] = g.next(0.0, 1.0);
  for (int d = 0; d < 3; ++d)
    for (size_t i = 0; i < N; ++i) csi[3 * i + d] = g.next(0.0, 1.0);
  for (int d = 0; d < 3; ++d)
    for (size_t i = 0; i < N; ++i) k[3 * i + d] = g.next(0.0, 0.5);
  for (size_t i = 0; i < N; ++i) omega[i] = g.next(0.0, 1.0);
  // p = zet x k, q = csi x k (src/rfg.F90:87-90)
  for (size_t i = 0; i < N; ++i) {
    const double* a = &zet[3 * i];
    const double* b = &csi[3 * i];
    const double* kk = &k[3 * i];
    p[3 * i + 0] = a[1] * kk[2] - a[2] * kk[1];
    p[3 * i + 1] = a[2] * kk[0] - a[0] * kk[2];
    p[3 * i + 2] = a[0] * kk[1] - a[1] * kk[0];
    q[3 * i + 0] = b[1] * kk[2] - b[2] * kk[1];
    q[3 * i + 1] = b[2] * kk[0] - b[0] * kk[2];
    q[3 * i + 2] = b[0] * kk[1] - b[1] * kk[0];
  }
  return 0;
}

int desalm_rfg_set(desalm_ctx* ctx, const desalm_rfg* r) {
  if (!ctx) return DESALM_EINVAL;
  if (ctx->L.empty()) return DESALM_ENOTREADY;
  auto bad = [&](const std::string& why) { ctx->err = "rfg_set: " + why; return DESALM_EINVAL; };
  if (r && r->nmodes != 0) {
    if (r->nmodes < 0 || r->nmodes > kRfgMaxModes) return bad("nmodes must be 1.." + std::to_string(kRfgMaxModes));
    if (!r->p || !r->q || !r->k || !r->omega || !r->um || !r->uij || !r->t_ts || !r->t_ls) return bad("missing table");
    if (!ctx->have_grid) { ctx->err = "rfg_set: set the grid first (the inflow nodes' coordinates)"; return DESALM_ENOTREADY; }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  rfg_free(ctx);
  if (!r || r->nmodes == 0) return 0;
  const Level& F = ctx->L[0];
  const size_t nm = (size_t)r->nmodes, njk = (size_t)F.jm * F.km;
  std::vector<double> modes(nm * RFG_MODE);
  for (size_t i = 0; i < nm; ++i) {
    double* o = &modes[i * RFG_MODE];
    for (int d = 0; d < 3; ++d) {
      o[d] = r->p[3 * i + d];
      o[3 + d] = r->q[3 * i + d];
      o[6 + d] = r->k[3 * i + d];
    }
    o[9] = r->omega[i];
  }
  RfgDev& D = ctx->rfg.dev;
  auto up = [&](const double* h, size_t n, const double** out) -> int {
    void* d = nullptr;
    if (dalloc(ctx, ctx->rfg.allocs, &d, n * sizeof(double))) return DESALM_ENOMEM;
    if (h) CK(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    *out = (const double*)d;
    return 0;
  };
  int rc = 0;
  const double* tmp = nullptr;
  if (!rc) rc = up(modes.data(), nm * RFG_MODE, &D.modes);
  if (!rc) rc = up(r->um, 3 * njk, &D.um);
  if (!rc) rc = up(r->uij, 6 * njk, &D.uij);
  if (!rc) rc = up(r->t_ts, njk, &D.ts);
  if (!rc) rc = up(r->t_ls, njk, &D.ls);
  if (!rc) { rc = up(nullptr, RFG_NODE * njk, &tmp); D.node = const_cast<double*>(tmp); }
  if (!rc) { rc = up(nullptr, 3 * njk, &tmp); D.x1 = const_cast<double*>(tmp); }
  int* dbad = nullptr;
  if (!rc && dalloc(ctx, ctx->rfg.allocs, (void**)&dbad, sizeof(int))) rc = DESALM_ENOMEM;
  if (rc) { rfg_free(ctx); return rc; }
  D.nm = r->nmodes;
  D.im = F.im; D.jm = F.jm; D.km = F.km;
  CK(cudaMemsetAsync(dbad, 0, sizeof(int), ctx->stream));
  const long nn = (long)(F.jm - 2) * (F.km - 2);
  LAUNCH(KC_MISC, 0, double(nn), launch_k(k_rfg_prep, cdiv(nn, RFG_THREADS), RFG_THREADS, 0, ctx->stream, D,
                                          (const double*)ctx->x, (const double*)ctx->y, (const double*)ctx->z, dbad));
  CKL();
  int hbad = 0;
  CK(cudaMemcpyAsync(&hbad, dbad, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (hbad) {
    rfg_free(ctx);
    return bad(std::to_string(hbad) + " inflow nodes have a correlation tensor that is not positive definite, "
               "or a time or length scale that is not positive");
  }
  ctx->rfg.on = true;
  return 0;
}

int desalm_rfg_inlet(desalm_ctx* ctx, double time) {
  if (!ctx) return DESALM_EINVAL;
  if (!ctx->rfg.on) { ctx->err = "rfg_inlet: no generator tables (desalm_rfg_set)"; return DESALM_EINVAL; }
  if (!ctx->have_state) { ctx->err = "rfg_inlet: state not set"; return DESALM_ENOTREADY; }
  RET(rfg_launch(ctx, time));
  ctx->rfg.time = time;
  ctx->rfg.armed = true;
  return 0;
}

}  // extern "C"

// ------------------------------------------------------------ overset blocks
// Blocks of an overset grid exchange donor data inside the V-cycle: after
// each fine-level turbulence update the donee nodes of every block receive the
// turbulence fields trilinearly interpolated from their host cells in other
// blocks (mg_bintp_tur), and after each fine-level DAF step the momentum
// fields q(1:4) (mg_bintp_mom, src/mg_bintp_mom.F90:100-122; called at
// src/mg_driver.F90:237-244).  The reference sends the values with
// mpi_alltoallv between the ranks of different zones; here every block is a
// context on the same GPU, and the exchange is a gather of all interpolated
// values (reads of the host blocks' current fields) followed by a scatter
// into the donee blocks, on a stream that waits for every block and that
// every block then waits for.
namespace {

struct OvEntry {
  int db, dl;        // donee block, node index (0-based, i fastest)
  int hb, hl;        // host block, node index of the host cell's lower corner
  int hsj, hsk;      // the host block's j and k strides
  double c[3];       // xco, yco, zco
};

// Trilinear weights and corners in the reference's order (v000, v100, v010,
// v001, v101, v011, v110, v111; src/mg_bintp_mom.F90:100-122).  Fields
// f0..f1-1 of the per-block table tab[block * 6 + field] (q(1..5), omega).
__global__ void k_ov_gather(const OvEntry* E, int n, double* const* tab, int f0, int f1, double* buf) {
  pdl_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const OvEntry& x = E[e];
  const double xco = x.c[0], yco = x.c[1], zco = x.c[2], one = 1.0;
  const double c000 = (one - xco) * (one - yco) * (one - zco);
  const double c100 = xco * (one - yco) * (one - zco);
  const double c010 = (one - xco) * yco * (one - zco);
  const double c001 = (one - xco) * (one - yco) * zco;
  const double c101 = xco * (one - yco) * zco;
  const double c011 = (one - xco) * yco * zco;
  const double c110 = xco * yco * (one - zco);
  const double c111 = xco * yco * zco;
  const int l = x.hl, sj = x.hsj, sk = x.hsk;
  for (int f = f0; f < f1; ++f) {
    const double* v = tab[x.hb * 6 + f];
    buf[(size_t)e * 6 + f] = v[l] * c000 + v[l + 1] * c100 + v[l + sj] * c010 + v[l + sk] * c001 +
                             v[l + 1 + sk] * c101 + v[l + sj + sk] * c011 + v[l + 1 + sj] * c110 +
                             v[l + 1 + sj + sk] * c111;
  }
}

__global__ void k_ov_scatter(const OvEntry* E, int n, double* const* tab, int f0, int f1, const double* buf) {
  pdl_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const OvEntry& x = E[e];
  for (int f = f0; f < f1; ++f) tab[x.db * 6 + f][x.dl] = buf[(size_t)e * 6 + f];
}

// Point lists of a rank's share of a sharded overset exchange: the
// interpolated values of fields f0..f1-1 packed point-major, nf = f1 - f0 per
// point (the send buffer of src/mg_bintp_mom.F90:100-135 for one
// destination after another), and their write into donee nodes.
__global__ void k_ovl_gather(const OvEntry* E, int n, double* const* tab, int f0, int f1, double* buf) {
  pdl_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const OvEntry& x = E[e];
  const double xco = x.c[0], yco = x.c[1], zco = x.c[2], one = 1.0;
  const double c000 = (one - xco) * (one - yco) * (one - zco);
  const double c100 = xco * (one - yco) * (one - zco);
  const double c010 = (one - xco) * yco * (one - zco);
  const double c001 = (one - xco) * (one - yco) * zco;
  const double c101 = xco * (one - yco) * zco;
  const double c011 = (one - xco) * yco * zco;
  const double c110 = xco * yco * (one - zco);
  const double c111 = xco * yco * zco;
  const int l = x.hl, sj = x.hsj, sk = x.hsk, nf = f1 - f0;
  for (int f = f0; f < f1; ++f) {
    const double* v = tab[x.hb * 6 + f];
    buf[(size_t)e * nf + (f - f0)] = v[l] * c000 + v[l + 1] * c100 + v[l + sj] * c010 + v[l + sk] * c001 +
                                     v[l + 1 + sk] * c101 + v[l + sj + sk] * c011 + v[l + 1 + sj] * c110 +
                                     v[l + 1 + sj + sk] * c111;
  }
}

__global__ void k_ovl_scatter(const OvEntry* E, int n, double* const* tab, int f0, int f1, const double* buf) {
  pdl_wait();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const OvEntry& x = E[e];
  const int nf = f1 - f0;
  for (int f = f0; f < f1; ++f) tab[x.db * 6 + f][x.dl] = buf[(size_t)e * nf + (f - f0)];
}

}  // namespace

struct desalm_ov_list {
  std::vector<desalm_ctx*> blocks;
  int n = 0;
  bool gather = false;             // host cells and weights (else donee nodes)
  OvEntry* entries = nullptr;      // device
  double** tab = nullptr;          // device [blocks][6] field pointers of each block's fine level
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<cudaEvent_t> bev;
  std::string err;
};

namespace {

// Device field table [block][6] of the blocks' fine levels: q(1..5), omega.
int ov_field_table(desalm_ctx* const* ctxs, int nblocks, std::vector<double*>& tab) {
  tab.assign(6L * nblocks, nullptr);
  for (int b = 0; b < nblocks; ++b) {
    for (int f = 0; f < 5; ++f) {
      void* p = nullptr;
      int esz = 0;
      if (field_ptr(ctxs[b], 0, DESALM_F_Q + f, &p, &esz) || esz != 8) return DESALM_EINVAL;
      tab[6 * b + f] = (double*)p;
    }
    tab[6 * b + 5] = ctxs[b]->c.turbulence == 2 ? ctxs[b]->kw.a[0] : nullptr;
  }
  return 0;
}

}  // namespace

struct desalm_overset {
  std::vector<desalm_ctx*> blocks;
  int n = 0;                       // donee nodes
  OvEntry* entries = nullptr;      // device
  double** tab = nullptr;          // device [blocks][6] field pointers of each block's fine level
  double* buf = nullptr;           // device [n][6]
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  std::vector<cudaEvent_t> bev;    // one per block
  std::string err;
};

namespace {

int ov_fail(desalm_overset* ov, const std::string& why, int code) {
  ov->err = why;
  return code;
}

// The exchange of fields f0..f1-1 after every block's queued work.
int ov_exchange(desalm_overset* ov, int f0, int f1) {
  if (ov->n == 0) return 0;
  const int nb = (int)ov->blocks.size();
  for (int b = 0; b < nb; ++b) {
    if (cudaEventRecord(ov->bev[b], ov->blocks[b]->stream) != cudaSuccess ||
        cudaStreamWaitEvent(ov->s, ov->bev[b], 0) != cudaSuccess)
      return ov_fail(ov, "overset: event", DESALM_ECUDA);
  }
  const unsigned g = (unsigned)((ov->n + 127) / 128);
  if (launch_k(k_ov_gather, g, 128, 0, ov->s, (const OvEntry*)ov->entries, ov->n, (double* const*)ov->tab, f0, f1,
               ov->buf) != cudaSuccess ||
      launch_k(k_ov_scatter, g, 128, 0, ov->s, (const OvEntry*)ov->entries, ov->n, (double* const*)ov->tab, f0, f1,
               (const double*)ov->buf) != cudaSuccess)
    return ov_fail(ov, "overset: exchange launch", DESALM_ECUDA);
  if (cudaEventRecord(ov->ev, ov->s) != cudaSuccess) return ov_fail(ov, "overset: event", DESALM_ECUDA);
  for (int b = 0; b < nb; ++b)
    if (cudaStreamWaitEvent(ov->blocks[b]->stream, ov->ev, 0) != cudaSuccess)
      return ov_fail(ov, "overset: event", DESALM_ECUDA);
  return 0;
}

int ov_turb_fields(const desalm_ctx* ctx, int& f0, int& f1) {
  f0 = 4;
  f1 = ctx->c.turbulence == 2 ? 6 : (ctx->c.turbulence == 1 ? 5 : 4);
  return 0;
}

}  // namespace

extern "C" {

int desalm_overset_create(desalm_ctx* const* ctxs, int nblocks, const desalm_overset_map* map, desalm_overset** out) {
  if (!ctxs || nblocks < 1 || !map || !out || map->n < 0 || (map->n > 0 && (!map->donee || !map->host || !map->coef)))
    return DESALM_EINVAL;
  *out = nullptr;
  for (int b = 0; b < nblocks; ++b) {
    if (!ctxs[b]) return DESALM_EINVAL;
    const desalm_case& a = ctxs[0]->c;
    const desalm_case& c = ctxs[b]->c;
    bool same = c.ng == a.ng && c.itmax == a.itmax && c.it_min == a.it_min && c.er_min == a.er_min &&
                c.eo_min == a.eo_min && c.turbulence == a.turbulence && c.wall_functions == a.wall_functions;
    for (int n = 0; n < 4; ++n) same = same && c.iter[n] == a.iter[n];
    if (!same) {
      ctxs[b]->err = "overset blocks must share ng, iter, itmax, it_min, er_min, eo_min, the turbulence model and "
                     "the wall-function switch";
      return DESALM_EINVAL;
    }
  }
  std::vector<OvEntry> E(map->n);
  for (int e = 0; e < map->n; ++e) {
    const int* d = map->donee + 4 * e;
    const int* h = map->host + 4 * e;
    if (d[0] < 0 || d[0] >= nblocks || h[0] < 0 || h[0] >= nblocks) return DESALM_EINVAL;
    const Level& D = ctxs[d[0]]->L[0];
    const Level& H = ctxs[h[0]]->L[0];
    if (d[1] < 1 || d[1] > D.im || d[2] < 1 || d[2] > D.jm || d[3] < 1 || d[3] > D.km) return DESALM_EINVAL;
    // the host cell's eight corners lie inside the host block
    if (h[1] < 1 || h[1] > H.im - 1 || h[2] < 1 || h[2] > H.jm - 1 || h[3] < 1 || h[3] > H.km - 1) return DESALM_EINVAL;
    OvEntry& x = E[e];
    x.db = d[0];
    x.dl = (d[1] - 1) + D.im * ((d[2] - 1) + D.jm * (d[3] - 1));
    x.hb = h[0];
    x.hl = (h[1] - 1) + H.im * ((h[2] - 1) + H.jm * (h[3] - 1));
    x.hsj = H.im;
    x.hsk = H.im * H.jm;
    for (int t = 0; t < 3; ++t) x.c[t] = map->coef[3 * e + t];
  }
  std::vector<double*> tab;
  RET(ov_field_table(ctxs, nblocks, tab));
  desalm_overset* ov = new desalm_overset();
  ov->blocks.assign(ctxs, ctxs + nblocks);
  ov->n = map->n;
  bool ok = cudaMalloc((void**)&ov->entries, std::max<size_t>(1, E.size()) * sizeof(OvEntry)) == cudaSuccess &&
            cudaMalloc((void**)&ov->tab, tab.size() * sizeof(double*)) == cudaSuccess &&
            cudaMalloc((void**)&ov->buf, std::max<size_t>(1, 6 * E.size()) * sizeof(double)) == cudaSuccess &&
            cudaStreamCreateWithFlags(&ov->s, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&ov->ev, cudaEventDisableTiming) == cudaSuccess;
  ov->bev.assign(nblocks, nullptr);
  for (int b = 0; b < nblocks && ok; ++b) ok = cudaEventCreateWithFlags(&ov->bev[b], cudaEventDisableTiming) == cudaSuccess;
  if (ok && !E.empty()) ok = cudaMemcpy(ov->entries, E.data(), E.size() * sizeof(OvEntry), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok) ok = cudaMemcpy(ov->tab, tab.data(), tab.size() * sizeof(double*), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    desalm_overset_destroy(ov);
    return DESALM_ENOMEM;
  }
  *out = ov;
  return 0;
}

void desalm_overset_destroy(desalm_overset* ov) {
  if (!ov) return;
  if (ov->s) cudaStreamSynchronize(ov->s);
  cudaFree(ov->entries);
  cudaFree(ov->tab);
  cudaFree(ov->buf);
  for (cudaEvent_t e : ov->bev)
    if (e) cudaEventDestroy(e);
  if (ov->ev) cudaEventDestroy(ov->ev);
  if (ov->s) cudaStreamDestroy(ov->s);
  delete ov;
}

const char* desalm_overset_last_error(const desalm_overset* ov) { return ov ? ov->err.c_str() : "null overset"; }

int desalm_overset_exchange(desalm_overset* ov, int what) {
  if (!ov || (what != 0 && what != 1)) return DESALM_EINVAL;
  int f0 = 0, f1 = 4;
  if (what == 1) ov_turb_fields(ov->blocks[0], f0, f1);
  RET(ov_exchange(ov, f0, f1));
  for (desalm_ctx* b : ov->blocks)
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return ov_fail(ov, "overset: synchronize", DESALM_ECUDA);
  return 0;
}

int desalm_ov_list_create(desalm_ctx* const* ctxs, int nctx, int n, const int* pts, const double* coef,
                          desalm_ov_list** out) {
  if (!ctxs || nctx < 1 || n < 0 || !out || (n > 0 && !pts)) return DESALM_EINVAL;
  *out = nullptr;
  for (int b = 0; b < nctx; ++b)
    if (!ctxs[b] || ctxs[b]->c.turbulence != ctxs[0]->c.turbulence) return DESALM_EINVAL;
  std::vector<OvEntry> E(n);
  for (int e = 0; e < n; ++e) {
    const int* q = pts + 4 * e;
    if (q[0] < 0 || q[0] >= nctx) return DESALM_EINVAL;
    const Level& G = ctxs[q[0]]->L[0];
    OvEntry& x = E[e];
    const int l = (q[1] - 1) + G.im * ((q[2] - 1) + G.jm * (q[3] - 1));
    if (coef) {
      // the host cell's eight corners lie inside the block
      if (q[1] < 1 || q[1] > G.im - 1 || q[2] < 1 || q[2] > G.jm - 1 || q[3] < 1 || q[3] > G.km - 1) return DESALM_EINVAL;
      x.hb = q[0];
      x.hl = l;
      x.hsj = G.im;
      x.hsk = G.im * G.jm;
      for (int t = 0; t < 3; ++t) x.c[t] = coef[3 * e + t];
      x.db = 0;
      x.dl = 0;
    } else {
      if (q[1] < 1 || q[1] > G.im || q[2] < 1 || q[2] > G.jm || q[3] < 1 || q[3] > G.km) return DESALM_EINVAL;
      x.db = q[0];
      x.dl = l;
      x.hb = 0;
      x.hl = 0;
      x.hsj = x.hsk = 0;
      x.c[0] = x.c[1] = x.c[2] = 0.0;
    }
  }
  std::vector<double*> tab;
  RET(ov_field_table(ctxs, nctx, tab));
  desalm_ov_list* L = new desalm_ov_list();
  L->blocks.assign(ctxs, ctxs + nctx);
  L->n = n;
  L->gather = coef != nullptr;
  bool ok = cudaMalloc((void**)&L->entries, std::max<size_t>(1, E.size()) * sizeof(OvEntry)) == cudaSuccess &&
            cudaMalloc((void**)&L->tab, tab.size() * sizeof(double*)) == cudaSuccess &&
            cudaStreamCreateWithFlags(&L->s, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&L->ev, cudaEventDisableTiming) == cudaSuccess;
  L->bev.assign(nctx, nullptr);
  for (int b = 0; b < nctx && ok; ++b) ok = cudaEventCreateWithFlags(&L->bev[b], cudaEventDisableTiming) == cudaSuccess;
  if (ok && !E.empty()) ok = cudaMemcpy(L->entries, E.data(), E.size() * sizeof(OvEntry), cudaMemcpyHostToDevice) == cudaSuccess;
  if (ok) ok = cudaMemcpy(L->tab, tab.data(), tab.size() * sizeof(double*), cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok) {
    desalm_ov_list_destroy(L);
    return DESALM_ENOMEM;
  }
  *out = L;
  return 0;
}

void desalm_ov_list_destroy(desalm_ov_list* L) {
  if (!L) return;
  if (L->s) cudaStreamSynchronize(L->s);
  cudaFree(L->entries);
  cudaFree(L->tab);
  for (cudaEvent_t e : L->bev)
    if (e) cudaEventDestroy(e);
  if (L->ev) cudaEventDestroy(L->ev);
  if (L->s) cudaStreamDestroy(L->s);
  delete L;
}

const char* desalm_ov_list_last_error(const desalm_ov_list* L) { return L ? L->err.c_str() : "null list"; }

int desalm_ov_list_fields(const desalm_ov_list* L, int what) {
  if (!L || (what != 0 && what != 1)) return DESALM_EINVAL;
  if (what == 0) return 4;
  int f0 = 0, f1 = 0;
  ov_turb_fields(L->blocks[0], f0, f1);
  return f1 - f0;
}

namespace {
// The list's kernel on its stream after every block's queued work, the
// blocks' streams after it, then the list's stream drained (the buffer is
// the caller's once this returns).
int ovl_run(desalm_ov_list* L, int what, double* buf) {
  if (!L || (what != 0 && what != 1) || (L->n > 0 && !buf)) return DESALM_EINVAL;
  if (L->n == 0) return 0;
  int f0 = 0, f1 = 4;
  if (what == 1) ov_turb_fields(L->blocks[0], f0, f1);
  if (f1 == f0) return 0;
  const int nb = (int)L->blocks.size();
  for (int b = 0; b < nb; ++b)
    if (cudaEventRecord(L->bev[b], L->blocks[b]->stream) != cudaSuccess || cudaStreamWaitEvent(L->s, L->bev[b], 0) != cudaSuccess) {
      L->err = "overset list: event";
      return DESALM_ECUDA;
    }
  const unsigned g = (unsigned)((L->n + 127) / 128);
  cudaError_t e = L->gather
                      ? launch_k(k_ovl_gather, g, 128, 0, L->s, (const OvEntry*)L->entries, L->n, (double* const*)L->tab, f0, f1, buf)
                      : launch_k(k_ovl_scatter, g, 128, 0, L->s, (const OvEntry*)L->entries, L->n, (double* const*)L->tab, f0, f1,
                                 (const double*)buf);
  if (e == cudaSuccess) e = cudaEventRecord(L->ev, L->s);
  for (int b = 0; b < nb && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(L->blocks[b]->stream, L->ev, 0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(L->s);
  if (e != cudaSuccess) {
    L->err = std::string("overset list: ") + cudaGetErrorString(e);
    return DESALM_ECUDA;
  }
  return 0;
}
}  // namespace

int desalm_ov_list_gather(desalm_ov_list* L, int what, double* out) {
  if (L && !L->gather) { L->err = "not a gather list (created without weights)"; return DESALM_EINVAL; }
  return ovl_run(L, what, out);
}

int desalm_ov_list_scatter(desalm_ov_list* L, int what, const double* in) {
  if (L && L->gather) { L->err = "not a scatter list (created with weights)"; return DESALM_EINVAL; }
  return ovl_run(L, what, const_cast<double*>(in));
}

int desalm_overset_mg_driver(desalm_overset* ov, desalm_step_report* reps) {
  if (!ov) return DESALM_EINVAL;
  const int nb = (int)ov->blocks.size();
  desalm_ctx* c0 = ov->blocks[0];
  const desalm_case& c = c0->c;
  for (desalm_ctx* b : ov->blocks) {
    const int rc = desalm_begin_step(b);
    if (rc) return ov_fail(ov, std::string("overset: begin_step: ") + b->err, rc);
  }
  int tf0 = 4, tf1 = 4;
  ov_turb_fields(c0, tf0, tf1);
  double init_resd[5] = {0, 0, 0, 0, 0}, res[5] = {0, 0, 0, 0, 0};
  bool conv = false;
  int itc = 0, piv = 0, plines = 0;
  // interior nodes of block 0: the reference divides the sum over every zone
  // by its root's zone's count (src/mg_residual.F90:31,80)
  const Level& G0 = c0->L[0];
  const double tnu0 = double(G0.im - 2) * (G0.jm - 2) * (G0.km - 2);
  while (!conv && itc < c.itmax) {
    ++itc;
    for (desalm_ctx* b : ov->blocks) b->itc = itc;
    for (int itr = 1; itr <= c.iter[0]; ++itr) {
      for (desalm_ctx* b : ov->blocks) {
        const int rc = enqueue_fine(b, itr, 0);
        if (rc) return ov_fail(ov, std::string("overset: ") + b->err, rc);
      }
      if (tf1 > tf0) RET(ov_exchange(ov, tf0, tf1));
      for (desalm_ctx* b : ov->blocks) {
        const int rc = enqueue_fine(b, itr, 1);
        if (rc) return ov_fail(ov, std::string("overset: ") + b->err, rc);
      }
      RET(ov_exchange(ov, 0, 4));
    }
    double sum[5] = {0, 0, 0, 0, 0};
    for (desalm_ctx* b : ov->blocks) {  // every block's coarse levels in flight at once
      const int rc = enqueue_coarse(b);
      if (rc) return ov_fail(ov, std::string("overset: ") + b->err, rc);
    }
    for (int bi = 0; bi < nb; ++bi) {
      desalm_ctx* b = ov->blocks[bi];
      double r[5];
      const int rc = do_norm(b, 0, 1, r);   // also qold_mg <- q for the next iteration
      if (rc) return ov_fail(ov, std::string("overset: ") + b->err, rc);
      for (int m = 0; m < 5; ++m) sum[m] += b->h_norm[m];   // the block's sum of |q - qold_mg|
      int hflags[3] = {0, 0, 0};
      if (cudaMemcpy(hflags, b->flags, 3 * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return ov_fail(ov, "overset: flags", DESALM_ECUDA);
      if (hflags[1]) return ov_fail(ov, "overset: zero pivot in a line solve", DESALM_ESINGULAR);
      piv += hflags[0];
      plines += hflags[2];
    }
    for (int m = 0; m < 5; ++m) res[m] = std::log10(sum[m] / tnu0);
    if (itc == 1)
      for (int m = 0; m < 5; ++m) init_resd[m] = res[m];
    for (int m = 1; m < 4; ++m)
      if (!std::isfinite(res[m])) return ov_fail(ov, "overset: non-finite convergence norm", DESALM_ENONFINITE);
    // mg_ck_conver (src/mg_driver.F90:372-398) on the combined norm
    const double eomax = std::max(res[1], std::max(res[2], res[3]));
    const double ermax = std::max(res[1] - init_resd[1], std::max(res[2] - init_resd[2], res[3] - init_resd[3]));
    conv = (itc > c.it_min && ermax < c.er_min) || (itc > c.it_min && eomax < c.eo_min);
  }
  if (reps)
    for (int bi = 0; bi < nb; ++bi) {
      desalm_step_report& r = reps[bi];
      r.iterations = itc;
      r.converged = conv ? 1 : 0;
      for (int m = 0; m < 5; ++m) { r.residual[m] = res[m]; r.init_residual[m] = init_resd[m]; }
      r.pivots = piv;
      r.pivot_lines = plines;
    }
  return 0;
}

}  // extern "C"
