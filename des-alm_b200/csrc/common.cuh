// common.cuh -- shared device types and helpers of the B200 DES-ALM path.
//
// Layout in HBM: one structure-of-arrays block per multigrid level.  Every
// field is a contiguous array of im*jm*km values, i fastest, then j, then k
// (the reference's Fortran order, src/init.F90:917-937, without concatenating
// the levels).  Node (i, j, k) with 0-based indices lives at
// i + im*(j + jm*k); interior nodes are 1..im-2 etc.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DESALM_DEV __device__ __forceinline__
#define DESALM_HD __host__ __device__

namespace desalm {

// Per-level device view passed by value to the kernels.  T is the storage and
// arithmetic type of the level's state (double; float for coarse levels in
// MIXED mode), W the type of the DAF work arrays (line sweeps).
template <class T, class W>
struct Lv {
  int im, jm, km;
  int N;           // im*jm*km
  int sj, sk;      // strides of j and k (im, im*jm)
  T dc, de, dz;    // inverse spacings dc(n) (src/init.F90:1117-1121)
  // state
  T* q[5];
  T* qn[5];
  T* qnm1[5];
  T* qold[5];
  T* rh[4];        // raw residual (restriction input), boundary nodes stay 0
  T* pk[4];        // FAS forcing
  T* nut;
  T* dtau;
  T* dtc;          // metric parts of dtau: the largest convective limit
  T* dtv;          // reciprocal, and the viscous one without (1/Re + nu_t)
  T* diss1;        // diss(1) of the first residual pass (reused by the recalc)
  // geometry
  const T* csi[3];
  const T* eta[3];
  const T* zet[3];
  const T* aj;
  const T* rj;      // 1/aj, formed once whenever aj is set
  const T* falm;    // actuator-line force added to rh(2:4), [3][N], or null
  const W* mw[9];   // csi, eta, zet rounded to W once (the same arrays when
                    // W = T): the modal transforms of the sweeps read these
  // DAF work: transformed residual and row coefficients
  W* wk[4];
  W* sig;          // sigma = sqrt(beta alpha) of each interior node, from the first residual pass
  W* tc[3];        // per direction: tmp = dtau ep spr dsq (diagonal part of each row)
  W* hc[3];        // per direction: dtau (dxi/2) spr (neighbour coupling of the
                   // characteristic rows); also set on the boundary nodes that
                   // precede/follow the interior lines
  W* bi;           // i-face boundary vectors: [2][4][jm*km]
  W* bj;           // j-face: [4][4][im*km]  (rows 2, 3, jm-1, jm-2 after the i sweep)
  W* bk;           // k-face: [4][4][im*jm]
  W* gs;           // line-solve scratch of k_gsweep: 16 arrays gss elements apart
  int gss;
  int* flags;      // [0] rows interchanged, [1] zero pivots, [2] line systems solved by the pivoting path
  int oute;        // 1: the characteristics outlet plane i = im is solved
                   // with the interior (fine level, btype(2) = 5)
};

// Scalar parameters of the case used by kernels (constant per context).
struct Par {
  double ren, beta, delti, es;   // es = e_source
  double cfl1, vnn1, pdiss;
  double ep1[3], ep2[3];
  double sa[4][6], sb[4][6];     // src/init.F90:482-509
  int btype[6];
  int fine;                      // 1 when the level is the finest
};

// Elements of one field of a shared-memory line slab: np nodes of nlp-strided
// lines, rounded up to a multiple of 32 plus 16, so that consecutive fields
// start on different banks.
DESALM_HD inline int slab_fs(int np, int nlp) { return ((np * nlp + 31) / 32) * 32 + 16; }

// Threads of a slab CTA: all of them copy the slab in and out, the first
// 8 NL (DAF sweeps, rsmooth) or 2 NL (SA sweeps) solve the lines.
constexpr int kSlabThreads = 256;

// Programmatic dependent launch: every kernel of the library is launched with
// programmatic stream serialisation, so its launch is processed while the
// grid before it finishes; pdl_wait() then blocks until the grids it depends
// on have completed and their writes are visible.  Every kernel calls it
// before its first global-memory access.  No kernel signals an early launch
// of its dependents (griddepcontrol.launch_dependents): that lets the next
// grid's CTAs take SM resources while this one still runs, and measured
// slower.
DESALM_DEV void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

template <class T> DESALM_DEV T dabs(T x) { return x < T(0) ? -x : x; }

// The line eliminations write every multiply-add as an explicit fused
// (fmaw: a b + c rounded once) or separate (mulw) operation, so that the
// kernels that solve the same line systems (the shared-memory slab and the
// lines-in-lanes variants) round alike: left to the compiler, a b + c is
// contracted or not depending on the code around it.
DESALM_DEV float fmaw(float a, float b, float c) { return __fmaf_rn(a, b, c); }
DESALM_DEV double fmaw(double a, double b, double c) { return __fma_rn(a, b, c); }
DESALM_DEV float mulw(float a, float b) { return __fmul_rn(a, b); }
DESALM_DEV double mulw(double a, double b) { return __dmul_rn(a, b); }
// Drops the 128-byte L2 line at p (128-byte aligned) without writing it
// back: for line-solve scratch that has been read for the last time.
DESALM_DEV void l2_discard(const void* p) { asm volatile("discard.global.L2 [%0], 128;\n" ::"l"(p) : "memory"); }

// a b - c d as fma(a, b, -(c d)) with c d rounded first (the middle 2x2
// block of a two-ended elimination)
DESALM_DEV float fms2(float a, float b, float c, float d) { return __fmaf_rn(a, b, -__fmul_rn(c, d)); }
DESALM_DEV double fms2(double a, double b, double c, double d) { return __fma_rn(a, b, -__dmul_rn(c, d)); }
// a b + c d likewise
DESALM_DEV float fma2(float a, float b, float c, float d) { return __fmaf_rn(a, b, __fmul_rn(c, d)); }
DESALM_DEV double fma2(double a, double b, double c, double d) { return __fma_rn(a, b, __dmul_rn(c, d)); }

// Reciprocal used by the line eliminations: in FP32 (the sweeps of MIXED mode,
// a preconditioner) the hardware approximation __fdividef (2 ulp), in FP64 the
// correctly rounded division.
DESALM_DEV float sweep_rcp(float x) { return __fdividef(1.0f, x); }
DESALM_DEV double sweep_rcp(double x) { return 1.0 / x; }

// Asynchronous global -> shared copy of one 4- or 8-byte element
// (cp.async, cached in L1); completion by cp_async_wait_all().
template <class E>
DESALM_DEV void cp_async_elem(E* smem, const E* gmem) {
  static_assert(sizeof(E) == 4 || sizeof(E) == 8, "cp.async element size");
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (sizeof(E) == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
DESALM_DEV void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
template <class T> DESALM_DEV T dmin(T a, T b) { return a < b ? a : b; }
template <class T> DESALM_DEV T dmax(T a, T b) { return a > b ? a : b; }

}  // namespace desalm
