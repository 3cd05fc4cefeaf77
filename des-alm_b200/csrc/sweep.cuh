// sweep.cuh -- K_I / K_J / K_K: the three scalar tridiagonal line sweeps of
// the diagonal approximate factorisation (src/rhs_diag_solver.F90:74-633).
//
// One thread owns one grid line and solves its four scalar systems
// (eigenvalue multipliers 0, 0, +1, -1; systems 1 and 2 share one matrix).
// The elimination is LAPACK SGTSV's no-interchange branch (src/sgtsv.f:107-
// 121, 232-243) evaluated in the same order; a row where SGTSV would swap
// rows (|d_i| < |dl_i|) is counted in flags[0] and a zero pivot in flags[1],
// so a caller can see when the oracle's partial pivoting would have taken the
// other branch.  Coefficients are rebuilt from dtau and the metrics, the
// semi-explicit boundary rows (brh) are applied to the first/last interior
// rows, and the epilogue applies the next modal transform (N1^-1 after the
// i sweep, N2^-1 after the j sweep) or, after the k sweep, Mc and the update
// q <- q + dq (src/solver_daf.F90:409-418).
//
// j and k lines are coalesced across threads (consecutive i); i lines are
// contiguous per thread and rely on L1 for sector reuse.
#pragma once
#include "modal.cuh"

namespace desalm {

template <class T, class W>
DESALM_DEV T spr_at(const Lv<T, W>& L, const Par& P, const T* const* m, int l) {
  T s, t;
  sigma_theta(L.dtau[l], P, s, t);
  T g = m[0][l] * m[0][l] + m[1][l] * m[1][l] + m[2][l] * m[2][l];
  return t * sqrt(g);
}

// brh vector of a face: M(lb) * (sa o r1 + sb o r2)
template <class T, class W, int KIND>
DESALM_DEV void face_vec(const Lv<T, W>& L, const Par& P, int lb, int b, const W* r1, const W* r2, int stride, T out[4]) {
  T v[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) v[m] = T(P.sa[m][b]) * T(r1[m * stride]) + T(P.sb[m][b]) * T(r2[m * stride]);
  M4<T> A;
  if (KIND == 0) mat_mai(L, P, lb, A);
  else if (KIND == 1) mat_n1i(L, P, lb, A);
  else mat_n2i(L, P, lb, A);
  mv4(A, v, out);
}

template <class T, class W, int DIR>
__global__ void __launch_bounds__(128) k_sweep(Lv<T, W> L, Par P, int blo, int bhi) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int b = blockIdx.y + 1;
  int amax, n, st, lb;
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; st = 1; lb = L.sj * a + L.sk * b; }
  else if (DIR == 1) { amax = L.im - 2; n = L.jm - 2; st = L.sj; lb = a + L.sk * b; }
  else { amax = L.im - 2; n = L.km - 2; st = L.sk; lb = a + L.sj * b; }
  if (a > amax) return;
  const T* const* mt = DIR == 0 ? L.csi : (DIR == 1 ? L.eta : L.zet);
  const T dsp = DIR == 0 ? L.dc : (DIR == 1 ? L.de : L.dz);
  const T ep = T(P.ep1[DIR]);
  const T dsq = dsp * dsp;
  const T dh = T(0.5) * dsp;

  // semi-explicit boundary vectors (fine level only; flags from the host)
  T bw[4] = {0, 0, 0, 0}, be[4] = {0, 0, 0, 0};
  if (DIR == 0) {
    if (blo) {
      const int S = L.jm * L.km, o = a + L.jm * b;
      face_vec<T, W, 0>(L, P, lb, 0, L.bi + o, L.bi + 4 * S + o, S, bw);
    }
  } else if (DIR == 1) {
    const int S = L.im * L.km, o = a + L.im * b;
    if (blo) face_vec<T, W, 1>(L, P, lb, 2, L.bj + o, L.bj + 4 * S + o, S, bw);
    if (bhi) face_vec<T, W, 1>(L, P, lb + (n + 1) * st, 3, L.bj + 8 * S + o, L.bj + 12 * S + o, S, be);
  } else {
    const int S = L.im * L.jm, o = a + L.im * b;
    if (blo) face_vec<T, W, 2>(L, P, lb, 4, L.bk + o, L.bk + 4 * S + o, S, bw);
    if (bhi) face_vec<T, W, 2>(L, P, lb + (n + 1) * st, 5, L.bk + 8 * S + o, L.bk + 12 * S + o, S, be);
  }

  // ---- forward elimination
  T dtw = L.dtau[lb], sw = spr_at(L, P, mt, lb);
  T dt0 = L.dtau[lb + st], s0 = spr_at(L, P, mt, lb + st);
  T dp12 = 0, dp3 = 0, dp4 = 0, du12 = 0, du3 = 0, du4 = 0;
  T bp[4] = {0, 0, 0, 0};
  int npiv = 0, nzero = 0;
  for (int p = 0; p < n; ++p) {
    const int l = lb + (p + 1) * st;
    T dte = L.dtau[l + st], se = spr_at(L, P, mt, l + st);
    T dtc = dt0 == T(0) ? T(0) : T(1);
    T tmp = dt0 * ep * s0 * dsq;
    T ap = T(1) + T(2) * tmp;
    T ddsw = dtc * dtw * dh * sw;
    T ddse = dtc * dte * dh * se;
    T aw12 = -tmp, ae12 = -tmp;
    T aw3 = -ddsw - tmp, ae3 = ddse - tmp;
    T aw4 = ddsw - tmp, ae4 = -ddse - tmp;
    T r[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) r[m] = T(L.wk[m][l]);
    if (p == 0) {
      r[0] = r[0] - aw12 * bw[0]; r[1] = r[1] - aw12 * bw[1];
      r[2] = r[2] - aw3 * bw[2];  r[3] = r[3] - aw4 * bw[3];
    }
    if (p == n - 1) {
      r[0] = r[0] - ae12 * be[0]; r[1] = r[1] - ae12 * be[1];
      r[2] = r[2] - ae3 * be[2];  r[3] = r[3] - ae4 * be[3];
    }
    T d12, d3, d4;
    if (p == 0) {
      d12 = ap; d3 = ap; d4 = ap;
#pragma unroll
      for (int m = 0; m < 4; ++m) bp[m] = r[m];
    } else {
      npiv += (dabs(dp12) < dabs(aw12)) + (dabs(dp3) < dabs(aw3)) + (dabs(dp4) < dabs(aw4));
      nzero += (dp12 == T(0)) + (dp3 == T(0)) + (dp4 == T(0));
      T f12 = aw12 / dp12, f3 = aw3 / dp3, f4 = aw4 / dp4;
      d12 = ap - f12 * du12;
      d3 = ap - f3 * du3;
      d4 = ap - f4 * du4;
      bp[0] = r[0] - f12 * bp[0];
      bp[1] = r[1] - f12 * bp[1];
      bp[2] = r[2] - f3 * bp[2];
      bp[3] = r[3] - f4 * bp[3];
    }
    dp12 = d12; dp3 = d3; dp4 = d4;
    du12 = ae12; du3 = ae3; du4 = ae4;
    L.sd[0][l] = W(d12); L.sd[1][l] = W(d3); L.sd[2][l] = W(d4);
    L.su[0][l] = W(ae12); L.su[1][l] = W(ae3); L.su[2][l] = W(ae4);
#pragma unroll
    for (int m = 0; m < 4; ++m) L.wk[m][l] = W(bp[m]);
    dtw = dt0; sw = s0; dt0 = dte; s0 = se;
  }
  nzero += (dp12 == T(0)) + (dp3 == T(0)) + (dp4 == T(0));
  if (npiv) atomicAdd(&L.flags[0], npiv);
  if (nzero) atomicAdd(&L.flags[1], nzero);

  // ---- back substitution and epilogue
  T x[4];
  for (int p = n - 1; p >= 0; --p) {
    const int l = lb + (p + 1) * st;
    T d12 = T(L.sd[0][l]), d3 = T(L.sd[1][l]), d4 = T(L.sd[2][l]);
    T rb[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) rb[m] = T(L.wk[m][l]);
    if (p == n - 1) {
      x[0] = rb[0] / d12; x[1] = rb[1] / d12; x[2] = rb[2] / d3; x[3] = rb[3] / d4;
    } else {
      T u12 = T(L.su[0][l]), u3 = T(L.su[1][l]), u4 = T(L.su[2][l]);
      x[0] = (rb[0] - u12 * x[0]) / d12;
      x[1] = (rb[1] - u12 * x[1]) / d12;
      x[2] = (rb[2] - u3 * x[2]) / d3;
      x[3] = (rb[3] - u4 * x[3]) / d4;
    }
    if (DIR == 0) {
      // rows j = 2, 3, jm-1, jm-2 (1-based) feed the j-face boundary vectors
      const int S = L.im * L.km, o = (p + 1) + L.im * b;
      const int tgt[4] = {1, 2, L.jm - 2, L.jm - 3};
#pragma unroll
      for (int s = 0; s < 4; ++s)
        if (a == tgt[s])
#pragma unroll
          for (int m = 0; m < 4; ++m) L.bj[(s * 4 + m) * S + o] = W(x[m]);
      M4<T> A;
      mat_n1i(L, P, l, A);
      T y[4];
      mv4(A, x, y);
#pragma unroll
      for (int m = 0; m < 4; ++m) L.wk[m][l] = W(y[m]);
    } else if (DIR == 1) {
      // rows k = 2, 3, km-1, km-2 feed the k-face boundary vectors
      const int S = L.im * L.jm, o = a + L.im * (p + 1);
      const int tgt[4] = {1, 2, L.km - 2, L.km - 3};
#pragma unroll
      for (int s = 0; s < 4; ++s)
        if (b == tgt[s])
#pragma unroll
          for (int m = 0; m < 4; ++m) L.bk[(s * 4 + m) * S + o] = W(x[m]);
      M4<T> A;
      mat_n2i(L, P, l, A);
      T y[4];
      mv4(A, x, y);
#pragma unroll
      for (int m = 0; m < 4; ++m) L.wk[m][l] = W(y[m]);
    } else {
      M4<T> A;
      mat_mc(L, P, l, A);
      T y[4];
      mv4(A, x, y);
#pragma unroll
      for (int m = 0; m < 4; ++m) L.q[m][l] = L.q[m][l] + y[m];
    }
  }
}

}  // namespace desalm

namespace desalm {

// ---------------------------------------------------------------------------
// Second-generation sweep: one thread per (line, system).  A CTA owns 32
// lines; warp m solves system m of all 32 lines, so for j and k lines every
// row access is coalesced across the warp.  The row coefficients come from
// the per-node tc/hc arrays written by K_R (no spectral radii recomputed
// here).  The forward elimination keeps SGTSV's no-interchange order and
// writes the eliminated right-hand side in place and the eliminated diagonal
// to sd[m]; the back substitution leaves x in wk.  After a barrier, phase 2
// walks the CTA's nodes with coalesced indexing and applies the next modal
// transform (N1^-1, N2^-1) or Mc and the update q <- q + dq.
// ---------------------------------------------------------------------------
template <class T, class W, int DIR>
__global__ void __launch_bounds__(128) k_sweep2(Lv<T, W> L, Par P, int blo, int bhi) {
  __shared__ W sbw[32][4], sbe[32][4];
  const int lane = threadIdx.x & 31, m = threadIdx.x >> 5;
  const int a0 = blockIdx.x * 32 + 1;
  const int a = a0 + lane;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa;  // sa: stride between consecutive lines of the CTA
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; st = 1; sa = L.sj; }
  else if (DIR == 1) { amax = L.im - 2; n = L.jm - 2; st = L.sj; sa = 1; }
  else { amax = L.im - 2; n = L.km - 2; st = L.sk; sa = 1; }
  const int base = (DIR == 0) ? L.sk * b : (DIR == 1 ? L.sk * b : L.sj * b);  // line a = 0 at row -1
  const bool act = a <= amax;
  const int lb = base + a * sa;  // boundary node before the line

  // ---- phase 0: semi-explicit boundary vectors (fine level)
  if (m == 0) {
    T bw[4] = {0, 0, 0, 0}, be[4] = {0, 0, 0, 0};
    if (act) {
      if (DIR == 0) {
        if (blo) {
          const int S = L.jm * L.km, o = a + L.jm * b;
          face_vec<T, W, 0>(L, P, lb, 0, L.bi + o, L.bi + 4 * S + o, S, bw);
        }
      } else if (DIR == 1) {
        const int S = L.im * L.km, o = a + L.im * b;
        if (blo) face_vec<T, W, 1>(L, P, lb, 2, L.bj + o, L.bj + 4 * S + o, S, bw);
        if (bhi) face_vec<T, W, 1>(L, P, lb + (n + 1) * st, 3, L.bj + 8 * S + o, L.bj + 12 * S + o, S, be);
      } else {
        const int S = L.im * L.jm, o = a + L.im * b;
        if (blo) face_vec<T, W, 2>(L, P, lb, 4, L.bk + o, L.bk + 4 * S + o, S, bw);
        if (bhi) face_vec<T, W, 2>(L, P, lb + (n + 1) * st, 5, L.bk + 8 * S + o, L.bk + 12 * S + o, S, be);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) { sbw[lane][q] = W(bw[q]); sbe[lane][q] = W(be[q]); }
  }
  __syncthreads();

  // ---- phase 1: scalar tridiagonal solve of system m along the line.
  // Rows are processed in blocks of R: all loads of a block are issued
  // before any of its stores, so R rows of memory latency overlap.
  if (act) {
    constexpr int R = 8;
    const W bwm = sbw[lane][m], bem = sbe[lane][m];
    const W* tc = L.tc[DIR];
    const W* hc = L.hc[DIR];
    W* r = L.wk[m];
    W* sd = L.sd[m];
    W hw = hc[lb];            // h of the node before the current row
    W hcur = hc[lb + st];     // h of the current row's node
    W dprev = 0, duprev = 0, bprev = 0;
    int npiv = 0, nzero = 0;
    for (int p0 = 0; p0 < n; p0 += R) {
      W bt[R], bh[R], br[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p < n) {
          const int l = lb + (p + 1) * st;
          bt[u] = tc[l];
          bh[u] = hc[l + st];
          br[u] = r[l];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p < n) {
          const int l = lb + (p + 1) * st;
          const W t = bt[u];
          const W he = bh[u];
          const W dw = t != W(0) ? hw : W(0);
          const W de = t != W(0) ? he : W(0);
          W aw, ae;
          if (m < 2) { aw = -t; ae = -t; }
          else if (m == 2) { aw = -dw - t; ae = de - t; }
          else { aw = dw - t; ae = -de - t; }
          const W ap = W(1) + W(2) * t;
          W rr = br[u];
          if (p == 0) rr = rr - aw * bwm;
          if (p == n - 1) rr = rr - ae * bem;
          W d;
          if (p == 0) {
            d = ap;
            bprev = rr;
          } else {
            npiv += dabs(dprev) < dabs(aw);
            nzero += dprev == W(0);
            const W f = aw / dprev;
            d = ap - f * duprev;
            bprev = rr - f * bprev;
          }
          sd[l] = d;
          r[l] = bprev;
          dprev = d;
          duprev = ae;
          hw = hcur;
          hcur = he;
        }
      }
    }
    nzero += dprev == W(0);
    if (npiv) atomicAdd(&L.flags[0], npiv);
    if (nzero) atomicAdd(&L.flags[1], nzero);
    W x = 0;
    for (int p1 = n - 1; p1 >= 0; p1 -= R) {
      W bb[R], bd[R], bt[R], bh[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p1 - u;
        if (p >= 0) {
          const int l = lb + (p + 1) * st;
          bb[u] = r[l];
          bd[u] = sd[l];
          bt[u] = tc[l];
          bh[u] = hc[l + st];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p1 - u;
        if (p >= 0) {
          const int l = lb + (p + 1) * st;
          if (p == n - 1) {
            x = bb[u] / bd[u];
          } else {
            const W t = bt[u];
            const W de = t != W(0) ? bh[u] : W(0);
            W ae;
            if (m < 2) ae = -t;
            else if (m == 2) ae = de - t;
            else ae = -de - t;
            x = (bb[u] - ae * x) / bd[u];
          }
          r[l] = x;
        }
      }
    }
  }
  __syncthreads();

  // ---- phase 2: per-node transform of the CTA's lines
  const int nl = min(32, amax - a0 + 1);
  const int total = nl * n;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int li, p;
    if (DIR == 0) { li = t / n; p = t - li * n; }  // consecutive threads walk along i
    else { p = t / nl; li = t - p * nl; }          // consecutive threads walk across lines (i)
    const int aa = a0 + li;
    const int l = base + aa * sa + (p + 1) * st;
    T xv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) xv[q] = T(L.wk[q][l]);
    if (DIR == 0) {
      // rows j = 2, 3, jm-1, jm-2 (1-based) feed the j-face boundary vectors
      const int S = L.im * L.km, o = (p + 1) + L.im * b;
      const int tgt[4] = {1, 2, L.jm - 2, L.jm - 3};
#pragma unroll
      for (int s = 0; s < 4; ++s)
        if (aa == tgt[s])
#pragma unroll
          for (int q = 0; q < 4; ++q) L.bj[(s * 4 + q) * S + o] = W(xv[q]);
      M4<T> A;
      mat_n1i(L, P, l, A);
      T y[4];
      mv4(A, xv, y);
#pragma unroll
      for (int q = 0; q < 4; ++q) L.wk[q][l] = W(y[q]);
    } else if (DIR == 1) {
      const int S = L.im * L.jm, o = aa + L.im * (p + 1);
      const int tgt[4] = {1, 2, L.km - 2, L.km - 3};
#pragma unroll
      for (int s = 0; s < 4; ++s)
        if (b == tgt[s])
#pragma unroll
          for (int q = 0; q < 4; ++q) L.bk[(s * 4 + q) * S + o] = W(xv[q]);
      M4<T> A;
      mat_n2i(L, P, l, A);
      T y[4];
      mv4(A, xv, y);
#pragma unroll
      for (int q = 0; q < 4; ++q) L.wk[q][l] = W(y[q]);
    } else {
      M4<T> A;
      mat_mc(L, P, l, A);
      T y[4];
      mv4(A, xv, y);
#pragma unroll
      for (int q = 0; q < 4; ++q) L.q[q][l] = L.q[q][l] + y[q];
    }
  }
}

}  // namespace desalm

namespace desalm {

// ---------------------------------------------------------------------------
// Third-generation sweep: two-ended elimination.  A CTA owns 32 lines and
// has 8 warps: warp m (< 4) eliminates the upper half of system m top-down
// (SGTSV's no-interchange order), warp 4 + m eliminates the lower half
// bottom-up; the two meet in a 2x2 solve at the middle rows, then each warp
// back-substitutes its own half.  Twice the threads of k_sweep2 and half the
// dependent chain per line; the result differs from one top-down pass by
// round-off only.  Phase 2 (modal transform / update) is the same.
// ---------------------------------------------------------------------------
template <class T, class W, int DIR>
__global__ void __launch_bounds__(256) k_sweep3(Lv<T, W> L, Par P, int blo, int bhi) {
  __shared__ W sbw[32][4], sbe[32][4];
  __shared__ W mt_d[32][4], mt_u[32][4], mt_b[32][4];   // top half's last eliminated row
  __shared__ W mb_d[32][4], mb_l[32][4], mb_b[32][4];   // bottom half's last eliminated row
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m = w & 3, half = w >> 2;
  const int a0 = blockIdx.x * 32 + 1;
  const int a = a0 + lane;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa;
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; st = 1; sa = L.sj; }
  else if (DIR == 1) { amax = L.im - 2; n = L.jm - 2; st = L.sj; sa = 1; }
  else { amax = L.im - 2; n = L.km - 2; st = L.sk; sa = 1; }
  const int base = (DIR == 2) ? L.sj * b : L.sk * b;
  const bool act = a <= amax;
  const int lb = base + a * sa;
  const int h = n / 2;  // rows 0..h-1 top, h..n-1 bottom (n >= 3)

  if (w == 0) {
    T bw[4] = {0, 0, 0, 0}, be[4] = {0, 0, 0, 0};
    if (act) {
      if (DIR == 0) {
        if (blo) {
          const int S = L.jm * L.km, o = a + L.jm * b;
          face_vec<T, W, 0>(L, P, lb, 0, L.bi + o, L.bi + 4 * S + o, S, bw);
        }
      } else if (DIR == 1) {
        const int S = L.im * L.km, o = a + L.im * b;
        if (blo) face_vec<T, W, 1>(L, P, lb, 2, L.bj + o, L.bj + 4 * S + o, S, bw);
        if (bhi) face_vec<T, W, 1>(L, P, lb + (n + 1) * st, 3, L.bj + 8 * S + o, L.bj + 12 * S + o, S, be);
      } else {
        const int S = L.im * L.jm, o = a + L.im * b;
        if (blo) face_vec<T, W, 2>(L, P, lb, 4, L.bk + o, L.bk + 4 * S + o, S, bw);
        if (bhi) face_vec<T, W, 2>(L, P, lb + (n + 1) * st, 5, L.bk + 8 * S + o, L.bk + 12 * S + o, S, be);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) { sbw[lane][q] = W(bw[q]); sbe[lane][q] = W(be[q]); }
  }
  __syncthreads();

  const W* tc = L.tc[DIR];
  const W* hc = L.hc[DIR];
  W* r = L.wk[m];
  W* sd = L.sd[m];
  // row coefficients of system m: aw uses h of the west node, ae of the east
  auto coef = [&](W t, W hw_, W he_, W& aw, W& ae) {
    const W dw = t != W(0) ? hw_ : W(0);
    const W de = t != W(0) ? he_ : W(0);
    if (m < 2) { aw = -t; ae = -t; }
    else if (m == 2) { aw = -dw - t; ae = de - t; }
    else { aw = dw - t; ae = -de - t; }
  };
  constexpr int R = 8;
  int npiv = 0;
  if (act && half == 0) {
    // ---- top half, top-down
    const W bwm = sbw[lane][m];
    W hw = hc[lb], hcur = hc[lb + st];
    W dprev = 0, duprev = 0, bprev = 0;
    for (int p0 = 0; p0 < h; p0 += R) {
      W bt[R], bh[R], br[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p < h) { const int l = lb + (p + 1) * st; bt[u] = tc[l]; bh[u] = hc[l + st]; br[u] = r[l]; }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p < h) {
          const int l = lb + (p + 1) * st;
          W aw, ae;
          coef(bt[u], hw, bh[u], aw, ae);
          const W ap = W(1) + W(2) * bt[u];
          W rr = br[u];
          if (p == 0) rr = rr - aw * bwm;
          W d;
          if (p == 0) { d = ap; bprev = rr; }
          else {
            npiv += dabs(dprev) < dabs(aw);
            const W f = aw / dprev;
            d = ap - f * duprev;
            bprev = rr - f * bprev;
          }
          sd[l] = d;
          r[l] = bprev;
          dprev = d; duprev = ae;
          hw = hcur; hcur = bh[u];
        }
      }
    }
    mt_d[lane][m] = dprev; mt_u[lane][m] = duprev; mt_b[lane][m] = bprev;
  } else if (act && half == 1) {
    // ---- bottom half, bottom-up: eliminate the super-diagonal
    const W bem = sbe[lane][m];
    W he = hc[lb + (n + 1) * st];           // h of the node after the line
    W hcur = hc[lb + n * st];               // h of row n-1's node
    W dprev = 0, awprev = 0, bprev = 0;     // row p+1 after elimination, and its aw
    for (int p0 = n - 1; p0 >= h; p0 -= R) {
      W bt[R], bh[R], br[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 - u;
        if (p >= h) { const int l = lb + (p + 1) * st; bt[u] = tc[l]; bh[u] = hc[l - st]; br[u] = r[l]; }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 - u;
        if (p >= h) {
          const int l = lb + (p + 1) * st;
          W aw, ae;
          coef(bt[u], bh[u], he, aw, ae);
          const W ap = W(1) + W(2) * bt[u];
          W rr = br[u];
          if (p == n - 1) rr = rr - ae * bem;
          W d;
          if (p == n - 1) { d = ap; bprev = rr; }
          else {
            npiv += dabs(dprev) < dabs(ae);
            const W f = ae / dprev;
            d = ap - f * awprev;
            bprev = rr - f * bprev;
          }
          sd[l] = d;
          r[l] = bprev;
          dprev = d; awprev = aw;
          he = hcur; hcur = bh[u];
        }
      }
    }
    mb_d[lane][m] = dprev; mb_l[lane][m] = awprev; mb_b[lane][m] = bprev;
  }
  if (npiv) atomicAdd(&L.flags[0], npiv);
  __syncthreads();
  if (act) {
    // ---- the two middle rows: d1 x1 + u1 x2 = b1 (row h-1), l2 x1 + d2 x2 = b2 (row h)
    const W d1 = mt_d[lane][m], u1 = mt_u[lane][m], b1 = mt_b[lane][m];
    const W d2 = mb_d[lane][m], l2 = mb_l[lane][m], b2 = mb_b[lane][m];
    const W det = d1 * d2 - u1 * l2;
    const W x1 = (b1 * d2 - u1 * b2) / det;
    const W x2 = (d1 * b2 - l2 * b1) / det;
    if (half == 0) {
      W x = x1;
      r[lb + h * st] = x1;
      for (int p1 = h - 2; p1 >= 0; p1 -= R) {
        W bb[R], bd[R], bt[R], bh[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
          const int p = p1 - u;
          if (p >= 0) { const int l = lb + (p + 1) * st; bb[u] = r[l]; bd[u] = sd[l]; bt[u] = tc[l]; bh[u] = hc[l + st]; }
        }
#pragma unroll
        for (int u = 0; u < R; ++u) {
          const int p = p1 - u;
          if (p >= 0) {
            W aw, ae;
            coef(bt[u], W(0), bh[u], aw, ae);
            x = (bb[u] - ae * x) / bd[u];
            r[lb + (p + 1) * st] = x;
          }
        }
      }
    } else {
      W x = x2;
      r[lb + (h + 1) * st] = x2;
      for (int p0 = h + 1; p0 < n; p0 += R) {
        W bb[R], bd[R], bt[R], bh[R];
#pragma unroll
        for (int u = 0; u < R; ++u) {
          const int p = p0 + u;
          if (p < n) { const int l = lb + (p + 1) * st; bb[u] = r[l]; bd[u] = sd[l]; bt[u] = tc[l]; bh[u] = hc[l - st]; }
        }
#pragma unroll
        for (int u = 0; u < R; ++u) {
          const int p = p0 + u;
          if (p < n) {
            W aw, ae;
            coef(bt[u], bh[u], W(0), aw, ae);
            x = (bb[u] - aw * x) / bd[u];
            r[lb + (p + 1) * st] = x;
          }
        }
      }
    }
  }
  __syncthreads();

  // ---- phase 2: per-node transform of the CTA's lines, in the sweep
  // precision W (FP64 in FP64 mode, FP32 in MIXED mode)
  const int nl = min(32, amax - a0 + 1);
  const int total = nl * n;
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    int li, p;
    if (DIR == 0) { li = t / n; p = t - li * n; }
    else { p = t / nl; li = t - p * nl; }
    const int aa = a0 + li;
    const int l = base + aa * sa + (p + 1) * st;
    W xv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) xv[q] = L.wk[q][l];
    if (DIR == 0) {
      const int S = L.im * L.km, o = (p + 1) + L.im * b;
      const int tgt[4] = {1, 2, L.jm - 2, L.jm - 3};
#pragma unroll
      for (int s = 0; s < 4; ++s)
        if (aa == tgt[s])
#pragma unroll
          for (int q = 0; q < 4; ++q) L.bj[(s * 4 + q) * S + o] = xv[q];
      M4<W> A;
      mat_n1i_c<W>(L, P, l, A);
      W y[4];
      mv4(A, xv, y);
#pragma unroll
      for (int q = 0; q < 4; ++q) L.wk[q][l] = y[q];
    } else if (DIR == 1) {
      const int S = L.im * L.jm, o = aa + L.im * (p + 1);
      const int tgt[4] = {1, 2, L.km - 2, L.km - 3};
#pragma unroll
      for (int s = 0; s < 4; ++s)
        if (b == tgt[s])
#pragma unroll
          for (int q = 0; q < 4; ++q) L.bk[(s * 4 + q) * S + o] = xv[q];
      M4<W> A;
      mat_n2i_c<W>(L, P, l, A);
      W y[4];
      mv4(A, xv, y);
#pragma unroll
      for (int q = 0; q < 4; ++q) L.wk[q][l] = y[q];
    } else {
      M4<W> A;
      mat_mc_c<W>(L, P, l, A);
      W y[4];
      mv4(A, xv, y);
#pragma unroll
      for (int q = 0; q < 4; ++q) L.q[q][l] = L.q[q][l] + T(y[q]);
    }
  }
}

}  // namespace desalm
