// sweep.cuh -- K_I / K_J / K_K: the three scalar tridiagonal line sweeps of
// the diagonal approximate factorisation (src/rhs_diag_solver.F90:74-633).
//
// Each grid line carries four scalar systems (eigenvalue multipliers 0, 0,
// +1, -1).  Row coefficients come from the per-node tc/hc arrays written by
// K_R; the semi-explicit boundary rows (brh) are applied to the first/last
// interior rows; the elimination follows LAPACK SGTSV's no-interchange
// branch (src/sgtsv.f:107-121, 232-243), and a row where SGTSV would swap
// rows (|d_i| < |dl_i|) is counted in flags[0], a zero pivot in flags[1].
// After the solve each node gets the next modal transform (N1^-1 after the i
// sweep, N2^-1 after the j sweep) or, after the k sweep, Mc and the update
// q <- q + dq (src/solver_daf.F90:409-418).
#pragma once
#include "modal.cuh"

namespace desalm {

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

}  // namespace desalm

namespace desalm {

// ---------------------------------------------------------------------------
// Two-ended line sweep.  A CTA owns 32 lines and
// has 8 warps: warp m (< 4) eliminates the upper half of system m top-down
// (SGTSV's no-interchange order), warp 4 + m eliminates the lower half
// bottom-up; the two meet in a 2x2 solve at the middle rows, then each warp
// back-substitutes its own half: twice the threads of a one-ended solve and
// half the dependent chain per line; the result differs from one top-down
// pass by round-off only.  Phase 2 walks the CTA's nodes with coalesced
// indexing and applies the modal transform (or the update).
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
