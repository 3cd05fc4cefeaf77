// sweep.cuh -- K_I / K_J / K_K: the three scalar tridiagonal line sweeps of
// the diagonal approximate factorisation (src/rhs_diag_solver.F90:74-633).
//
// Each grid line carries four scalar systems (eigenvalue multipliers 0, 0,
// +1, -1).  Row coefficients come from the per-node tc/hc arrays written by
// K_R; the semi-explicit boundary rows (brh) are applied to the first/last
// interior rows; the elimination follows LAPACK SGTSV's no-interchange
// branch (src/sgtsv.f:107-121, 232-243), and a row where SGTSV would swap
// rows (|d_i| < |dl_i|) is counted in flags[0], a zero pivot (where SGTSV
// returns INFO > 0, src/sgtsv.f:112-119) or a singular middle 2x2 block in
// flags[1].
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
// Shared-memory slab sweep.  A CTA owns NL lines of one plane (consecutive in
// the transverse index that is contiguous in memory, or, for the i sweep,
// NL rows of contiguous i lines) and 8 NL threads.
//   phase 0  tc, hc and the four transformed residuals of the slab are copied
//            once (cp.async, all copies in flight, coalesced along the fastest
//            global index) into shared memory laid out [node][line] (line
//            stride NL + 1, so that the transposed i-sweep stores are free of
//            bank conflicts);
//   phase 1  thread (line, system m, half) eliminates its half-line in shared
//            memory exactly as the two-ended sweep does (same operations,
//            same order); the halves meet in the 2x2 middle solve and
//            back-substitute; the eliminated diagonal never leaves the SM;
//   phase 2  every node of the slab gets the next modal transform (or the
//            update) from the solved values in shared memory and writes its
//            four results once.
// Shared memory: 10 fields (tc, hc, r[4], d[4]) of slab_fs(n + 2, NL + 1)
// elements of W.
// ---------------------------------------------------------------------------
DESALM_HD inline int slab_fs(int np, int nlp) { return ((np * nlp + 31) / 32) * 32 + 16; }

template <class T, class W, int DIR, int NL>
__global__ void __launch_bounds__(8 * NL) k_sweep4(Lv<T, W> L, Par P, int blo, int bhi) {
  constexpr int NT = 8 * NL, NLP = NL + 1;
  extern __shared__ __align__(16) unsigned char sweep_slab[];
  __shared__ W sbw[NL][4], sbe[NL][4];
  __shared__ W mt_d[NL][4], mt_u[NL][4], mt_b[NL][4];   // top half's last eliminated row
  __shared__ W mb_d[NL][4], mb_l[NL][4], mb_b[NL][4];   // bottom half's last eliminated row
  const int tid = threadIdx.x;
  const int a0 = blockIdx.x * NL + 1;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa;
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; st = 1; sa = L.sj; }
  else if (DIR == 1) { amax = L.im - 2; n = L.jm - 2; st = L.sj; sa = 1; }
  else { amax = L.im - 2; n = L.km - 2; st = L.sk; sa = 1; }
  const int base = (DIR == 2) ? L.sj * b : L.sk * b;
  const int nl = min(NL, amax - a0 + 1);
  const int np = n + 2;
  const int fs = slab_fs(np, NLP);
  W* s_tc = reinterpret_cast<W*>(sweep_slab);
  W* s_hc = s_tc + fs;
  W* s_r = s_tc + 2 * fs;  // system q at s_r + q fs
  W* s_d = s_tc + 6 * fs;

  // ---- phase 0: slab -> shared memory, every copy in flight at once
  {
    const W* tc = L.tc[DIR];
    const W* hc = L.hc[DIR];
    const int total = nl * np;
    for (int t = tid; t < total; t += NT) {
      int li, p;
      if (DIR == 0) { li = t / np; p = t - li * np; }
      else { p = t / nl; li = t - p * nl; }
      const int l = base + (a0 + li) * sa + p * st;
      const int so = p * NLP + li;
      cp_async_elem(s_hc + so, hc + l);
      if (p >= 1 && p <= n) {
        cp_async_elem(s_tc + so, tc + l);
#pragma unroll
        for (int q = 0; q < 4; ++q) cp_async_elem(s_r + q * fs + so, L.wk[q] + l);
      }
    }
  }
  // semi-explicit boundary rows of each line
  if (tid < NL) {
    T bw[4] = {0, 0, 0, 0}, be[4] = {0, 0, 0, 0};
    if (tid < nl) {
      const int a = a0 + tid;
      const int lb = base + a * sa;
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
    for (int q = 0; q < 4; ++q) { sbw[tid][q] = W(bw[q]); sbe[tid][q] = W(be[q]); }
  }
  cp_async_wait_all();
  __syncthreads();

  // ---- phase 1: two-ended elimination in shared memory
  const int li = tid % NL, combo = tid / NL;
  const int m = combo & 3, half = combo >> 2;
  const bool act = li < nl;
  W* __restrict__ r = s_r + m * fs;
  W* __restrict__ sd = s_d + m * fs;
  const W* __restrict__ ctc = s_tc;
  const W* __restrict__ chc = s_hc;
  auto at = [&](int p) { return p * NLP + li; };
  auto coef = [&](W t, W hw_, W he_, W& aw, W& ae) {
    const W dw = t != W(0) ? hw_ : W(0);
    const W de = t != W(0) ? he_ : W(0);
    if (m < 2) { aw = -t; ae = -t; }
    else if (m == 2) { aw = -dw - t; ae = de - t; }
    else { aw = dw - t; ae = -de - t; }
  };
  const int h = n / 2;  // rows 0..h-1 top (nodes 1..h), h..n-1 bottom (nodes h+1..n)
  int npiv = 0, nzero = 0;
  if (act && half == 0) {
    const W bwm = sbw[li][m];
    W hw = chc[at(0)], hcur = chc[at(1)];
    W dprev = 0, duprev = 0, bprev = 0;
    for (int p = 1; p <= h; ++p) {
      const W t = ctc[at(p)], hn = chc[at(p + 1)];
      W aw, ae;
      coef(t, hw, hn, aw, ae);
      const W ap = W(1) + W(2) * t;
      W rr = r[at(p)];
      W d;
      if (p == 1) { rr = rr - aw * bwm; d = ap; bprev = rr; }
      else {
        npiv += dabs(dprev) < dabs(aw);
        const W f = aw / dprev;
        d = ap - f * duprev;
        bprev = rr - f * bprev;
      }
      nzero += d == W(0);
      sd[at(p)] = d;
      r[at(p)] = bprev;
      dprev = d; duprev = ae;
      hw = hcur; hcur = hn;
    }
    mt_d[li][m] = dprev; mt_u[li][m] = duprev; mt_b[li][m] = bprev;
  } else if (act && half == 1) {
    const W bem = sbe[li][m];
    W he = chc[at(n + 1)], hcur = chc[at(n)];
    W dprev = 0, awprev = 0, bprev = 0;
    for (int p = n; p > h; --p) {
      const W t = ctc[at(p)], hwv = chc[at(p - 1)];
      W aw, ae;
      coef(t, hwv, he, aw, ae);
      const W ap = W(1) + W(2) * t;
      W rr = r[at(p)];
      W d;
      if (p == n) { rr = rr - ae * bem; d = ap; bprev = rr; }
      else {
        npiv += dabs(dprev) < dabs(ae);
        const W f = ae / dprev;
        d = ap - f * awprev;
        bprev = rr - f * bprev;
      }
      nzero += d == W(0);
      sd[at(p)] = d;
      r[at(p)] = bprev;
      dprev = d; awprev = aw;
      he = hcur; hcur = hwv;
    }
    mb_d[li][m] = dprev; mb_l[li][m] = awprev; mb_b[li][m] = bprev;
  }
  if (npiv) atomicAdd(&L.flags[0], npiv);
  __syncthreads();
  if (act) {
    // the two middle rows: d1 x1 + u1 x2 = b1 (row h-1), l2 x1 + d2 x2 = b2 (row h)
    const W d1 = mt_d[li][m], u1 = mt_u[li][m], b1 = mt_b[li][m];
    const W d2 = mb_d[li][m], l2 = mb_l[li][m], b2 = mb_b[li][m];
    const W det = d1 * d2 - u1 * l2;
    nzero += half == 0 && det == W(0);
    if (nzero) atomicAdd(&L.flags[1], nzero);
    if (half == 0) {
      W x = (b1 * d2 - u1 * b2) / det;
      r[at(h)] = x;
      for (int p = h - 1; p >= 1; --p) {
        W aw, ae;
        coef(ctc[at(p)], W(0), chc[at(p + 1)], aw, ae);
        x = (r[at(p)] - ae * x) / sd[at(p)];
        r[at(p)] = x;
      }
    } else {
      W x = (d1 * b2 - l2 * b1) / det;
      r[at(h + 1)] = x;
      for (int p = h + 2; p <= n; ++p) {
        W aw, ae;
        coef(ctc[at(p)], chc[at(p - 1)], W(0), aw, ae);
        x = (r[at(p)] - aw * x) / sd[at(p)];
        r[at(p)] = x;
      }
    }
  }
  __syncthreads();

  // ---- phase 2: per-node transform in the sweep precision W, U nodes per
  // thread at a time: all their global reads are issued before any store
  const int total = nl * n;
  constexpr int U = 4;
  const T* const* m1 = DIR == 0 ? L.csi : (DIR == 1 ? L.eta : L.zet);  // forward matrix metrics
  const T* const* m2 = DIR == 0 ? L.eta : L.zet;                       // inverse matrix metrics
  for (int t0 = tid; t0 < total; t0 += NT * U) {
    int lnode[U], aan[U], pn[U];
    W a1[U][3], a2[U][3], sgv[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int t = t0 + u * NT;
      lnode[u] = -1;
      aan[u] = a0; pn[u] = 0;
      if (t < total) {
        int lq, p;
        if (DIR == 0) { lq = t / n; p = t - lq * n; }
        else { p = t / nl; lq = t - p * nl; }
        aan[u] = a0 + lq;
        pn[u] = p;
        const int l = base + aan[u] * sa + (p + 1) * st;
        lnode[u] = l;
        sgv[u] = __ldg(L.sig + l);
#pragma unroll
        for (int x = 0; x < 3; ++x) a1[u][x] = W(__ldg(m1[x] + l));
        if (DIR < 2)
#pragma unroll
          for (int x = 0; x < 3; ++x) a2[u][x] = W(__ldg(m2[x] + l));
      }
    }
    T qv[U][4];
    if (DIR == 2) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (lnode[u] >= 0)
#pragma unroll
          for (int q = 0; q < 4; ++q) qv[u][q] = L.q[q][lnode[u]];
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (lnode[u] < 0) continue;
      const int l = lnode[u], p = pn[u], aa = aan[u];
      const int so = (p + 1) * NLP + (aa - a0);
      W xv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) xv[q] = s_r[q * fs + so];
      W y[4], z[4];
      if (DIR == 0) {
        const int S = L.im * L.km, o = (p + 1) + L.im * b;
        const int tgt[4] = {1, 2, L.jm - 2, L.jm - 3};
#pragma unroll
        for (int s = 0; s < 4; ++s)
          if (aa == tgt[s])
#pragma unroll
            for (int q = 0; q < 4; ++q) L.bj[(s * 4 + q) * S + o] = xv[q];
        // N1^-1 x = Mb^-1 (Ma x)
        mfwd_apply<W>(a1[u][0], a1[u][1], a1[u][2], sgv[u], xv, y);
        minv_apply<W>(a2[u][0], a2[u][1], a2[u][2], sgv[u], y, z);
#pragma unroll
        for (int q = 0; q < 4; ++q) L.wk[q][l] = z[q];
      } else if (DIR == 1) {
        const int S = L.im * L.jm, o = aa + L.im * (p + 1);
        const int tgt[4] = {1, 2, L.km - 2, L.km - 3};
#pragma unroll
        for (int s = 0; s < 4; ++s)
          if (b == tgt[s])
#pragma unroll
            for (int q = 0; q < 4; ++q) L.bk[(s * 4 + q) * S + o] = xv[q];
        // N2^-1 x = Mc^-1 (Mb x)
        mfwd_apply<W>(a1[u][0], a1[u][1], a1[u][2], sgv[u], xv, y);
        minv_apply<W>(a2[u][0], a2[u][1], a2[u][2], sgv[u], y, z);
#pragma unroll
        for (int q = 0; q < 4; ++q) L.wk[q][l] = z[q];
      } else {
        mfwd_apply<W>(a1[u][0], a1[u][1], a1[u][2], sgv[u], xv, y);
#pragma unroll
        for (int q = 0; q < 4; ++q) L.q[q][l] = qv[u][q] + T(y[q]);
      }
    }
  }
}

}  // namespace desalm
