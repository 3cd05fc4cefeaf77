// sweep.cuh -- K_I / K_J / K_K: the three scalar tridiagonal line sweeps of
// the diagonal approximate factorisation (src/rhs_diag_solver.F90:74-633).
//
// Each grid line carries four scalar systems (eigenvalue multipliers 0, 0,
// +1, -1).  Row coefficients come from the per-node tc/hc arrays written by
// K_R; the semi-explicit boundary rows (brh) are applied to the first/last
// interior rows; the elimination follows LAPACK SGTSV's no-interchange
// branch (src/sgtsv.f:107-121, 232-243) wherever every column of the line's
// matrix is diagonally dominant (partial pivoting then interchanges no rows);
// other line systems are solved again by SGTSV's pivoting elimination, whose
// interchanges are counted in flags[0].  A zero pivot (where SGTSV returns
// INFO > 0, src/sgtsv.f:112-119) or a singular middle 2x2 block is counted in
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
// NL rows of contiguous i lines) and NT >= 8 NL threads.
//   phase 0  tc, hc and the four transformed residuals of the slab are copied
//            once (cp.async, all copies in flight, coalesced along the fastest
//            global index) into shared memory laid out [node][line] (line
//            stride NL + 1, so that the transposed i-sweep stores are free of
//            bank conflicts);
//   phase 1  thread (line, system m, half) eliminates its half-line in shared
//            memory exactly as the two-ended sweep does (same operations,
//            same order); the halves meet in the 2x2 middle solve and
//            back-substitute; the eliminated diagonal never leaves the SM;
//   phase 2  the solved values go back to wk; k_xform then applies the next
//            modal transform (or the update) per node at full occupancy.
// Shared memory: 10 fields (tc, hc, r[4], d[4]) of slab_fs(n + 2, NL + 1)
// elements of W.
// ---------------------------------------------------------------------------

template <class T, class W, int DIR, int NL, int NT>
__global__ void __launch_bounds__(NT) k_sweep4(Lv<T, W> L, Par P, int blo, int bhi) {
  pdl_wait();
  constexpr int NLP = NL + 1;
  static_assert(NT >= 8 * NL, "every solver thread is part of the CTA");
  extern __shared__ __align__(16) unsigned char sweep_slab[];
  __shared__ W sbw[NL][4], sbe[NL][4];
  __shared__ W mt_d[NL][4], mt_u[NL][4], mt_b[NL][4];   // top half's last eliminated row
  __shared__ W mb_d[NL][4], mb_l[NL][4], mb_b[NL][4];   // bottom half's last eliminated row
  __shared__ int s_ndom[NL][4];   // columns of (line, system) that are not diagonally dominant
  __shared__ int s_nz[NL][4];     // zero pivots of the two-ended elimination
  const int tid = threadIdx.x;
  const int a0 = blockIdx.x * NL + 1;
  const int b = blockIdx.y + 1;
  // oute: the fine level's characteristics outlet plane i = im is solved
  // too (idend = i_myend + 1, src/solver_daf.F90:371-373): one more row on
  // each i line, one more line of j and k lines per plane
  int amax, n, st, sa;
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; st = 1; sa = L.sj; }
  else if (DIR == 1) { amax = L.im - 2 + L.oute; n = L.jm - 2; st = L.sj; sa = 1; }
  else { amax = L.im - 2 + L.oute; n = L.km - 2; st = L.sk; sa = 1; }
  const int ext = DIR == 0 ? L.oute : 0;
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
      if (p >= 1 && p <= n) cp_async_elem(s_tc + so, tc + l);
      if (p >= 1 && p <= n + ext) {
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
  if (tid < 4 * NL) { (&s_ndom[0][0])[tid] = 0; (&s_nz[0][0])[tid] = 0; }
  cp_async_wait_all();
  __syncthreads();

  // ---- phase 1: two-ended elimination in shared memory.  Each half also
  // checks that the columns of its rows are diagonally dominant, |ap_p| >=
  // |ae_{p-1}| + |aw_{p+1}|: then Gaussian elimination with partial pivoting
  // interchanges no rows, so SGTSV (src/sgtsv.f:107-135) takes its
  // no-interchange branch throughout, which is the elimination done here.
  // A line system with a column that is not dominant is solved again below
  // with SGTSV's pivoting elimination.
  const int li = tid % NL, combo = tid / NL;
  const int m = combo & 3, half = combo >> 2;
  const bool act = tid < 8 * NL && li < nl;  // solver threads
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
  int nzero = 0, ndom = 0;
  W apc = 0, aec2 = 0;   // ap of the previous row and ae of the row before it (top half), or ap and aw of
                         // the next rows (bottom half): the column checks
  constexpr int R = 4;  // rows whose shared-memory operands are read ahead of the elimination chain
  // sd holds 1/d of every eliminated row, so that back-substitution multiplies
  if (act && half == 0) {
    const W bwm = sbw[li][m];
    W hw = chc[at(0)], hcur = chc[at(1)];
    W dprev = 0, rdprev = 0, duprev = 0, bprev = 0;
    for (int p0 = 1; p0 <= h; p0 += R) {
      W bt[R], bh[R], br[R];
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (p0 + u <= h) { bt[u] = ctc[at(p0 + u)]; bh[u] = chc[at(p0 + u + 1)]; br[u] = r[at(p0 + u)]; }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p <= h) {
          W aw, ae;
          coef(bt[u], hw, bh[u], aw, ae);
          const W ap = W(1) + W(2) * bt[u];
          W rr = br[u];
          W d;
          if (p == 1) { rr = rr - aw * bwm; d = ap; bprev = rr; }
          else {
            ndom += dabs(apc) < dabs(aec2) + dabs(aw);   // column p - 1
            const W f = aw * rdprev;
            d = ap - f * duprev;
            bprev = rr - f * bprev;
          }
          aec2 = duprev; apc = ap;
          nzero += d == W(0);
          rdprev = sweep_rcp(d);
          sd[at(p)] = rdprev;
          r[at(p)] = bprev;
          dprev = d; duprev = ae;
          hw = hcur; hcur = bh[u];
        }
      }
    }
    mt_d[li][m] = dprev; mt_u[li][m] = duprev; mt_b[li][m] = bprev;
  } else if (act && half == 1) {
    const W bem = sbe[li][m];
    W he = chc[at(n + 1)], hcur = chc[at(n)];
    W dprev = 0, rdprev = 0, awprev = 0, bprev = 0;
    if (ext) {
      // the outlet row (src/rhs_diag_solver.F90:207-221): ap = 1, 1,
      // 1 + dtau dc spr, 1 and aw = 0, 0, -dtau(im-1) dc spr(im-1), 0;
      // dtau dc spr = 2 h exactly
      const W d = m == 2 ? W(1) + W(2) * he : W(1);
      nzero += d == W(0);
      rdprev = sweep_rcp(d);
      sd[at(n + 1)] = rdprev;
      bprev = r[at(n + 1)];
      dprev = d;
      awprev = m == 2 ? -(W(2) * hcur) : W(0);
      apc = d;
    }
    for (int p0 = n; p0 > h; p0 -= R) {
      W bt[R], bh[R], br[R];
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (p0 - u > h) { bt[u] = ctc[at(p0 - u)]; bh[u] = chc[at(p0 - u - 1)]; br[u] = r[at(p0 - u)]; }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 - u;
        if (p > h) {
          W aw, ae;
          coef(bt[u], bh[u], he, aw, ae);
          const W ap = W(1) + W(2) * bt[u];
          W rr = br[u];
          W d;
          if (p == n && !ext) { rr = rr - ae * bem; d = ap; bprev = rr; }
          else {
            ndom += dabs(apc) < dabs(ae) + dabs(aec2);   // column p + 1
            const W f = ae * rdprev;
            d = ap - f * awprev;
            bprev = rr - f * bprev;
          }
          aec2 = awprev; apc = ap;
          nzero += d == W(0);
          rdprev = sweep_rcp(d);
          sd[at(p)] = rdprev;
          r[at(p)] = bprev;
          dprev = d; awprev = aw;
          he = hcur; hcur = bh[u];
        }
      }
    }
    mb_d[li][m] = dprev; mb_l[li][m] = awprev; mb_b[li][m] = bprev;
  }
  __syncthreads();
  if (act) {
    // the two middle rows: d1 x1 + u1 x2 = b1 (row h-1), l2 x1 + d2 x2 = b2 (row h)
    const W d1 = mt_d[li][m], u1 = mt_u[li][m], b1 = mt_b[li][m];
    const W d2 = mb_d[li][m], l2 = mb_l[li][m], b2 = mb_b[li][m];
    const W det = d1 * d2 - u1 * l2;
    nzero += half == 0 && det == W(0);
    // the two middle columns: column h needs the bottom half's aw_{h+1}
    // (l2), column h+1 the top half's ae_h (u1)
    if (half == 0) ndom += dabs(apc) < dabs(aec2) + dabs(l2);
    else ndom += dabs(apc) < dabs(u1) + dabs(aec2);
    if (ndom) atomicAdd(&s_ndom[li][m], ndom);
    if (nzero) atomicAdd(&s_nz[li][m], nzero);
    if (half == 0) {
      W x = (b1 * d2 - u1 * b2) / det;
      r[at(h)] = x;
      for (int p0 = h - 1; p0 >= 1; p0 -= R) {
        W bt[R], bh[R], br[R], bd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 - u >= 1) { bt[u] = ctc[at(p0 - u)]; bh[u] = chc[at(p0 - u + 1)]; br[u] = r[at(p0 - u)]; bd[u] = sd[at(p0 - u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u) {
          if (p0 - u >= 1) {
            W aw, ae;
            coef(bt[u], W(0), bh[u], aw, ae);
            x = (br[u] - ae * x) * bd[u];
            r[at(p0 - u)] = x;
          }
        }
      }
    } else {
      W x = (d1 * b2 - l2 * b1) / det;
      r[at(h + 1)] = x;
      for (int p0 = h + 2; p0 <= n; p0 += R) {
        W bt[R], bh[R], br[R], bd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 + u <= n) { bt[u] = ctc[at(p0 + u)]; bh[u] = chc[at(p0 + u - 1)]; br[u] = r[at(p0 + u)]; bd[u] = sd[at(p0 + u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u) {
          if (p0 + u <= n) {
            W aw, ae;
            coef(bt[u], bh[u], W(0), aw, ae);
            x = (br[u] - aw * x) * bd[u];
            r[at(p0 + u)] = x;
          }
        }
      }
      if (ext) {
        const W aw = m == 2 ? -(W(2) * chc[at(n)]) : W(0);
        x = (r[at(n + 1)] - aw * x) * sd[at(n + 1)];
        r[at(n + 1)] = x;
      }
    }
  }
  __syncthreads();

  // ---- a line system with a column that is not dominant: solved again from
  // its original rows by SGTSV's elimination with partial pivoting
  // (src/sgtsv.f:107-162, back-substitution :232-257), one thread per line,
  // its systems in turn.  The 1/d columns of the line are free now; three
  // of them hold d, du and dl (dl keeps the fill-in of a swap, as SGTSV
  // does).  Rows that interchange are counted in flags[0], zero pivots
  // (SGTSV's INFO > 0) in flags[1].
  if (tid < nl) {
    const int lf = tid;
    int nsw = 0, nz = 0;
    for (int q = 0; q < 4; ++q) {
      if (!s_ndom[lf][q]) { nz += s_nz[lf][q]; continue; }
      const int N = n + ext;                       // rows 1..N
      W* bq = s_r + q * fs;
      W* dd = s_d;                                 // d
      W* du = s_d + fs;                            // du (and du2 after a swap goes to dl)
      W* dl = s_d + 2 * fs;                        // dl
      auto fat = [&](int p) { return p * NLP + lf; };
      const int l0 = base + (a0 + lf) * sa;
      for (int p = 1; p <= N; ++p) {
        W aw, ae, ap;
        if (p <= n) {
          const W t = s_tc[fat(p)];
          const W hw_ = s_hc[fat(p - 1)], he_ = s_hc[fat(p + 1)];
          const W dw = t != W(0) ? hw_ : W(0), de = t != W(0) ? he_ : W(0);
          if (q < 2) { aw = -t; ae = -t; }
          else if (q == 2) { aw = -dw - t; ae = de - t; }
          else { aw = dw - t; ae = -de - t; }
          ap = W(1) + W(2) * t;
        } else {  // the outlet row
          ap = q == 2 ? W(1) + W(2) * s_hc[fat(n + 1)] : W(1);
          aw = q == 2 ? -(W(2) * s_hc[fat(n)]) : W(0);
          ae = W(0);
        }
        W b = L.wk[q][l0 + p * st];
        if (p == 1) b = b - aw * sbw[lf][q];
        if (p == n && !ext) b = b - ae * sbe[lf][q];
        bq[fat(p)] = b;
        dd[fat(p)] = ap;
        du[fat(p)] = ae;                           // row p's super-diagonal
        dl[fat(p)] = p > 1 ? aw : W(0);            // dl[p] couples row p to row p - 1
      }
      // forward elimination (0-based i of SGTSV = row i + 1 here)
      bool sing = false;
      for (int p = 1; p <= N - 1 && !sing; ++p) {
        const W dlp = dl[fat(p + 1)];
        if (dabs(dd[fat(p)]) >= dabs(dlp)) {
          if (dd[fat(p)] != W(0)) {
            const W fact = dlp / dd[fat(p)];
            dd[fat(p + 1)] = dd[fat(p + 1)] - fact * du[fat(p)];
            bq[fat(p + 1)] = bq[fat(p + 1)] - fact * bq[fat(p)];
          } else {
            sing = true;
          }
          dl[fat(p + 1)] = W(0);
        } else {
          ++nsw;
          const W fact = dd[fat(p)] / dlp;
          dd[fat(p)] = dlp;
          const W temp = dd[fat(p + 1)];
          dd[fat(p + 1)] = du[fat(p)] - fact * temp;
          if (p <= N - 2) {
            dl[fat(p + 1)] = du[fat(p + 1)];                 // fill-in of row p: du2
            du[fat(p + 1)] = -fact * dl[fat(p + 1)];
          } else {
            dl[fat(p + 1)] = W(0);
          }
          du[fat(p)] = temp;
          const W tb = bq[fat(p)];
          bq[fat(p)] = bq[fat(p + 1)];
          bq[fat(p + 1)] = tb - fact * bq[fat(p + 1)];
        }
      }
      if (sing || dd[fat(N)] == W(0)) { ++nz; continue; }
      // back-substitution: x_p = (b_p - du_p x_{p+1} - du2_p x_{p+2}) / d_p,
      // du2_p held in dl[p + 1]
      bq[fat(N)] = bq[fat(N)] / dd[fat(N)];
      if (N > 1) bq[fat(N - 1)] = (bq[fat(N - 1)] - du[fat(N - 1)] * bq[fat(N)]) / dd[fat(N - 1)];
      for (int p = N - 2; p >= 1; --p)
        bq[fat(p)] = (bq[fat(p)] - du[fat(p)] * bq[fat(p + 1)] - dl[fat(p + 1)] * bq[fat(p + 2)]) / dd[fat(p)];
    }
    if (nsw) atomicAdd(&L.flags[0], nsw);
    if (nz) atomicAdd(&L.flags[1], nz);
  }
  __syncthreads();

  // ---- phase 2: the solved values back to wk (the modal transform follows
  // in k_xform, at full occupancy)
  const int ne = n + ext;
  const int total = nl * ne;
  for (int t = tid; t < total; t += NT) {
    int lq, p;
    if (DIR == 0) { lq = t / ne; p = t - lq * ne; }
    else { p = t / nl; lq = t - p * nl; }
    const int l = base + (a0 + lq) * sa + (p + 1) * st;
    const int so = (p + 1) * NLP + lq;
#pragma unroll
    for (int q = 0; q < 4; ++q) L.wk[q][l] = s_r[q * fs + so];
  }
}

// Per-node step after a line sweep, in the sweep precision W, one thread per
// interior node: after the i sweep the semi-explicit rows of the j faces are
// copied out (rows 2, 3, jm-1, jm-2) and wk <- N1^-1 wk = Mb^-1 (Ma wk);
// after the j sweep the k-face rows are copied and wk <- N2^-1 wk =
// Mc^-1 (Mb wk); after the k sweep q <- q + Mc wk (src/rhs_diag_solver.F90:
// 240-258, 416-434, 600-633; src/solver_daf.F90:409-418).
template <class T, class W, int DIR>
__global__ void __launch_bounds__(128) k_xform(Lv<T, W> L) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > L.im - 2 + L.oute || j > L.jm - 2) return;
  const int l = i + L.sj * j + L.sk * k;
  W xv[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) xv[q] = L.wk[q][l];
  const W sg = L.sig[l];
  W y[4], z[4];
  if (DIR == 0) {
    const int S = L.im * L.km, o = i + L.im * k;
    const int tgt[4] = {1, 2, L.jm - 2, L.jm - 3};
#pragma unroll
    for (int s = 0; s < 4; ++s)
      if (j == tgt[s])
#pragma unroll
        for (int q = 0; q < 4; ++q) L.bj[(s * 4 + q) * S + o] = xv[q];
    mfwd_apply<W>(L.mw[0][l], L.mw[1][l], L.mw[2][l], sg, xv, y);
    minv_apply<W>(L.mw[3][l], L.mw[4][l], L.mw[5][l], sg, y, z);
#pragma unroll
    for (int q = 0; q < 4; ++q) L.wk[q][l] = z[q];
  } else if (DIR == 1) {
    const int S = L.im * L.jm, o = i + L.im * j;
    const int tgt[4] = {1, 2, L.km - 2, L.km - 3};
#pragma unroll
    for (int s = 0; s < 4; ++s)
      if (k == tgt[s])
#pragma unroll
        for (int q = 0; q < 4; ++q) L.bk[(s * 4 + q) * S + o] = xv[q];
    mfwd_apply<W>(L.mw[3][l], L.mw[4][l], L.mw[5][l], sg, xv, y);
    minv_apply<W>(L.mw[6][l], L.mw[7][l], L.mw[8][l], sg, y, z);
#pragma unroll
    for (int q = 0; q < 4; ++q) L.wk[q][l] = z[q];
  } else {
    mfwd_apply<W>(L.mw[6][l], L.mw[7][l], L.mw[8][l], sg, xv, y);
#pragma unroll
    for (int q = 0; q < 4; ++q) L.q[q][l] = L.q[q][l] + T(y[q]);
  }
}

}  // namespace desalm
