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
  for (int m = 0; m < 4; ++m) v[m] = fma2(T(P.sa[m][b]), T(r1[m * stride]), T(P.sb[m][b]), T(r2[m * stride]));
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
          const W ap = fmaw(W(2), bt[u], W(1));
          W rr = br[u];
          W d;
          if (p == 1) { rr = fmaw(-aw, bwm, rr); d = ap; bprev = rr; }
          else {
            ndom += dabs(apc) < dabs(aec2) + dabs(aw);   // column p - 1
            const W f = mulw(aw, rdprev);
            d = fmaw(-f, duprev, ap);
            bprev = fmaw(-f, bprev, rr);
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
      const W d = m == 2 ? fmaw(W(2), he, W(1)) : W(1);
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
          const W ap = fmaw(W(2), bt[u], W(1));
          W rr = br[u];
          W d;
          if (p == n && !ext) { rr = fmaw(-ae, bem, rr); d = ap; bprev = rr; }
          else {
            ndom += dabs(apc) < dabs(ae) + dabs(aec2);   // column p + 1
            const W f = mulw(ae, rdprev);
            d = fmaw(-f, awprev, ap);
            bprev = fmaw(-f, bprev, rr);
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
    const W det = fms2(d1, d2, u1, l2);
    nzero += half == 0 && det == W(0);
    // the two middle columns: column h needs the bottom half's aw_{h+1}
    // (l2), column h+1 the top half's ae_h (u1)
    if (half == 0) ndom += dabs(apc) < dabs(aec2) + dabs(l2);
    else ndom += dabs(apc) < dabs(u1) + dabs(aec2);
    if (ndom) atomicAdd(&s_ndom[li][m], ndom);
    if (nzero) atomicAdd(&s_nz[li][m], nzero);
    if (half == 0) {
      W x = fms2(b1, d2, u1, b2) / det;
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
            x = mulw(fmaw(-ae, x, br[u]), bd[u]);
            r[at(p0 - u)] = x;
          }
        }
      }
    } else {
      W x = fms2(d1, b2, l2, b1) / det;
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
            x = mulw(fmaw(-aw, x, br[u]), bd[u]);
            r[at(p0 + u)] = x;
          }
        }
      }
      if (ext) {
        const W aw = m == 2 ? -(W(2) * chc[at(n)]) : W(0);
        x = mulw(fmaw(-aw, x, r[at(n + 1)]), sd[at(n + 1)]);
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
  // (SGTSV's INFO > 0) in flags[1], the systems solved this way in flags[2].
  if (tid < nl) {
    const int lf = tid;
    int nsw = 0, nz = 0, npl = 0;
    for (int q = 0; q < 4; ++q) {
      if (!s_ndom[lf][q]) { nz += s_nz[lf][q]; continue; }
      ++npl;
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
          ap = fmaw(W(2), t, W(1));
        } else {  // the outlet row
          ap = q == 2 ? fmaw(W(2), s_hc[fat(n + 1)], W(1)) : W(1);
          aw = q == 2 ? -(W(2) * s_hc[fat(n)]) : W(0);
          ae = W(0);
        }
        W b = L.wk[q][l0 + p * st];
        if (p == 1) b = fmaw(-aw, sbw[lf][q], b);
        if (p == n && !ext) b = fmaw(-ae, sbe[lf][q], b);
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
            dd[fat(p + 1)] = fmaw(-fact, du[fat(p)], dd[fat(p + 1)]);
            bq[fat(p + 1)] = fmaw(-fact, bq[fat(p)], bq[fat(p + 1)]);
          } else {
            sing = true;
          }
          dl[fat(p + 1)] = W(0);
        } else {
          ++nsw;
          const W fact = dd[fat(p)] / dlp;
          dd[fat(p)] = dlp;
          const W temp = dd[fat(p + 1)];
          dd[fat(p + 1)] = fmaw(-fact, temp, du[fat(p)]);
          if (p <= N - 2) {
            dl[fat(p + 1)] = du[fat(p + 1)];                 // fill-in of row p: du2
            du[fat(p + 1)] = -fact * dl[fat(p + 1)];
          } else {
            dl[fat(p + 1)] = W(0);
          }
          du[fat(p)] = temp;
          const W tb = bq[fat(p)];
          bq[fat(p)] = bq[fat(p + 1)];
          bq[fat(p + 1)] = fmaw(-fact, bq[fat(p + 1)], tb);
        }
      }
      if (sing || dd[fat(N)] == W(0)) { ++nz; continue; }
      // back-substitution: x_p = (b_p - du_p x_{p+1} - du2_p x_{p+2}) / d_p,
      // du2_p held in dl[p + 1]
      bq[fat(N)] = bq[fat(N)] / dd[fat(N)];
      if (N > 1) bq[fat(N - 1)] = fmaw(-du[fat(N - 1)], bq[fat(N)], bq[fat(N - 1)]) / dd[fat(N - 1)];
      for (int p = N - 2; p >= 1; --p)
        bq[fat(p)] = fmaw(-dl[fat(p + 1)], bq[fat(p + 2)], fmaw(-du[fat(p)], bq[fat(p + 1)], bq[fat(p)])) / dd[fat(p)];
    }
    if (nsw) atomicAdd(&L.flags[0], nsw);
    if (nz) atomicAdd(&L.flags[1], nz);
    if (npl) atomicAdd(&L.flags[2], npl);
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

// ---------------------------------------------------------------------------
// The DAF line sweep with the lines in the lanes.  A CTA owns 32 neighbouring
// lines of one plane (the lanes) and eight warps: warp w solves system
// m = w & 3 of the top (w < 4) or bottom half of every line.  The rows are
// read from global memory one block ahead of the elimination (coalesced
// across the lanes for the j and k sweeps; the i sweep's rows come through L1
// sectors, which the four systems of a half share), and each eliminated row
// (1/d and b') goes to a scratch laid out [row][line], coalesced across the
// lanes, for the back-substitution, which writes the solution straight into
// wk.  Without a staged slab the occupancy is set by registers, and every
// line of a level is in flight at once.  The operations and their order are
// k_sweep4's (two-ended elimination, SGTSV's no-interchange branch where
// every column is diagonally dominant, its pivoting elimination otherwise),
// so both kernels give the same values.
// The scratch of a row lives a few microseconds: the back-substitution reads
// it in the reverse order of the elimination, then drops its L2 lines
// without write-back (the lines of a plane are padded to a multiple of 32, so
// that a warp's row is whole 128-byte lines), so that it need not reach HBM.
// Rows are not dropped where a lane of the warp takes the pivoting path,
// which reuses them.
// Scratch (L.gs, arrays L.gss elements apart): per system m the arrays
// 4m + 0..3 = 1/d (d in the pivoting elimination), b', du and dl; row p of
// line (a, b) at (p - 1) nln + (a - 1) + amaxp (b - 1), amaxp = amax rounded
// up to 32.
// ---------------------------------------------------------------------------
// Build-time tuning knobs of k_gsweep: resident CTAs per SM requested, and
// rows loaded one block ahead of the elimination in FP32 (half that in FP64).
#ifndef DESALM_GS_MINBLOCKS
#define DESALM_GS_MINBLOCKS 2
#endif
#ifndef DESALM_GS_ROWS
#define DESALM_GS_ROWS 8
#endif
template <class T, class W, int DIR>
__global__ void __launch_bounds__(256, DESALM_GS_MINBLOCKS) k_gsweep(Lv<T, W> L, Par P, int blo, int bhi) {
  pdl_wait();
  constexpr int R = sizeof(W) == 4 ? DESALM_GS_ROWS : DESALM_GS_ROWS / 2;  // rows loaded one block ahead
  __shared__ W mt_d[4][32], mt_u[4][32], mt_b[4][32];
  __shared__ W mb_d[4][32], mb_l[4][32], mb_b[4][32];
  __shared__ int s_ndom[4][32], s_nz[4][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m = w & 3, half = w >> 2;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa;
  if (DIR == 0) { amax = L.jm - 2; n = L.im - 2; st = 1; sa = L.sj; }
  else if (DIR == 1) { amax = L.im - 2 + L.oute; n = L.jm - 2; st = L.sj; sa = 1; }
  else { amax = L.im - 2 + L.oute; n = L.km - 2; st = L.sk; sa = 1; }
  const int ext = DIR == 0 ? L.oute : 0;
  const int base = (DIR == 2) ? L.sj * b : L.sk * b;
  const int a = blockIdx.x * 32 + lane + 1;
  const bool act = a <= amax;
  const int amaxp = (amax + 31) & ~31;
  const int nln = amaxp * (int)gridDim.y;
  const int line = (a - 1) + amaxp * (b - 1);
  const int line0 = line - lane;               // the warp's first line: 128-byte aligned rows
  const unsigned wact = __ballot_sync(0xffffffffu, act);
  const int lb = base + a * sa;                // node 0 of the line
  const W* __restrict__ tc = L.tc[DIR];
  const W* __restrict__ hc = L.hc[DIR];
  W* __restrict__ r = L.wk[m];
  W* __restrict__ gd = L.gs + (size_t)(4 * m) * L.gss;
  W* __restrict__ gb = L.gs + (size_t)(4 * m + 1) * L.gss;
  auto sc = [&](int p) { return (p - 1) * nln + line; };   // row p = node p of the line, 1..n + ext
  auto coef = [&](W t, W hw_, W he_, W& aw, W& ae) {
    const W dw = t != W(0) ? hw_ : W(0);
    const W de = t != W(0) ? he_ : W(0);
    if (m < 2) { aw = -t; ae = -t; }
    else if (m == 2) { aw = -dw - t; ae = de - t; }
    else { aw = dw - t; ae = -de - t; }
  };
  // semi-explicit boundary rows of the 32 lines, all four components: warp 0
  // forms the west rows, warp 4 the east rows (before the elimination, so
  // that the modal matrices' registers are not held through it)
  __shared__ W s_bw[4][32], s_be[4][32];
  if (w == 0 || w == 4) {
    const int hi = w == 4;
    T v[4] = {0, 0, 0, 0};
    if (act) {
      if (DIR == 0) {
        if (!hi && blo) {
          const int S = L.jm * L.km, o = a + L.jm * b;
          face_vec<T, W, 0>(L, P, lb, 0, L.bi + o, L.bi + 4 * S + o, S, v);
        }
      } else if (DIR == 1) {
        const int S = L.im * L.km, o = a + L.im * b;
        if (!hi && blo) face_vec<T, W, 1>(L, P, lb, 2, L.bj + o, L.bj + 4 * S + o, S, v);
        if (hi && bhi) face_vec<T, W, 1>(L, P, lb + (n + 1) * st, 3, L.bj + 8 * S + o, L.bj + 12 * S + o, S, v);
      } else {
        const int S = L.im * L.jm, o = a + L.im * b;
        if (!hi && blo) face_vec<T, W, 2>(L, P, lb, 4, L.bk + o, L.bk + 4 * S + o, S, v);
        if (hi && bhi) face_vec<T, W, 2>(L, P, lb + (n + 1) * st, 5, L.bk + 8 * S + o, L.bk + 12 * S + o, S, v);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) (hi ? s_be : s_bw)[q][lane] = W(v[q]);
  }
  if (half == 0) { s_ndom[m][lane] = 0; s_nz[m][lane] = 0; }
  __syncthreads();
  const int h = n / 2;  // nodes 1..h top, h+1..n bottom
  int nzero = 0, ndom = 0;
  W apc = 0, aec2 = 0;
  if (act && half == 0) {
    const W bwm = s_bw[m][lane];
    W hw = hc[lb], hcur = hc[lb + st];
    W dprev = 0, rdprev = 0, duprev = 0, bprev = 0;
    W ct[R], ch[R], cr[R];
#pragma unroll
    for (int u = 0; u < R; ++u)
      if (1 + u <= h) { const int l = lb + (1 + u) * st; ct[u] = tc[l]; ch[u] = hc[l + st]; cr[u] = r[l]; }
    for (int p0 = 1; p0 <= h; p0 += R) {
      W nt[R], nh[R], nr[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        nt[u] = nh[u] = nr[u] = W(0);
        if (p0 + R + u <= h) { const int l = lb + (p0 + R + u) * st; nt[u] = tc[l]; nh[u] = hc[l + st]; nr[u] = r[l]; }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p <= h) {
          W aw, ae;
          coef(ct[u], hw, ch[u], aw, ae);
          const W ap = fmaw(W(2), ct[u], W(1));
          W rr = cr[u];
          W d;
          if (p == 1) { rr = fmaw(-aw, bwm, rr); d = ap; bprev = rr; }
          else {
            ndom += dabs(apc) < dabs(aec2) + dabs(aw);
            const W f = mulw(aw, rdprev);
            d = fmaw(-f, duprev, ap);
            bprev = fmaw(-f, bprev, rr);
          }
          aec2 = duprev; apc = ap;
          nzero += d == W(0);
          rdprev = sweep_rcp(d);
          gd[sc(p)] = rdprev;
          gb[sc(p)] = bprev;
          dprev = d; duprev = ae;
          hw = hcur; hcur = ch[u];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) { ct[u] = nt[u]; ch[u] = nh[u]; cr[u] = nr[u]; }
    }
    mt_d[m][lane] = dprev; mt_u[m][lane] = duprev; mt_b[m][lane] = bprev;
  } else if (act && half == 1) {
    const W bem = s_be[m][lane];
    W he = hc[lb + (n + 1) * st], hcur = hc[lb + n * st];
    W dprev = 0, rdprev = 0, awprev = 0, bprev = 0;
    if (ext) {
      // the outlet row (src/rhs_diag_solver.F90:207-221)
      const W d = m == 2 ? fmaw(W(2), he, W(1)) : W(1);
      nzero += d == W(0);
      rdprev = sweep_rcp(d);
      gd[sc(n + 1)] = rdprev;
      bprev = r[lb + (n + 1) * st];
      gb[sc(n + 1)] = bprev;
      dprev = d;
      awprev = m == 2 ? -(W(2) * hcur) : W(0);
      apc = d;
    }
    W ct[R], ch[R], cr[R];
#pragma unroll
    for (int u = 0; u < R; ++u)
      if (n - u > h) { const int l = lb + (n - u) * st; ct[u] = tc[l]; ch[u] = hc[l - st]; cr[u] = r[l]; }
    for (int p0 = n; p0 > h; p0 -= R) {
      W nt[R], nh[R], nr[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        nt[u] = nh[u] = nr[u] = W(0);
        if (p0 - R - u > h) { const int l = lb + (p0 - R - u) * st; nt[u] = tc[l]; nh[u] = hc[l - st]; nr[u] = r[l]; }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 - u;
        if (p > h) {
          W aw, ae;
          coef(ct[u], ch[u], he, aw, ae);
          const W ap = fmaw(W(2), ct[u], W(1));
          W rr = cr[u];
          W d;
          if (p == n && !ext) { rr = fmaw(-ae, bem, rr); d = ap; bprev = rr; }
          else {
            ndom += dabs(apc) < dabs(ae) + dabs(aec2);
            const W f = mulw(ae, rdprev);
            d = fmaw(-f, awprev, ap);
            bprev = fmaw(-f, bprev, rr);
          }
          aec2 = awprev; apc = ap;
          nzero += d == W(0);
          rdprev = sweep_rcp(d);
          gd[sc(p)] = rdprev;
          gb[sc(p)] = bprev;
          dprev = d; awprev = aw;
          he = hcur; hcur = ch[u];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) { ct[u] = nt[u]; ch[u] = nh[u]; cr[u] = nr[u]; }
    }
    mb_d[m][lane] = dprev; mb_l[m][lane] = awprev; mb_b[m][lane] = bprev;
  }
  __syncthreads();
  W d1 = 0, u1 = 0, b1 = 0, d2 = 0, l2 = 0, b2 = 0, det = 0;
  if (act) {
    d1 = mt_d[m][lane]; u1 = mt_u[m][lane]; b1 = mt_b[m][lane];
    d2 = mb_d[m][lane]; l2 = mb_l[m][lane]; b2 = mb_b[m][lane];
    det = fms2(d1, d2, u1, l2);
    nzero += half == 0 && det == W(0);
    if (half == 0) ndom += dabs(apc) < dabs(aec2) + dabs(l2);
    else ndom += dabs(apc) < dabs(u1) + dabs(aec2);
    if (ndom) atomicAdd(&s_ndom[m][lane], ndom);
    if (nzero) atomicAdd(&s_nz[m][lane], nzero);
  }
  __syncthreads();
  // the warp drops its scratch rows as it reads them back when none of its
  // lines takes the pivoting path (which reuses them)
  const bool wdisc = __all_sync(0xffffffffu, !act || !s_ndom[m][lane]);
  if (!act) return;
  // rows pb, pb + dir, ... (R of them, those in [lo, hi]) of the warp's 32
  // lines read for the last time: lane t < 2 R SEG drops one 128-byte line
  // of the b' (t / SEG even) or 1/d column
  auto drop = [&](int pb, int dir, int lo, int hi) {
    if (!wdisc) return;
    __syncwarp(wact);
    constexpr int SEG = 32 * (int)sizeof(W) / 128;   // 128-byte lines per warp row
    static_assert(R * 2 * SEG <= 32, "one 128-byte line per lane");
    if (lane < R * 2 * SEG) {
      const int u = lane / (2 * SEG), col = (lane / SEG) & 1, piece = lane % SEG;
      const int p = pb + dir * u;
      if (p >= lo && p <= hi) l2_discard((col ? gd : gb) + (p - 1) * nln + line0 + piece * (128 / (int)sizeof(W)));
    }
  };
  if (!s_ndom[m][lane]) {
    if (half == 0) {
      const int nz = s_nz[m][lane];
      if (nz) atomicAdd(&L.flags[1], nz);
      W x = fms2(b1, d2, u1, b2) / det;
      r[lb + h * st] = x;
      drop(h, 1, h, h);                  // the middle row is not read back
      for (int p0 = h - 1; p0 >= 1; p0 -= R) {
        W bt[R], bh[R], br[R], bd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 - u >= 1) { const int l = lb + (p0 - u) * st; bt[u] = tc[l]; bh[u] = hc[l + st]; br[u] = gb[sc(p0 - u)]; bd[u] = gd[sc(p0 - u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u) {
          if (p0 - u >= 1) {
            W aw, ae;
            coef(bt[u], W(0), bh[u], aw, ae);
            x = mulw(fmaw(-ae, x, br[u]), bd[u]);
            r[lb + (p0 - u) * st] = x;
          }
        }
        drop(p0, -1, 1, h - 1);
      }
    } else {
      W x = fms2(d1, b2, l2, b1) / det;
      r[lb + (h + 1) * st] = x;
      drop(h + 1, 1, h + 1, h + 1);
      for (int p0 = h + 2; p0 <= n; p0 += R) {
        W bt[R], bh[R], br[R], bd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 + u <= n) { const int l = lb + (p0 + u) * st; bt[u] = tc[l]; bh[u] = hc[l - st]; br[u] = gb[sc(p0 + u)]; bd[u] = gd[sc(p0 + u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u) {
          if (p0 + u <= n) {
            W aw, ae;
            coef(bt[u], bh[u], W(0), aw, ae);
            x = mulw(fmaw(-aw, x, br[u]), bd[u]);
            r[lb + (p0 + u) * st] = x;
          }
        }
        drop(p0, 1, h + 2, n);
      }
      if (ext) {
        const W aw = m == 2 ? -(W(2) * hc[lb + n * st]) : W(0);
        x = mulw(fmaw(-aw, x, gb[sc(n + 1)]), gd[sc(n + 1)]);
        r[lb + (n + 1) * st] = x;
        drop(n + 1, 1, n + 1, n + 1);
      }
    }
    return;
  }
  if (half != 0) return;
  // ---- a system with a column that is not dominant: SGTSV's elimination
  // with partial pivoting (src/sgtsv.f:107-162, back-substitution :232-257)
  // from the original rows, in the system's scratch: d, b, du and dl (dl
  // keeps the fill-in of a swap, as SGTSV does)
  W* __restrict__ dd = gd;
  W* __restrict__ bq = gb;
  W* __restrict__ du = L.gs + (size_t)(4 * m + 2) * L.gss;
  W* __restrict__ dl = L.gs + (size_t)(4 * m + 3) * L.gss;
  const int N = n + ext;
  const W bwm = s_bw[m][lane], bem = s_be[m][lane];
  for (int p = 1; p <= N; ++p) {
    W aw, ae, ap;
    if (p <= n) {
      const W t = tc[lb + p * st];
      coef(t, hc[lb + (p - 1) * st], hc[lb + (p + 1) * st], aw, ae);
      ap = fmaw(W(2), t, W(1));
    } else {  // the outlet row
      ap = m == 2 ? fmaw(W(2), hc[lb + (n + 1) * st], W(1)) : W(1);
      aw = m == 2 ? -(W(2) * hc[lb + n * st]) : W(0);
      ae = W(0);
    }
    W bv = r[lb + p * st];
    if (p == 1) bv = fmaw(-aw, bwm, bv);
    if (p == n && !ext) bv = fmaw(-ae, bem, bv);
    bq[sc(p)] = bv;
    dd[sc(p)] = ap;
    du[sc(p)] = ae;
    dl[sc(p)] = p > 1 ? aw : W(0);
  }
  int nsw = 0;
  bool sing = false;
  for (int p = 1; p <= N - 1 && !sing; ++p) {
    const W dlp = dl[sc(p + 1)];
    const W dp = dd[sc(p)];
    if (dabs(dp) >= dabs(dlp)) {
      if (dp != W(0)) {
        const W fact = dlp / dp;
        dd[sc(p + 1)] = fmaw(-fact, du[sc(p)], dd[sc(p + 1)]);
        bq[sc(p + 1)] = fmaw(-fact, bq[sc(p)], bq[sc(p + 1)]);
      } else {
        sing = true;
      }
      dl[sc(p + 1)] = W(0);
    } else {
      ++nsw;
      const W fact = dp / dlp;
      dd[sc(p)] = dlp;
      const W temp = dd[sc(p + 1)];
      dd[sc(p + 1)] = fmaw(-fact, temp, du[sc(p)]);
      if (p <= N - 2) {
        dl[sc(p + 1)] = du[sc(p + 1)];               // fill-in of row p: du2
        du[sc(p + 1)] = -fact * dl[sc(p + 1)];
      } else {
        dl[sc(p + 1)] = W(0);
      }
      du[sc(p)] = temp;
      const W tb = bq[sc(p)];
      bq[sc(p)] = bq[sc(p + 1)];
      bq[sc(p + 1)] = fmaw(-fact, bq[sc(p + 1)], tb);
    }
  }
  if (sing || dd[sc(N)] == W(0)) {
    atomicAdd(&L.flags[1], 1);
  } else {
    bq[sc(N)] = bq[sc(N)] / dd[sc(N)];
    if (N > 1) bq[sc(N - 1)] = fmaw(-du[sc(N - 1)], bq[sc(N)], bq[sc(N - 1)]) / dd[sc(N - 1)];
    for (int p = N - 2; p >= 1; --p)
      bq[sc(p)] = fmaw(-dl[sc(p + 1)], bq[sc(p + 2)], fmaw(-du[sc(p)], bq[sc(p + 1)], bq[sc(p)])) / dd[sc(p)];
    for (int p = 1; p <= N; ++p) r[lb + p * st] = bq[sc(p)];
  }
  if (nsw) atomicAdd(&L.flags[0], nsw);
  atomicAdd(&L.flags[2], 1);
}

// ---------------------------------------------------------------------------
// Short lines (at most 32 rows: the coarse levels): one warp per line system,
// one row per lane, solved by parallel cyclic reduction with warp shuffles.
// In five steps every row eliminates its couplings to the rows s = 1, 2, 4,
// 8, 16 away (rows past the ends act as identity rows), after which each row
// stands alone: x = d / b.  The rows are k_gsweep's (coefficients, boundary
// rows, outlet row) and so is the column test; cyclic reduction is Gaussian
// elimination in another order, stable without interchanges when every
// column is diagonally dominant.  A system with a column that is not is
// solved by lane 0 with SGTSV's pivoting elimination in shared memory, as in
// k_gsweep.  The elimination order differs from the Thomas kernels', so the
// values agree with theirs to rounding.  A CTA is one line: warp m solves
// system m.
// ---------------------------------------------------------------------------
template <class T, class W, int DIR>
__global__ void __launch_bounds__(128) k_psweep(Lv<T, W> L, Par P, int blo, int bhi) {
  pdl_wait();
  const int lane = threadIdx.x & 31, m = threadIdx.x >> 5;
  const int a = blockIdx.x + 1, b = blockIdx.y + 1;
  int n, st, sa;
  if (DIR == 0) { n = L.im - 2; st = 1; sa = L.sj; }
  else if (DIR == 1) { n = L.jm - 2; st = L.sj; sa = 1; }
  else { n = L.km - 2; st = L.sk; sa = 1; }
  const int ext = DIR == 0 ? L.oute : 0;
  const int N = n + ext;  // rows 1..N (N <= 32)
  const int base = (DIR == 2) ? L.sj * b : L.sk * b;
  const int lb = base + a * sa;
  const W* __restrict__ tc = L.tc[DIR];
  const W* __restrict__ hc = L.hc[DIR];
  W* __restrict__ r = L.wk[m];
  __shared__ W s_bv[2][4];
  __shared__ W s_d[4][33], s_u[4][33], s_l[4][33], s_b[4][33];
  if (threadIdx.x == 0 || threadIdx.x == 32) {
    const int hi = threadIdx.x == 32;
    T v[4] = {0, 0, 0, 0};
    if (DIR == 0) {
      if (!hi && blo) {
        const int S = L.jm * L.km, o = a + L.jm * b;
        face_vec<T, W, 0>(L, P, lb, 0, L.bi + o, L.bi + 4 * S + o, S, v);
      }
    } else if (DIR == 1) {
      const int S = L.im * L.km, o = a + L.im * b;
      if (!hi && blo) face_vec<T, W, 1>(L, P, lb, 2, L.bj + o, L.bj + 4 * S + o, S, v);
      if (hi && bhi) face_vec<T, W, 1>(L, P, lb + (n + 1) * st, 3, L.bj + 8 * S + o, L.bj + 12 * S + o, S, v);
    } else {
      const int S = L.im * L.jm, o = a + L.im * b;
      if (!hi && blo) face_vec<T, W, 2>(L, P, lb, 4, L.bk + o, L.bk + 4 * S + o, S, v);
      if (hi && bhi) face_vec<T, W, 2>(L, P, lb + (n + 1) * st, 5, L.bk + 8 * S + o, L.bk + 12 * S + o, S, v);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) s_bv[hi][q] = W(v[q]);
  }
  __syncthreads();
  // row p = lane + 1: aw x_{p-1} + ap x_p + ae x_{p+1} = d
  const int p = lane + 1;
  W aw = 0, ap = 1, ae = 0, d = 0;
  if (p <= N) {
    if (p <= n) {
      const W t = tc[lb + p * st];
      const W hw = hc[lb + (p - 1) * st], he = hc[lb + (p + 1) * st];
      const W dw = t != W(0) ? hw : W(0), de = t != W(0) ? he : W(0);
      if (m < 2) { aw = -t; ae = -t; }
      else if (m == 2) { aw = -dw - t; ae = de - t; }
      else { aw = dw - t; ae = -de - t; }
      ap = fmaw(W(2), t, W(1));
    } else {  // the outlet row (src/rhs_diag_solver.F90:207-221)
      ap = m == 2 ? fmaw(W(2), hc[lb + (n + 1) * st], W(1)) : W(1);
      aw = m == 2 ? -(W(2) * hc[lb + n * st]) : W(0);
      ae = W(0);
    }
    d = r[lb + p * st];
    if (p == 1) d = fmaw(-aw, s_bv[0][m], d);
    if (p == n && !ext) d = fmaw(-ae, s_bv[1][m], d);
  }
  if (p == 1) aw = W(0);        // the couplings outside the system
  if (p >= N) ae = W(0);
  // column test: |ap_p| >= |ae_{p-1}| + |aw_{p+1}|
  // (every lane takes part in each shuffle; the ends are masked afterwards)
  W aeprev = __shfl_up_sync(0xffffffffu, ae, 1);
  W awnext = __shfl_down_sync(0xffffffffu, aw, 1);
  if (lane == 0) aeprev = W(0);
  if (lane == 31) awnext = W(0);
  const bool bad = p <= N && dabs(ap) < dabs(aeprev) + dabs(awnext);
  if (!__any_sync(0xffffffffu, bad)) {
    W ca = aw, cb = ap, cc = ae, cd = d;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      W am = __shfl_up_sync(0xffffffffu, ca, s), bm = __shfl_up_sync(0xffffffffu, cb, s);
      W cm = __shfl_up_sync(0xffffffffu, cc, s), dm = __shfl_up_sync(0xffffffffu, cd, s);
      W aq = __shfl_down_sync(0xffffffffu, ca, s), bq = __shfl_down_sync(0xffffffffu, cb, s);
      W cq = __shfl_down_sync(0xffffffffu, cc, s), dq = __shfl_down_sync(0xffffffffu, cd, s);
      if (lane < s) { am = W(0); bm = W(1); cm = W(0); dm = W(0); }
      if (lane + s > 31) { aq = W(0); bq = W(1); cq = W(0); dq = W(0); }
      const W k1 = ca / bm, k2 = cc / bq;
      ca = -(k1 * am);
      cc = -(k2 * cq);
      cb = fmaw(-k2, aq, fmaw(-k1, cm, cb));
      cd = fmaw(-k2, dq, fmaw(-k1, dm, cd));
    }
    if (p <= N) {
      if (cb == W(0)) atomicAdd(&L.flags[1], 1);
      r[lb + p * st] = cd / cb;
    }
    return;
  }
  // ---- SGTSV's elimination with partial pivoting (src/sgtsv.f:107-162,
  // 232-257) by lane 0 on the rows in shared memory (index = row)
  if (p <= N) { s_d[m][p] = ap; s_u[m][p] = ae; s_l[m][p] = aw; s_b[m][p] = d; }
  __syncwarp();
  if (lane == 0) {
    W* dd = s_d[m]; W* du = s_u[m]; W* dl = s_l[m]; W* bq = s_b[m];
    int nsw = 0;
    bool sing = false;
    for (int q = 1; q <= N - 1 && !sing; ++q) {
      const W dlp = dl[q + 1], dp = dd[q];
      if (dabs(dp) >= dabs(dlp)) {
        if (dp != W(0)) {
          const W fact = dlp / dp;
          dd[q + 1] = fmaw(-fact, du[q], dd[q + 1]);
          bq[q + 1] = fmaw(-fact, bq[q], bq[q + 1]);
        } else {
          sing = true;
        }
        dl[q + 1] = W(0);
      } else {
        ++nsw;
        const W fact = dp / dlp;
        dd[q] = dlp;
        const W temp = dd[q + 1];
        dd[q + 1] = fmaw(-fact, temp, du[q]);
        if (q <= N - 2) {
          dl[q + 1] = du[q + 1];                 // fill-in of row q: du2
          du[q + 1] = -fact * dl[q + 1];
        } else {
          dl[q + 1] = W(0);
        }
        du[q] = temp;
        const W tb = bq[q];
        bq[q] = bq[q + 1];
        bq[q + 1] = fmaw(-fact, bq[q + 1], tb);
      }
    }
    if (sing || dd[N] == W(0)) {
      atomicAdd(&L.flags[1], 1);
    } else {
      bq[N] = bq[N] / dd[N];
      if (N > 1) bq[N - 1] = fmaw(-du[N - 1], bq[N], bq[N - 1]) / dd[N - 1];
      for (int q = N - 2; q >= 1; --q) bq[q] = fmaw(-dl[q + 1], bq[q + 2], fmaw(-du[q], bq[q + 1], bq[q])) / dd[q];
    }
    if (nsw) atomicAdd(&L.flags[0], nsw);
    atomicAdd(&L.flags[2], 1);
  }
  __syncwarp();
  if (p <= N) r[lb + p * st] = s_b[m][p];
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
