// mg.cuh -- boundary conditions, multigrid transfers, convergence norm and
// setup kernels.
#pragma once
#include "common.cuh"

namespace desalm {

// ---------------------------------------------------------------- bcond_fm
// One face pair per kernel, in the reference's order i faces, j faces,
// k faces (src/bcond_fm.F90:79-306); each thread owns one boundary column
// and applies the low face before the high face.  i_mysta/i_myend are the
// boundary nodes themselves there (src/bcond_fm.F90:60-66), so every kernel
// covers the full transverse range (edges and corners included).
// The k-face kernel also reads the pressure reference value p(ifix, jfix,
// kfix) after the face updates (src/bcond_fm.F90:310), in the thread of the
// (i, j) column through that node: it is the only one that writes there, and
// the i and j face kernels before it have finished.
template <class T, class W, int DIR>
__global__ void k_bcond(Lv<T, W> L, Par P, const T* rat, int ratdim, int fix_a, int fix_b, int lfix, T* pfix) {
  pdl_wait();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  int amax, n, st, lb;
  if (DIR == 0) { amax = L.jm; n = L.im; st = 1; lb = L.sj * a + L.sk * b; }
  else if (DIR == 1) { amax = L.im; n = L.jm; st = L.sj; lb = a + L.sk * b; }
  else { amax = L.im; n = L.km; st = L.sk; lb = a + L.sj * b; }
  if (a >= amax) return;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int bi = 2 * DIR + side;
    const int bt = P.btype[bi];
    const int l = side == 0 ? lb : lb + (n - 1) * st;
    const int s = side == 0 ? st : -st;
    if (bt >= 1 && bt <= 3) {
#pragma unroll
      for (int m = 0; m < 4; ++m) L.q[m][l] = T(P.sa[m][bi]) * L.q[m][l + s] + T(P.sb[m][bi]) * L.q[m][l + 2 * s];
    } else if (bt == 4) {
      T r = rat[bi * ratdim * ratdim + a + ratdim * b];
      L.q[0][l] = (T(1) + r) * L.q[0][l + s] - r * L.q[0][l + 2 * s];
    } else if (bt == 6 && DIR > 0) {
      const int lo = side == 0 ? lb + (n - 1) * st : lb;  // the opposite boundary node
#pragma unroll
      for (int m = 0; m < 4; ++m) L.q[m][l] = L.q[m][lo];
    } else if (bt == 8 && DIR == 0 && side == 1) {
#pragma unroll
      for (int m = 0; m < 4; ++m) L.q[m][l] = L.q[m][l - 1];
    }
  }
  if (DIR == 2 && a == fix_a && b == fix_b) *pfix = L.q[0][lfix];
}
// p <- p - pfix over the whole level (src/bcond_fm.F90:316-322)
template <class T, class W>
__global__ void k_pfix_sub(Lv<T, W> L, const T* pfix) {
  pdl_wait();
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L.N) return;
  L.q[0][l] = L.q[0][l] - *pfix;
}

// ---------------------------------------------------------------- transfers
// mg_nlevel (src/mg_nlevel.F90:19-146) + mg_zero_pk_boundary
// (src/mg_driver.F90:407-466): injection of q and nu_t, qold_mg <- q, and
// the 27-point full-weighting restriction of the fine residual into pk.
template <class TF, class WF, class TC, class WC>
__global__ void k_nlevel(Lv<TF, WF> F, Lv<TC, WC> C, int icrs, int jcrs, int kcrs) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (i >= C.im || j >= C.jm) return;
  const int l = i + C.sj * j + C.sk * k;
  const int ii = icrs ? 2 * i : i, jj = jcrs ? 2 * j : j, kk = kcrs ? 2 * k : k;
  const int ll = ii + F.sj * jj + F.sk * kk;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    TC v = TC(F.q[m][ll]);
    C.q[m][l] = v;
    C.qold[m][l] = v;
  }
  C.nut[l] = TC(F.nut[ll]);
  const bool bnd = i == 0 || i == C.im - 1 || j == 0 || j == C.jm - 1 || k == 0 || k == C.km - 1;
  if (bnd) {
#pragma unroll
    for (int m = 0; m < 4; ++m) C.pk[m][l] = TC(0);
    return;
  }
  const int ic = 1, ie = F.sj, iz = F.sk;
  const TF p25 = TF(0.25), p5 = TF(0.5), two = TF(2), s16 = TF(1) / TF(16);
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const TF* r = F.rh[m];
    TF s = p25 * r[ll + ic + ie + iz];
    s = s + p5 * r[ll + ic + ie];
    s = s + p25 * r[ll + ic + ie - iz];
    s = s + p5 * r[ll + ie + iz];
    s = s + r[ll + ie];
    s = s + p5 * r[ll + ie - iz];
    s = s + p25 * r[ll - ic + ie + iz];
    s = s + p5 * r[ll - ic + ie];
    s = s + p25 * r[ll - ic + ie - iz];
    s = s + p5 * r[ll + ic + iz];
    s = s + r[ll + ic];
    s = s + p5 * r[ll + ic - iz];
    s = s + r[ll + iz];
    s = s + two * r[ll];
    s = s + r[ll - iz];
    s = s + p5 * r[ll - ic + iz];
    s = s + r[ll - ic];
    s = s + p5 * r[ll - ic - iz];
    s = s + p25 * r[ll + ic - ie + iz];
    s = s + p5 * r[ll + ic - ie];
    s = s + p25 * r[ll + ic - ie - iz];
    s = s + p5 * r[ll - ie + iz];
    s = s + r[ll - ie];
    s = s + p5 * r[ll - ie - iz];
    s = s + p25 * r[ll - ic - ie + iz];
    s = s + p5 * r[ll - ic - ie];
    s = s + p25 * r[ll - ic - ie - iz];
    C.pk[m][l] = TC(s * s16);
  }
}

// Correction of one fine node from the coarse-grid change dq = q_c - qold_c,
// linearly interpolated along k, then j, then i exactly as the reference's
// three passes (src/mg_prolong.F90:59-170): each pass averages the two
// neighbours filled by the previous pass.
template <class TF, class WF, class TC, class WC>
struct Interp {
  const Lv<TF, WF>* F;
  const Lv<TC, WC>* C;
  int icrs, jcrs, kcrs;
  DESALM_DEV TF c(int i, int j, int k, int m) const {  // injected point
    const int ic = icrs ? i / 2 : i, jc = jcrs ? j / 2 : j, kc = kcrs ? k / 2 : k;
    const int l = ic + C->sj * jc + C->sk * kc;
    return TF(C->q[m][l] - C->qold[m][l]);
  }
  DESALM_DEV TF fk(int i, int j, int k, int m) const {
    if (kcrs && (k & 1)) return TF(0.5) * c(i, j, k + 1, m) + TF(0.5) * c(i, j, k - 1, m);
    return c(i, j, k, m);
  }
  DESALM_DEV TF fj(int i, int j, int k, int m) const {
    if (jcrs && (j & 1)) return TF(0.5) * fk(i, j + 1, k, m) + TF(0.5) * fk(i, j - 1, k, m);
    return fk(i, j, k, m);
  }
  DESALM_DEV TF fi(int i, int j, int k, int m) const {
    if (icrs && (i & 1)) return TF(0.5) * fj(i + 1, j, k, m) + TF(0.5) * fj(i - 1, j, k, m);
    return fj(i, j, k, m);
  }
};

template <class TF, class WF, class TC, class WC>
__global__ void k_prolong_interp(Lv<TF, WF> F, Lv<TC, WC> C, WF* dq, int icrs, int jcrs, int kcrs) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > F.im - 2 || j > F.jm - 2) return;
  const int l = i + F.sj * j + F.sk * k;
  Interp<TF, WF, TC, WC> I{&F, &C, icrs, jcrs, kcrs};
#pragma unroll
  for (int m = 0; m < 4; ++m) dq[m * F.N + l] = WF(I.fi(i, j, k, m));
}

// ---------------------------------------------------------------- norm
// Per-block partial sums of |q - qold| over interior nodes, 5 fields
// (src/mg_residual.F90:58-67); optionally qold <- q for the next iteration.
template <class T, class W>
__global__ void __launch_bounds__(256) k_norm_partial(Lv<T, W> L, double* part, int nf, int copy) {
  pdl_wait();
  __shared__ double sh[5][256];
  const int ni = L.im - 2, nj = L.jm - 2, nk = L.km - 2;
  const long total = (long)ni * nj * nk;
  double acc[5] = {0, 0, 0, 0, 0};
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int i = int(t % ni) + 1;
    const long r = t / ni;
    const int j = int(r % nj) + 1;
    const int k = int(r / nj) + 1;
    const int l = i + L.sj * j + L.sk * k;
    for (int m = 0; m < nf; ++m) {
      T q = L.q[m][l];
      acc[m] += double(dabs(q - L.qold[m][l]));
      if (copy) L.qold[m][l] = q;
    }
  }
  for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] += sh[m][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) part[blockIdx.x * 5 + m] = sh[m][0];
}

// Deterministic sum of nblk x 5 partials by one 256-thread block: strided
// per-thread sums, then a fixed tree; every thread receives the five sums.
DESALM_DEV void block_sum5(const double* part, int nblk, double out[5]) {
  __shared__ double sh[5][256];
  double acc[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x)
    for (int m = 0; m < 5; ++m) acc[m] += part[b * 5 + m];
  for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int m = 0; m < 5; ++m) sh[m][threadIdx.x] += sh[m][threadIdx.x + s];
    __syncthreads();
  }
  for (int m = 0; m < 5; ++m) out[m] = sh[m][0];
}

__global__ void __launch_bounds__(256) k_norm_final(const double* part, int nblk, double* out) {
  pdl_wait();
  double sums[5];
  block_sum5(part, nblk, sums);
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) out[m] = sums[m];
}

// ---------------------------------------------------------------- helpers
template <class T>
__global__ void k_fill(T* a, T v, long n) {
  pdl_wait();
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) a[t] = v;
}
template <class TD, class TS>
__global__ void k_copy(TD* d, const TS* s, long n) {
  pdl_wait();
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) d[t] = TD(s[t]);
}
// q^{n+1,(0)} = 2 q^n - q^{n-1}
template <class T>
__global__ void k_extrapolate(T* q, const T* qn, const T* qnm1, long n) {
  pdl_wait();
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) q[t] = T(2) * qn[t] - qnm1[t];
}
// Reference-layout AoS (me, i, j, k) <-> SoA
template <class T, class S = double>
__global__ void k_aos_to_soa(T* const* dst, const S* src, int me, long n) {
  pdl_wait();
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  for (int m = 0; m < me; ++m) dst[m][t] = T(src[t * me + m]);
}
template <class T, class D = double>
__global__ void k_soa_to_aos(D* dst, T* const* src, int me, long n) {
  pdl_wait();
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  for (int m = 0; m < me; ++m) dst[t * me + m] = D(src[m][t]);
}

// Injection of one scalar field to the next coarser level (src/mg_inject.F90:26-62)
template <class TF, class TC>
__global__ void k_inject(TC* c, const TF* f, int cim, int cjm, int ckm, int fim, int fjm, int icrs, int jcrs, int kcrs) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int k = blockIdx.z;
  if (i >= cim) return;
  const int ii = icrs ? 2 * i : i, jj = jcrs ? 2 * j : j, kk = kcrs ? 2 * k : k;
  c[i + cim * (j + cjm * k)] = TC(f[ii + fim * (jj + fjm * kk)]);
}

// r = 1 / a element-wise (the reciprocal Jacobian of a level)
template <class T>
__global__ void k_recip(T* r, const T* a, long n) {
  pdl_wait();
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) r[t] = T(1) / a[t];
}

// Covariant metrics, Jacobian and contravariant metrics of one level
// (src/mg_metrics.F90:56-250).  cov[9] = xc, xe, xz, yc, ye, yz, zc, ze, zz.
__global__ void k_metrics(const double* x, const double* y, const double* z, int im, int jm, int km,
                          double dc, double de, double dz, double* const* cov, double* const* met, double* aj) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int k = blockIdx.z;
  if (i >= im) return;
  const int sj = im, sk = im * jm;
  const int l = i + sj * j + sk * k;
  const double* P[3] = {x, y, z};
  double d[3][3];  // d[coord][dir]
  const int st[3] = {1, sj, sk};
  const int pos[3] = {i, j, k};
  const int ext[3] = {im, jm, km};
  const double sp[3] = {dc, de, dz};
  for (int dir = 0; dir < 3; ++dir) {
    for (int c = 0; c < 3; ++c) {
      const double* v = P[c];
      if (pos[dir] == 0) d[c][dir] = sp[dir] * (v[l + st[dir]] - v[l]);
      else if (pos[dir] == ext[dir] - 1) d[c][dir] = sp[dir] * (v[l] - v[l - st[dir]]);
      else d[c][dir] = (0.5 * sp[dir]) * (v[l + st[dir]] - v[l - st[dir]]);
    }
  }
  const double xc = d[0][0], xe = d[0][1], xz = d[0][2];
  const double yc = d[1][0], ye = d[1][1], yz = d[1][2];
  const double zc = d[2][0], ze = d[2][1], zz = d[2][2];
  cov[0][l] = xc; cov[1][l] = xe; cov[2][l] = xz;
  cov[3][l] = yc; cov[4][l] = ye; cov[5][l] = yz;
  cov[6][l] = zc; cov[7][l] = ze; cov[8][l] = zz;
  double gj = xc * (ye * zz - yz * ze) + xe * (yz * zc - yc * zz) + xz * (yc * ze - ye * zc);
  double a = 1.0 / gj;
  aj[l] = a;
  met[0][l] = a * (ye * zz - yz * ze); met[1][l] = a * (xz * ze - xe * zz); met[2][l] = a * (xe * yz - xz * ye);
  met[3][l] = a * (yz * zc - yc * zz); met[4][l] = a * (xc * zz - xz * zc); met[5][l] = a * (xz * yc - xc * yz);
  met[6][l] = a * (yc * ze - ye * zc); met[7][l] = a * (xe * zc - xc * ze); met[8][l] = a * (xc * ye - xe * yc);
}

// SA pseudo-time step on the fine level (src/mg_metrics.F90:262-282)
__global__ void k_dtev(double* const* cov, double* dtev, long n, double cfl2, double vnn2, double ren, double delti, int unsteady) {
  pdl_wait();
  long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  double xc = cov[0][l], xe = cov[1][l], xz = cov[2][l], yc = cov[3][l], ye = cov[4][l], yz = cov[5][l];
  double zc = cov[6][l], ze = cov[7][l], zz = cov[8][l];
  double Sc = sqrt(xc * xc + yc * yc + zc * zc);
  double Se = sqrt(xe * xe + ye * ye + ze * ze);
  double Sz = sqrt(xz * xz + yz * yz + zz * zz);
  double SL = fmin(Sc, fmin(Se, Sz));
  double dt = SL * fmin(cfl2, vnn2 * ren * SL);
  if (unsteady) dt = fmin(dt, delti * 2.0 / 3.0);
  dtev[l] = dt;
}

}  // namespace desalm

namespace desalm {

// Constant-coefficient implicit smoothing (-e, 1+2e, -e) of the four
// correction components along one direction (src/rs_sweep.F90:163-284), as a
// shared-memory slab: a CTA owns NL lines of one plane (kSlabThreads threads).
//   phase 0  the slab of dq is copied into shared memory (cp.async);
//   phase 1  thread (line, component m, half) eliminates the upper half of
//            its line top-down or the lower half bottom-up with SGTSV's
//            multipliers fac and eliminated diagonal dpr for this line length
//            (built on the host in SGTSV's order, with 1/dpr after dpr; the
//            matrix is symmetric Toeplitz, so the bottom-up factors are the
//            top-down ones mirrored); the halves meet in a 2x2 solve and
//            back-substitute, multiplying by 1/dpr;
//   phase 2  dq gets the smoothed values, or, after the last direction (k),
//            q += dq on the interior (src/mg_prolong.F90:218-277: dq is zero
//            on the boundary).
// The correction dq is held in the sweep precision WF (FP32 in MIXED mode: it
// is part of the coarse-grid correction, a preconditioner) and added to the
// FP64 state at the end.  Shared memory: 4 components of slab_fs(n, NL + 1)
// elements of WF.
template <class TF, class WF, int DIR, int NL>
__global__ void __launch_bounds__(kSlabThreads) k_rsmooth4(Lv<TF, WF> F, WF* dq, const double* fac, const double* dpr, double e, int last) {
  pdl_wait();
  constexpr int NT = kSlabThreads, NLP = NL + 1;
  extern __shared__ __align__(16) unsigned char rs_slab[];
  __shared__ WF s_top[NL][4], s_bot[NL][4];  // eliminated b of the two middle rows
  const int tid = threadIdx.x;
  const int a0 = blockIdx.x * NL + 1;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa, base;
  if (DIR == 0) { amax = F.jm - 2; n = F.im - 2; st = 1; sa = F.sj; base = F.sk * b; }
  else if (DIR == 1) { amax = F.im - 2; n = F.jm - 2; st = F.sj; sa = 1; base = F.sk * b; }
  else { amax = F.im - 2; n = F.km - 2; st = F.sk; sa = 1; base = F.sj * b; }
  const int nl = min(NL, amax - a0 + 1);
  const int fs = slab_fs(n, NLP);  // row p (node p + 1) of component m at m fs + p NLP + line
  WF* sv = reinterpret_cast<WF*>(rs_slab);
  const int total = nl * n;
  auto node = [&](int t, int& li, int& p) {
    if (DIR == 0) { li = t / n; p = t - li * n; }
    else { p = t / nl; li = t - p * nl; }
    return base + (a0 + li) * sa + (p + 1) * st;
  };

  // ---- phase 0
  for (int t = tid; t < total; t += NT) {
    int li, p;
    const int l = node(t, li, p);
#pragma unroll
    for (int m = 0; m < 4; ++m) cp_async_elem(sv + m * fs + p * NLP + li, dq + (long)m * F.N + l);
  }
  cp_async_wait_all();
  __syncthreads();

  // ---- phase 1
  const int li = tid % NL, combo = tid / NL;
  const int m = combo & 3, half = combo >> 2;
  const bool act = tid < 8 * NL && li < nl;  // solver threads
  WF* v = sv + m * fs + li;
  const WF off = WF(-e);
  const int h = n / 2;
  const double* rdpr = dpr + n;  // 1 / dpr
  if (act && half == 0) {
    WF bp = 0;
    for (int p = 0; p < h; ++p) {
      WF x = v[p * NLP];
      if (p > 0) x = x - WF(__ldg(fac + p - 1)) * bp;
      bp = x;
      v[p * NLP] = x;
    }
    s_top[li][m] = bp;
  } else if (act && half == 1) {
    WF bp = 0;
    for (int p = n - 1; p >= h; --p) {
      WF x = v[p * NLP];
      if (p < n - 1) x = x - WF(__ldg(fac + n - 2 - p)) * bp;
      bp = x;
      v[p * NLP] = x;
    }
    s_bot[li][m] = bp;
  }
  __syncthreads();
  if (act) {
    const WF d1 = WF(__ldg(dpr + h - 1)), d2 = WF(__ldg(dpr + n - 1 - h));
    const WF b1 = s_top[li][m], b2 = s_bot[li][m];
    const WF det = d1 * d2 - off * off;
    if (half == 0) {
      WF x = (b1 * d2 - off * b2) / det;
      v[(h - 1) * NLP] = x;
      for (int p = h - 2; p >= 0; --p) {
        x = (v[p * NLP] - off * x) * WF(__ldg(rdpr + p));
        v[p * NLP] = x;
      }
    } else {
      WF x = (d1 * b2 - off * b1) / det;
      v[h * NLP] = x;
      for (int p = h + 1; p < n; ++p) {
        x = (v[p * NLP] - off * x) * WF(__ldg(rdpr + n - 1 - p));
        v[p * NLP] = x;
      }
    }
  }
  __syncthreads();

  // ---- phase 2
  for (int t = tid; t < total; t += NT) {
    int lq, p;
    const int l = node(t, lq, p);
    const int so = p * NLP + lq;
    if (last) {
      TF qv[4];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) qv[mm] = F.q[mm][l];
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) F.q[mm][l] = qv[mm] + TF(sv[mm * fs + so]);
    } else {
#pragma unroll
      for (int mm = 0; mm < 4; ++mm) dq[(long)mm * F.N + l] = sv[mm * fs + so];
    }
  }
}

}  // namespace desalm
