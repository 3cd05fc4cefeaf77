// oracle_core.hpp -- CPU restatement of DES-ALM's pseudo-time iteration.
//
// TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
// against; nothing in the product links, loads or calls it.  It is used by
// tests/, by __graft_entry__.smoke() as the checker, and by bench.py's CPU
// baseline leg.
//
// Parity status: the reference (Fortran 90 + MPI) cannot be compiled here
// (no Fortran compiler, no MPI) and ships no tests, fixtures or golden vectors,
// so this restatement is *parity unpinned* against reference output.  It is
// pinned instead by the identities the tests check (analytic inverses of the
// modal matrices, tridiagonal solves against dense solves, restriction weights,
// free-stream preservation, affine metrics) and by committed golden vectors it
// produced itself (regression pins).
//
// Real = double is the FP64 oracle; Real = float mirrors the reference's own
// arithmetic (src/precision.F90:11, rdf = selected_real_kind(p=6)).  Loop
// ranges, update order and the order of floating-point operations inside each
// expression follow the reference routines cited at each function, for one
// rank (no ghost layers: igp = jgp = kgp = 0, every face is a domain boundary).
//
// Indexing: 1-based (i, j, k), i fastest, one contiguous array per field and
// level (the reference concatenates levels in one vector, src/init.F90:917-937;
// only the addressing differs).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

// Loop nests whose iterations write disjoint elements run on every host
// thread when the oracle is built with OpenMP (each element is computed by
// the same expressions in the same order, so the results do not depend on
// the thread count); reductions stay serial.
#ifdef _OPENMP
#define ORC_PARFOR _Pragma("omp parallel for schedule(static)")
#else
#define ORC_PARFOR
#endif
#include <algorithm>
#include <limits>
#include <stdexcept>
#include <chrono>
#include "desalm.h"

namespace orc {

template <class R>
struct Level {
  int im = 0, jm = 0, km = 0;
  long N = 0;
  R dc = 1, de = 1, dz = 1;  // inverse grid spacings, src/init.F90:1117-1121
  std::vector<R> x, y, z;
  std::vector<R> xc, xe, xz, yc, ye, yz, zc, ze, zz;  // covariant metrics
  std::vector<R> csi[3], eta[3], zet[3], aj;
  std::vector<R> q[5], qn[5], qnm1[5], qold[5];
  std::vector<R> rh[4], pk[4];
  std::vector<R> nut, wd, dtev;
  std::vector<R> dtau, diss1;
  inline long id(int i, int j, int k) const {
    return (long)(i - 1) + (long)im * ((long)(j - 1) + (long)jm * (long)(k - 1));
  }
  void alloc() {
    N = (long)im * jm * km;
    auto a = [&](std::vector<R>& v) { v.assign(N, R(0)); };
    a(x); a(y); a(z);
    a(xc); a(xe); a(xz); a(yc); a(ye); a(yz); a(zc); a(ze); a(zz);
    for (int d = 0; d < 3; ++d) { a(csi[d]); a(eta[d]); a(zet[d]); }
    a(aj);
    for (int m = 0; m < 5; ++m) { a(q[m]); a(qn[m]); a(qnm1[m]); a(qold[m]); }
    for (int m = 0; m < 4; ++m) { a(rh[m]); a(pk[m]); }
    a(nut); a(wd); a(dtev); a(dtau); a(diss1);
  }
};

// ---------------------------------------------------------------------------
// LAPACK SGTSV (src/sgtsv.f:1-263, LAPACK 3.0, vendored by the reference):
// Gaussian elimination with partial pivoting of a tridiagonal system.
// dl[0..n-2] sub-diagonal, d[0..n-1] diagonal, du[0..n-2] super-diagonal,
// b[r*ldb + i] for right-hand side r.  Arrays are overwritten as in LAPACK.
// Returns info (0, or the 1-based row of a zero pivot, at which point the
// routine returns with b partially eliminated -- the reference ignores info,
// src/rhs_diag_solver.F90:242-249).  *npiv counts row interchanges.
// ---------------------------------------------------------------------------
template <class R>
int gtsv(int n, int nrhs, R* dl, R* d, R* du, R* b, int ldb, long* npiv) {
  if (n <= 0) return 0;
  for (int i = 0; i < n - 2; ++i) {  // rows 1..n-2 (sgtsv.f:107-135 / 163-195)
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      if (d[i] != R(0)) {
        R fact = dl[i] / d[i];
        d[i + 1] = d[i + 1] - fact * du[i];
        for (int r = 0; r < nrhs; ++r) b[r * ldb + i + 1] = b[r * ldb + i + 1] - fact * b[r * ldb + i];
      } else {
        return i + 1;
      }
      dl[i] = R(0);
    } else {
      if (npiv) ++*npiv;
      R fact = d[i] / dl[i];
      d[i] = dl[i];
      R temp = d[i + 1];
      d[i + 1] = du[i] - fact * temp;
      dl[i] = du[i + 1];
      du[i + 1] = -fact * dl[i];
      du[i] = temp;
      for (int r = 0; r < nrhs; ++r) {
        R t = b[r * ldb + i];
        b[r * ldb + i] = b[r * ldb + i + 1];
        b[r * ldb + i + 1] = t - fact * b[r * ldb + i + 1];
      }
    }
  }
  if (n > 1) {  // last elimination row (sgtsv.f:136-157)
    int i = n - 2;
    if (std::fabs(d[i]) >= std::fabs(dl[i])) {
      if (d[i] != R(0)) {
        R fact = dl[i] / d[i];
        d[i + 1] = d[i + 1] - fact * du[i];
        for (int r = 0; r < nrhs; ++r) b[r * ldb + i + 1] = b[r * ldb + i + 1] - fact * b[r * ldb + i];
      } else {
        return i + 1;
      }
    } else {
      if (npiv) ++*npiv;
      R fact = d[i] / dl[i];
      d[i] = dl[i];
      R temp = d[i + 1];
      d[i + 1] = du[i] - fact * temp;
      du[i] = temp;
      for (int r = 0; r < nrhs; ++r) {
        R t = b[r * ldb + i];
        b[r * ldb + i] = b[r * ldb + i + 1];
        b[r * ldb + i + 1] = t - fact * b[r * ldb + i + 1];
      }
    }
  }
  if (d[n - 1] == R(0)) return n;
  for (int r = 0; r < nrhs; ++r) {  // back solve (sgtsv.f:232-257)
    R* x = b + (long)r * ldb;
    x[n - 1] = x[n - 1] / d[n - 1];
    if (n > 1) x[n - 2] = (x[n - 2] - du[n - 2] * x[n - 1]) / d[n - 2];
    for (int i = n - 3; i >= 0; --i) x[i] = (x[i] - du[i] * x[i + 1] - dl[i] * x[i + 2]) / d[i];
  }
  return 0;
}

// 4x4 matrix in Fortran order a(row, col) -> a[row][col], 0-based.
template <class R> struct M4 { R a[4][4]; };

// matmul(a, r) as gfortran evaluates it: rp(i) = sum over k = 1..4 in order.
template <class R>
inline void mv4(const M4<R>& A, const R* r, R* rp) {
  for (int i = 0; i < 4; ++i) {
    R s = A.a[i][0] * r[0];
    s = s + A.a[i][1] * r[1];
    s = s + A.a[i][2] * r[2];
    s = s + A.a[i][3] * r[3];
    rp[i] = s;
  }
}

template <class R>
inline M4<R> mm4(const M4<R>& A, const M4<R>& B) {
  M4<R> C;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      R s = A.a[i][0] * B.a[0][j];
      s = s + A.a[i][1] * B.a[1][j];
      s = s + A.a[i][2] * B.a[2][j];
      s = s + A.a[i][3] * B.a[3][j];
      C.a[i][j] = s;
    }
  return C;
}

// Eigenvector matrices of one direction (src/rhs_modal_matrices.F90:64-259):
// with metric vector (c1, c2, c3) and sigma, build M (= Ma, Mb or Mc) and its
// analytic inverse Mi.
template <class R>
inline void modal_pair(R c1, R c2, R c3, R sigma, M4<R>& M, M4<R>& Mi) {
  const R one = 1, two = 2, pt5 = R(0.5), zero = 0;
  R c1s = c1 * c1, c2s = c2 * c2, c3s = c3 * c3;
  R g = c1s + c2s + c3s;
  R sg = std::sqrt(g);
  R dd = c2 - c3;
  R s = std::sqrt(two * g + dd * dd);
  R dm = g + two * c2 * c3 + c1 * c1;
  R r1 = c2 + c3, r2 = c2 - c3, r3 = c2s - c3s;
  M.a[0][0] = zero; M.a[0][1] = zero; M.a[0][2] = sigma; M.a[0][3] = sigma;
  M.a[1][0] = -(c2 + c3) / s;
  M.a[1][1] = c1 * (c3 - c2) / (s * sg);
  M.a[1][2] = c1 / sg;
  M.a[1][3] = -c1 / sg;
  M.a[2][0] = c1 / s;
  M.a[2][1] = (g + c2 * (c3 - c2)) / (s * sg);
  M.a[2][2] = c2 / sg;
  M.a[2][3] = -c2 / sg;
  M.a[3][0] = c1 / s;
  M.a[3][1] = -(g - c3 * (c3 - c2)) / (s * sg);
  M.a[3][2] = c3 / sg;
  M.a[3][3] = -c3 / sg;
  Mi.a[0][0] = zero;
  Mi.a[0][1] = -s * (c2 + c3) / dm;
  Mi.a[0][2] = s * c1 / dm;
  Mi.a[0][3] = Mi.a[0][2];
  R ssgd = s / sg / dm;
  R sgd2 = one / sg / dm / two;
  Mi.a[1][0] = zero;
  Mi.a[1][1] = c1 * (c3 - c2) * ssgd;
  Mi.a[1][2] = (c2 * c3 + c1s + c3s) * ssgd;
  Mi.a[1][3] = -(c2 * c3 + c1s + c2s) * ssgd;
  Mi.a[2][0] = pt5 / sigma;
  Mi.a[2][1] = c1 * (two * g + two * c2 * c3 - c2s - c3s) * sgd2;
  Mi.a[2][2] = (g * r1 + c1s * r2 + c3 * r3) * sgd2;
  Mi.a[2][3] = (g * r1 - c1s * r2 - c2 * r3) * sgd2;
  Mi.a[3][0] = pt5 / sigma;
  Mi.a[3][1] = -Mi.a[2][1];
  Mi.a[3][2] = -Mi.a[2][2];
  Mi.a[3][3] = -Mi.a[2][3];
}

template <class R>
struct Solver {
  desalm_case c;
  int ng;
  std::vector<Level<R>> L;  // L[0] = fine
  R sa[5][6], sb[5][6];     // src/init.F90:482-509
  std::vector<R> rat[6];    // src/init.F90:2750-2891
  int ratdim = 0;
  R es;                     // e_source
  bool have_grid = false, have_state = false;
  long pivots = 0;
  int itc = 0;
  R init_resd[5];
  double phase_s[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // residual, modal+sweeps, bc, transfers, sa, norm
  std::string err;

  // actuator-line forcing: the tables init_lines builds (src/init.F90:1156-1710)
  struct AlmTur {
    int nblades = 0, nelems = 0, nangles = 0, nker = 0;
    R tsr = 0, tur_rad = 0, hub_rad = 0, angle = 0;
    std::vector<int> node_index, polar_b, polar_a, ker_index;
    std::vector<R> node_pos, disk_dat, ker_pos, ker_dat;
  };
  bool alm_on = false;
  std::vector<AlmTur> alm;
  R alm_vel_infty = 0, alm_length_scale = 1;
  std::vector<int> polar_off, polar_cnt;
  std::vector<R> polar_rows;
  std::vector<R> forces_lines;  // (xf, yf, zf, fx, fy, fz) per turbine, blade, element
  std::vector<R> falm[3];       // what rhs_lines added to rh(2:4)

  explicit Solver(const desalm_case& cc) : c(cc) {
    ng = c.ng;
    L.resize(ng);
    L[0].im = c.im; L[0].jm = c.jm; L[0].km = c.km;
    for (int n = 1; n < ng; ++n) {  // src/init.F90:257-263
      L[n].im = (L[n - 1].im + c.icrs) / (1 << c.icrs);
      L[n].jm = (L[n - 1].jm + c.jcrs) / (1 << c.jcrs);
      L[n].km = (L[n - 1].km + c.kcrs) / (1 << c.kcrs);
    }
    for (int n = 0; n < ng; ++n) {
      L[n].dc = R(1) / std::pow(R(2), R(n * c.icrs));
      L[n].de = R(1) / std::pow(R(2), R(n * c.jcrs));
      L[n].dz = R(1) / std::pow(R(2), R(n * c.kcrs));
      L[n].alloc();
    }
    es = c.unsteady ? R(1) : R(0);
    // sa / sb: first-order extrapolation 4/3, -1/3; wall: no-slip; symmetry:
    // zero normal velocity (src/init.F90:482-509)
    for (int m = 0; m < 5; ++m)
      for (int b = 0; b < 6; ++b) { sa[m][b] = R(4) / R(3); sb[m][b] = -(R(1) / R(3)); }
    for (int b = 0; b < 6; ++b) {
      if (c.btype[b] == 1) for (int m = 1; m < 4; ++m) { sa[m][b] = 0; sb[m][b] = 0; }
      if (c.btype[b] == 2) {
        int m = c.bdir[b];  // 1 -> u, 2 -> v, 3 -> w
        if (m >= 1 && m <= 3) { sa[m][b] = 0; sb[m][b] = 0; }
      }
    }
    if (c.turbulence == 2) { om.assign(L[0].N, R(0)); omn = om; omnm1 = om; }
    ratdim = std::max(c.im, std::max(c.jm, c.km));
    for (int b = 0; b < 6; ++b) rat[b].assign((long)ratdim * ratdim, R(0));
    for (int m = 0; m < 5; ++m) init_resd[m] = 0;
  }

  // ---------------------------------------------------------------- setup
  // mg_inject for one scalar field (src/mg_inject.F90:26-62)
  void inject(std::vector<R> Level<R>::*f) {
    for (int n = 1; n < ng; ++n) {
      Level<R>& C = L[n]; Level<R>& F = L[n - 1];
      for (int k = 1; k <= C.km; ++k)
        for (int j = 1; j <= C.jm; ++j)
          for (int i = 1; i <= C.im; ++i) {
            int kk = (1 << c.kcrs) * k - c.kcrs, jj = (1 << c.jcrs) * j - c.jcrs, ii = (1 << c.icrs) * i - c.icrs;
            (C.*f)[C.id(i, j, k)] = (F.*f)[F.id(ii, jj, kk)];
          }
    }
  }
  void inject_arr(std::vector<R> (Level<R>::*f)[5], int m) {
    for (int n = 1; n < ng; ++n) {
      Level<R>& C = L[n]; Level<R>& F = L[n - 1];
      for (int k = 1; k <= C.km; ++k)
        for (int j = 1; j <= C.jm; ++j)
          for (int i = 1; i <= C.im; ++i) {
            int kk = (1 << c.kcrs) * k - c.kcrs, jj = (1 << c.jcrs) * j - c.jcrs, ii = (1 << c.icrs) * i - c.icrs;
            (C.*f)[m][C.id(i, j, k)] = (F.*f)[m][F.id(ii, jj, kk)];
          }
    }
  }

  // Metrics and Jacobian on every level (src/mg_metrics.F90:56-250) and the
  // SA pseudo-time step (src/mg_metrics.F90:262-282).
  void metrics() {
    for (int n = 0; n < ng; ++n) {
      Level<R>& G = L[n];
      const int im = G.im, jm = G.jm, km = G.km;
      R dum1 = G.dc, dum = R(0.5) * G.dc;
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
          for (int i = 2; i <= im - 1; ++i) {
            long l = G.id(i, j, k), lp = G.id(i + 1, j, k), lm = G.id(i - 1, j, k);
            G.xc[l] = dum * (G.x[lp] - G.x[lm]); G.yc[l] = dum * (G.y[lp] - G.y[lm]); G.zc[l] = dum * (G.z[lp] - G.z[lm]);
          }
          long l = G.id(1, j, k), lp = G.id(2, j, k);
          G.xc[l] = dum1 * (G.x[lp] - G.x[l]); G.yc[l] = dum1 * (G.y[lp] - G.y[l]); G.zc[l] = dum1 * (G.z[lp] - G.z[l]);
          l = G.id(im, j, k); long lm = G.id(im - 1, j, k);
          G.xc[l] = dum1 * (G.x[l] - G.x[lm]); G.yc[l] = dum1 * (G.y[l] - G.y[lm]); G.zc[l] = dum1 * (G.z[l] - G.z[lm]);
        }
      dum1 = G.de; dum = R(0.5) * G.de;
      for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) {
          for (int j = 2; j <= jm - 1; ++j) {
            long l = G.id(i, j, k), lp = G.id(i, j + 1, k), lm = G.id(i, j - 1, k);
            G.xe[l] = dum * (G.x[lp] - G.x[lm]); G.ye[l] = dum * (G.y[lp] - G.y[lm]); G.ze[l] = dum * (G.z[lp] - G.z[lm]);
          }
          long l = G.id(i, 1, k), lp = G.id(i, 2, k);
          G.xe[l] = dum1 * (G.x[lp] - G.x[l]); G.ye[l] = dum1 * (G.y[lp] - G.y[l]); G.ze[l] = dum1 * (G.z[lp] - G.z[l]);
          l = G.id(i, jm, k); long lm = G.id(i, jm - 1, k);
          G.xe[l] = dum1 * (G.x[l] - G.x[lm]); G.ye[l] = dum1 * (G.y[l] - G.y[lm]); G.ze[l] = dum1 * (G.z[l] - G.z[lm]);
        }
      dum1 = G.dz; dum = R(0.5) * G.dz;
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          for (int k = 2; k <= km - 1; ++k) {
            long l = G.id(i, j, k), lp = G.id(i, j, k + 1), lm = G.id(i, j, k - 1);
            G.xz[l] = dum * (G.x[lp] - G.x[lm]); G.yz[l] = dum * (G.y[lp] - G.y[lm]); G.zz[l] = dum * (G.z[lp] - G.z[lm]);
          }
          long l = G.id(i, j, 1), lp = G.id(i, j, 2);
          G.xz[l] = dum1 * (G.x[lp] - G.x[l]); G.yz[l] = dum1 * (G.y[lp] - G.y[l]); G.zz[l] = dum1 * (G.z[lp] - G.z[l]);
          l = G.id(i, j, km); long lm = G.id(i, j, km - 1);
          G.xz[l] = dum1 * (G.x[l] - G.x[lm]); G.yz[l] = dum1 * (G.y[l] - G.y[lm]); G.zz[l] = dum1 * (G.z[l] - G.z[lm]);
        }
      for (long l = 0; l < G.N; ++l) {
        R xc = G.xc[l], xe = G.xe[l], xz = G.xz[l], yc = G.yc[l], ye = G.ye[l], yz = G.yz[l];
        R zc = G.zc[l], ze = G.ze[l], zz = G.zz[l];
        R gj = xc * (ye * zz - yz * ze) + xe * (yz * zc - yc * zz) + xz * (yc * ze - ye * zc);
        R a = R(1) / gj;
        G.aj[l] = a;
        G.csi[0][l] = a * (ye * zz - yz * ze); G.csi[1][l] = a * (xz * ze - xe * zz); G.csi[2][l] = a * (xe * yz - xz * ye);
        G.eta[0][l] = a * (yz * zc - yc * zz); G.eta[1][l] = a * (xc * zz - xz * zc); G.eta[2][l] = a * (xz * yc - xc * yz);
        G.zet[0][l] = a * (yc * ze - ye * zc); G.zet[1][l] = a * (xe * zc - xc * ze); G.zet[2][l] = a * (xc * ye - xe * yc);
      }
    }
    Level<R>& F = L[0];
    for (long l = 0; l < F.N; ++l) {
      R Sc = std::sqrt(F.xc[l] * F.xc[l] + F.yc[l] * F.yc[l] + F.zc[l] * F.zc[l]);
      R Se = std::sqrt(F.xe[l] * F.xe[l] + F.ye[l] * F.ye[l] + F.ze[l] * F.ze[l]);
      R Sz = std::sqrt(F.xz[l] * F.xz[l] + F.yz[l] * F.yz[l] + F.zz[l] * F.zz[l]);
      R SL = std::min(Sc, std::min(Se, Sz));
      R dt = SL * std::min(R(c.cfl2), R(c.vnn2) * R(c.ren) * SL);
      if (c.unsteady) dt = std::min(dt, R(c.delti) * R(2) / R(3));
      F.dtev[l] = dt;
    }
  }

  // Inflow extrapolation ratios (src/init.F90:2750-2891).  For the k faces
  // the reference's guard 'btype == 4 .and. btype == 5' is never true, so
  // rat(:,:,5:6) is never assigned; this restatement keeps them zero.
  void outlet_ratios() {
    Level<R>& F = L[0];
    const int im = F.im, jm = F.jm, km = F.km;
    auto X = [&](int dir) -> std::vector<R>& { return dir == 1 ? F.x : (dir == 2 ? F.y : F.z); };
    for (int b = 0; b < 4; ++b) {
      if (!(c.btype[b] == 4 || c.btype[b] == 5)) continue;
      int dir = c.bdir[b];
      if (dir < 1 || dir > 3) continue;
      std::vector<R>& v = X(dir);
      if (b < 2) {
        for (int k = 1; k <= km; ++k)
          for (int j = 1; j <= jm; ++j) {
            R r;
            if (b == 0) { long l0 = F.id(1, j, k), l1 = F.id(2, j, k), l2 = F.id(3, j, k); r = (v[l1] - v[l0]) / (v[l2] - v[l1]); }
            else { long l0 = F.id(im, j, k), l1 = F.id(im - 1, j, k), l2 = F.id(im - 2, j, k); r = (v[l0] - v[l1]) / (v[l1] - v[l2]); }
            rat[b][(long)(j - 1) + (long)ratdim * (k - 1)] = r;
          }
      } else {
        for (int k = 1; k <= km; ++k)
          for (int i = 1; i <= im; ++i) {
            R r;
            if (b == 2) { long l0 = F.id(i, 1, k), l1 = F.id(i, 2, k), l2 = F.id(i, 3, k); r = (v[l1] - v[l0]) / (v[l2] - v[l1]); }
            else { long l0 = F.id(i, jm, k), l1 = F.id(i, jm - 1, k), l2 = F.id(i, jm - 2, k); r = (v[l0] - v[l1]) / (v[l1] - v[l2]); }
            rat[b][(long)(i - 1) + (long)ratdim * (k - 1)] = r;
          }
      }
    }
  }
  inline R ratv(int b, int a1, int a2) const { return rat[b][(long)(a1 - 1) + (long)ratdim * (a2 - 1)]; }

  void set_grid(const double* x, const double* y, const double* z, const double* wd) {
    Level<R>& F = L[0];
    for (long l = 0; l < F.N; ++l) {
      F.x[l] = R(x[l]); F.y[l] = R(y[l]); F.z[l] = R(z[l]);
      F.wd[l] = wd ? R(wd[l]) : R(0);
    }
    inject(&Level<R>::x); inject(&Level<R>::y); inject(&Level<R>::z); inject(&Level<R>::wd);
    metrics();
    outlet_ratios();
    have_grid = true;
  }

  // ------------------------------------------------------- residual pieces
  // rhs_contra_j (src/rhs_contra_j.F90:14-29) on all nodes.
  void contra_j(const Level<R>& G, std::vector<R>* ucn) const {
    ORC_PARFOR
    for (long l = 0; l < G.N; ++l) {
      R tmp = R(1) / G.aj[l];
      R u = G.q[1][l], v = G.q[2][l], w = G.q[3][l];
      ucn[0][l] = tmp * (G.csi[0][l] * u + G.csi[1][l] * v + G.csi[2][l] * w);
      ucn[1][l] = tmp * (G.eta[0][l] * u + G.eta[1][l] * v + G.eta[2][l] * w);
      ucn[2][l] = tmp * (G.zet[0][l] * u + G.zet[1][l] * v + G.zet[2][l] * w);
    }
  }

  // rhs_daf_dtau (src/rhs_daf_dtau.F90:34-117) on all nodes.
  void daf_dtau(Level<R>& G) const {
    const R cfl = R(c.cfl1), vnn = R(c.vnn1), rei = R(1) / R(c.ren);
    const R dcsq = G.dc * G.dc, desq = G.de * G.de, dzsq = G.dz * G.dz;
    ORC_PARFOR
    for (long l = 0; l < G.N; ++l) {
      R g1 = G.csi[0][l] * G.csi[0][l] + G.csi[1][l] * G.csi[1][l] + G.csi[2][l] * G.csi[2][l];
      R g2 = G.eta[0][l] * G.eta[0][l] + G.eta[1][l] * G.eta[1][l] + G.eta[2][l] * G.eta[2][l];
      R g3 = G.zet[0][l] * G.zet[0][l] + G.zet[1][l] * G.zet[1][l] + G.zet[2][l] * G.zet[2][l];
      R e1 = std::sqrt(g1), e2 = std::sqrt(g2), e3 = std::sqrt(g3);
      R dti1 = cfl / e1 / G.dc, dti2 = cfl / e2 / G.de, dti3 = cfl / e3 / G.dz;
      R ret = rei + G.nut[l];
      R dtv1 = vnn / ret / dcsq / g1, dtv2 = vnn / ret / desq / g2, dtv3 = vnn / ret / dzsq / g3;
      R m = dti1;
      m = std::min(m, dti2); m = std::min(m, dti3); m = std::min(m, dtv1); m = std::min(m, dtv2); m = std::min(m, dtv3);
      G.dtau[l] = m;
    }
  }

  // rhs_viscous (src/rhs_viscous.F90:55-329): visc(1:3) on interior nodes.
  void viscous(const Level<R>& G, std::vector<R>* visc) const {
    const int im = G.im, jm = G.jm, km = G.km;
    const R rei = R(1) / R(c.ren);
    const R dc = G.dc, de = G.de, dz = G.dz;
    const R dc4 = R(0.25) * dc, de4 = R(0.25) * de, dz4 = R(0.25) * dz;
    std::vector<R> fv[3];
    for (int m = 0; m < 3; ++m) { fv[m].assign(G.N, R(0)); visc[m].assign(G.N, R(0)); }
    auto ret = [&](long l) { return rei + G.nut[l]; };
    const std::vector<R>* Q = G.q;
    // face flux between nodes l0 and l1 = l0 + step along direction dir.
    // da/db/dc are derivatives along csi/eta/zet; pick the face normal's pair.
    auto flux = [&](int dir, long l0, long l1, R uc, R vc, R wc, R ue, R ve, R we, R uz, R vz, R wz, R* out) {
      R a1 = G.csi[0][l1] + G.csi[0][l0], a2 = G.csi[1][l1] + G.csi[1][l0], a3 = G.csi[2][l1] + G.csi[2][l0];
      R b1 = G.eta[0][l1] + G.eta[0][l0], b2 = G.eta[1][l1] + G.eta[1][l0], b3 = G.eta[2][l1] + G.eta[2][l0];
      R c1 = G.zet[0][l1] + G.zet[0][l0], c2 = G.zet[1][l1] + G.zet[1][l0], c3 = G.zet[2][l1] + G.zet[2][l0];
      R uu1 = a1 * uc + b1 * ue + c1 * uz, vv1 = a1 * vc + b1 * ve + c1 * vz, ww1 = a1 * wc + b1 * we + c1 * wz;
      R uu2 = a2 * uc + b2 * ue + c2 * uz, vv2 = a2 * vc + b2 * ve + c2 * vz, ww2 = a2 * wc + b2 * we + c2 * wz;
      R uu3 = a3 * uc + b3 * ue + c3 * uz, vv3 = a3 * vc + b3 * ve + c3 * vz, ww3 = a3 * wc + b3 * we + c3 * wz;
      R n1, n2, n3, k1, k2, k3;
      if (dir == 0) { n1 = a1; n2 = a2; n3 = a3; k1 = a1 * a1 + a2 * a2 + a3 * a3; k2 = a1 * b1 + a2 * b2 + a3 * b3; k3 = a1 * c1 + a2 * c2 + a3 * c3; }
      else if (dir == 1) { n1 = b1; n2 = b2; n3 = b3; k1 = b1 * a1 + b2 * a2 + b3 * a3; k2 = b1 * b1 + b2 * b2 + b3 * b3; k3 = b1 * c1 + b2 * c2 + b3 * c3; }
      else { n1 = c1; n2 = c2; n3 = c3; k1 = c1 * a1 + c2 * a2 + c3 * a3; k2 = c1 * b1 + c2 * b2 + c3 * b3; k3 = c1 * c1 + c2 * c2 + c3 * c3; }
      R vtj = R(0.25) * (ret(l1) + ret(l0)) / (G.aj[l1] + G.aj[l0]);
      out[0] = vtj * (n1 * uu1 + n2 * vv1 + n3 * ww1 + k1 * uc + k2 * ue + k3 * uz);
      out[1] = vtj * (n1 * uu2 + n2 * vv2 + n3 * ww2 + k1 * vc + k2 * ve + k3 * vz);
      out[2] = vtj * (n1 * uu3 + n2 * vv3 + n3 * ww3 + k1 * wc + k2 * we + k3 * wz);
    };
    // csi faces (src/rhs_viscous.F90:112-166)
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 1; i <= im - 1; ++i) {
          long l0 = G.id(i, j, k), l1 = G.id(i + 1, j, k);
          long a = G.id(i + 1, j + 1, k), b = G.id(i + 1, j - 1, k), cc = G.id(i, j + 1, k), d = G.id(i, j - 1, k);
          long e = G.id(i + 1, j, k + 1), f = G.id(i + 1, j, k - 1), g = G.id(i, j, k + 1), h = G.id(i, j, k - 1);
          R U[3], E[3], Z[3];
          for (int m = 0; m < 3; ++m) {
            const std::vector<R>& v = Q[m + 1];
            U[m] = dc * (v[l1] - v[l0]);
            E[m] = de4 * (v[a] - v[b] + v[cc] - v[d]);
            Z[m] = dz4 * (v[e] - v[f] + v[g] - v[h]);
          }
          R o[3];
          flux(0, l0, l1, U[0], U[1], U[2], E[0], E[1], E[2], Z[0], Z[1], Z[2], o);
          for (int m = 0; m < 3; ++m) fv[m][l0] = o[m];
        }
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k), lm = G.id(i - 1, j, k);
          for (int m = 0; m < 3; ++m) visc[m][l] = dc * (fv[m][l] - fv[m][lm]);
        }
    // eta faces (src/rhs_viscous.F90:189-243)
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 1; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l0 = G.id(i, j, k), l1 = G.id(i, j + 1, k);
          long a = G.id(i + 1, j + 1, k), b = G.id(i - 1, j + 1, k), cc = G.id(i + 1, j, k), d = G.id(i - 1, j, k);
          long e = G.id(i, j + 1, k + 1), f = G.id(i, j + 1, k - 1), g = G.id(i, j, k + 1), h = G.id(i, j, k - 1);
          R U[3], E[3], Z[3];
          for (int m = 0; m < 3; ++m) {
            const std::vector<R>& v = Q[m + 1];
            U[m] = dc4 * (v[a] - v[b] + v[cc] - v[d]);
            E[m] = de * (v[l1] - v[l0]);
            Z[m] = dz4 * (v[e] - v[f] + v[g] - v[h]);
          }
          R o[3];
          flux(1, l0, l1, U[0], U[1], U[2], E[0], E[1], E[2], Z[0], Z[1], Z[2], o);
          for (int m = 0; m < 3; ++m) fv[m][l0] = o[m];
        }
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k), lm = G.id(i, j - 1, k);
          for (int m = 0; m < 3; ++m) visc[m][l] = visc[m][l] + de * (fv[m][l] - fv[m][lm]);
        }
    // zeta faces (src/rhs_viscous.F90:263-316)
    ORC_PARFOR
    for (int k = 1; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l0 = G.id(i, j, k), l1 = G.id(i, j, k + 1);
          long a = G.id(i + 1, j, k + 1), b = G.id(i - 1, j, k + 1), cc = G.id(i + 1, j, k), d = G.id(i - 1, j, k);
          long e = G.id(i, j + 1, k + 1), f = G.id(i, j - 1, k + 1), g = G.id(i, j + 1, k), h = G.id(i, j - 1, k);
          R U[3], E[3], Z[3];
          for (int m = 0; m < 3; ++m) {
            const std::vector<R>& v = Q[m + 1];
            U[m] = dc4 * (v[a] - v[b] + v[cc] - v[d]);
            E[m] = de4 * (v[e] - v[f] + v[g] - v[h]);
            Z[m] = dz * (v[l1] - v[l0]);
          }
          R o[3];
          flux(2, l0, l1, U[0], U[1], U[2], E[0], E[1], E[2], Z[0], Z[1], Z[2], o);
          for (int m = 0; m < 3; ++m) fv[m][l0] = o[m];
        }
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k), lm = G.id(i, j, k - 1);
          for (int m = 0; m < 3; ++m) visc[m][l] = visc[m][l] + dz * (fv[m][l] - fv[m][lm]);
        }
  }

  // rhs_diss_p (src/rhs_diss_p.F90:33-203): diss(1) on interior nodes.
  void diss_p(Level<R>& G) const {
    const int im = G.im, jm = G.jm, km = G.km;
    const R dcsq = G.dc * G.dc, desq = G.de * G.de, dzsq = G.dz * G.dz;
    std::vector<R> fv[3];
    for (int m = 0; m < 3; ++m) fv[m].assign(G.N, R(0));
    const std::vector<R>& p = G.q[0];
    ORC_PARFOR
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k);
          R g1 = G.csi[0][l] * G.csi[0][l] + G.csi[1][l] * G.csi[1][l] + G.csi[2][l] * G.csi[2][l];
          R tmp1 = g1 * G.dtau[l] / G.aj[l];
          R tmp2 = dcsq * (p[G.id(i + 1, j, k)] - R(2) * p[l] + p[G.id(i - 1, j, k)]);
          fv[0][l] = tmp1 * tmp2;
        }
    ORC_PARFOR
    for (int k = 1; k <= km; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 1; i <= im; ++i) {
          long l = G.id(i, j, k);
          R g2 = G.eta[0][l] * G.eta[0][l] + G.eta[1][l] * G.eta[1][l] + G.eta[2][l] * G.eta[2][l];
          R tmp1 = g2 * G.dtau[l] / G.aj[l];
          R tmp2 = desq * (p[G.id(i, j + 1, k)] - R(2) * p[l] + p[G.id(i, j - 1, k)]);
          fv[1][l] = tmp1 * tmp2;
        }
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          long l = G.id(i, j, k);
          R g3 = G.zet[0][l] * G.zet[0][l] + G.zet[1][l] * G.zet[1][l] + G.zet[2][l] * G.zet[2][l];
          R tmp1 = g3 * G.dtau[l] / G.aj[l];
          R tmp2 = dzsq * (p[G.id(i, j, k + 1)] - R(2) * p[l] + p[G.id(i, j, k - 1)]);
          fv[2][l] = tmp1 * tmp2;
        }
    // boundary copies (src/rhs_diss_p.F90:124-129)
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j) {
        fv[0][G.id(1, j, k)] = fv[0][G.id(2, j, k)];
        fv[0][G.id(im, j, k)] = fv[0][G.id(im - 1, j, k)];
      }
    for (int k = 1; k <= km; ++k)
      for (int i = 1; i <= im; ++i) {
        fv[1][G.id(i, 1, k)] = fv[1][G.id(i, 2, k)];
        fv[1][G.id(i, jm, k)] = fv[1][G.id(i, jm - 1, k)];
      }
    for (int j = 1; j <= jm; ++j)
      for (int i = 1; i <= im; ++i) {
        fv[2][G.id(i, j, 1)] = fv[2][G.id(i, j, 2)];
        fv[2][G.id(i, j, km)] = fv[2][G.id(i, j, km - 1)];
      }
    std::fill(G.diss1.begin(), G.diss1.end(), R(0));
    const R pd = R(c.pdiss_coef);
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k);
          G.diss1[l] = pd * ((fv[0][G.id(i + 1, j, k)] - R(2) * fv[0][l] + fv[0][G.id(i - 1, j, k)]) +
                             (fv[1][G.id(i, j + 1, k)] - R(2) * fv[1][l] + fv[1][G.id(i, j - 1, k)]) +
                             (fv[2][G.id(i, j, k + 1)] - R(2) * fv[2][l] + fv[2][G.id(i, j, k - 1)]));
        }
  }

  // rhs_flux_sans_convec (src/rhs_flux_sans_convec.F90:44-136): assigns
  // rh(1:4) on interior nodes.
  void flux_sans_convec(Level<R>& G, const std::vector<R>* ucn) const {
    const int im = G.im, jm = G.jm, km = G.km;
    const R dc2 = R(0.5) * G.dc, de2 = R(0.5) * G.de, dz2 = R(0.5) * G.dz;
    std::vector<R> p(G.N, R(0));
    for (long l = 0; l < G.N; ++l) p[l] = G.q[0][l] / G.aj[l];
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k);
          long ip = G.id(i + 1, j, k), imn = G.id(i - 1, j, k);
          long jp = G.id(i, j + 1, k), jmn = G.id(i, j - 1, k);
          long kp = G.id(i, j, k + 1), kmn = G.id(i, j, k - 1);
          for (int d = 0; d < 3; ++d) {
            R v = dc2 * (p[ip] * G.csi[d][ip] - p[imn] * G.csi[d][imn]);
            v = v + de2 * (p[jp] * G.eta[d][jp] - p[jmn] * G.eta[d][jmn]);
            v = v + dz2 * (p[kp] * G.zet[d][kp] - p[kmn] * G.zet[d][kmn]);
            G.rh[d + 1][l] = v;
          }
          R dudx = dc2 * (ucn[0][ip] - ucn[0][imn]);
          R dvdy = de2 * (ucn[1][jp] - ucn[1][jmn]);
          R dwdz = dz2 * (ucn[2][kp] - ucn[2][kmn]);
          G.rh[0][l] = dudx + dvdy + dwdz;
        }
  }

  // rhs_convec_quick (src/rhs_convec_quick.F90:53-433): adds the momentum
  // convection.  decide_upwind = 1: first-order upwind everywhere; 2: QUICK
  // (coefficient 1/8) with first-order upwind at the nodes next to boundaries.
  void convec_quick(Level<R>& G, const std::vector<R>* ucn, int upwind) const {
    const int im = G.im, jm = G.jm, km = G.km;
    const R coef = R(0.125);
    const R dsp[3] = {G.dc, G.de, G.dz};
    const int ext[3] = {im, jm, km};
    for (int dir = 0; dir < 3; ++dir) {
      const long st = dir == 0 ? 1 : (dir == 1 ? (long)im : (long)im * jm);
      const R h = dsp[dir];
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = G.id(i, j, k);
            int pos = dir == 0 ? i : (dir == 1 ? j : k);
            R ucon = R(0.5) * ucn[dir][l];
            R up = ucon + std::fabs(ucon), um = ucon - std::fabs(ucon);
            bool first = (upwind == 1) || pos == 2 || pos == ext[dir] - 1;
            for (int m = 0; m < 3; ++m) {
              const std::vector<R>& v = G.q[m + 1];
              R f;
              if (first) {
                f = h * (up * (v[l] - v[l - st]) + um * (v[l + st] - v[l]));
              } else {
                f = coef * h * (up * (R(3) * v[l + st] + R(3) * v[l] - R(7) * v[l - st] + v[l - 2 * st]) +
                                um * (-R(3) * v[l - st] - R(3) * v[l] + R(7) * v[l + st] - v[l + 2 * st]));
              }
              G.rh[m + 1][l] = G.rh[m + 1][l] + f;
            }
          }
    }
  }

  // rhs_unst_visc_diss (src/rhs_unst_visc_diss.F90:35-50).  diss(2:4) is zero
  // after rhs_convec_quick (src/rhs_convec_quick.F90:433).
  void unst_visc_diss(Level<R>& G, const std::vector<R>* visc) const {
    const int im = G.im, jm = G.jm, km = G.km;
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k);
          R dtaj = R(2) * R(c.delti) * G.aj[l];
          G.rh[0][l] = G.rh[0][l] + G.diss1[l];
          for (int m = 1; m < 4; ++m) {
            R dq = es * (R(3) * G.q[m][l] - R(4) * G.qn[m][l] + G.qnm1[m][l]) / dtaj;
            G.rh[m][l] = G.rh[m][l] + R(0) + dq - visc[m - 1][l];
          }
        }
  }

  // rhs_pk (src/rhs_pk.F90:35-67) over interior + one ring (the full level).
  void rhs_pk(Level<R>& G, int calc) const {
    for (int m = 0; m < 4; ++m)
      for (long l = 0; l < G.N; ++l) {
        if (calc) G.pk[m][l] = G.pk[m][l] - G.rh[m][l];
        G.rh[m][l] = G.rh[m][l] + G.pk[m][l];
      }
  }

  void zero_rh_boundary(Level<R>& G) const {
    const int im = G.im, jm = G.jm, km = G.km;
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i)
          if (i == 1 || i == im || j == 1 || j == jm || k == 1 || k == km)
            for (int m = 0; m < 4; ++m) G.rh[m][G.id(i, j, k)] = R(0);
  }

  // Residual assembly: rhs_contra_j .. rhs_pk .. boundary zeroing
  // (src/solver_daf.F90:199-306 for the first pass, :432-477 for the
  // recalculation, which keeps the first pass's diss(1) and dtau).
  void residual(Level<R>& G, int n, bool first_pass, int calc_pk) {
    auto t0 = std::chrono::steady_clock::now();
    std::vector<R> ucn[3], visc[3];
    for (int d = 0; d < 3; ++d) ucn[d].assign(G.N, R(0));
    contra_j(G, ucn);
    if (first_pass) daf_dtau(G);
    viscous(G, visc);
    if (first_pass) diss_p(G);
    flux_sans_convec(G, ucn);
    convec_quick(G, ucn, n == 0 ? 2 : 1);
    unst_visc_diss(G, visc);
    if (n > 0) rhs_pk(G, first_pass ? calc_pk : 0);
    zero_rh_boundary(G);
    phase_s[0] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // Characteristics outlet on the front face (btype(2) = 5), fine level,
  // after the interior residual and the boundary zeroing
  // (src/solver_daf.F90:318-358): mg_brhs (src/mg_brhs.F90:58-97) forms the
  // residual of the plane i = im from its eta and zeta derivatives alone --
  //   brhs_viscous          src/brhs_viscous.F90:40-160
  //   brhs_diss_p           src/brhs_diss_p.F90:33-89
  //   brhs_flux_sans_convec src/brhs_flux_sans_convec.F90:45-86
  //   brhs_convec_quick(2)  src/brhs_convec_quick.F90:41-205
  //   brhs_unst_visc_diss   src/brhs_unst_visc_diss.F90:30-44
  // -- then nonreflect_ibc (src/nonreflect_ibc.F90:86-242) adds the LODI
  // csi terms from the one-sided difference q(im) - q(im-1).  Interior j, k
  // of the plane only; the plane's edges keep rh = 0.  The back face's call
  // (inout = 1) writes the plane i = 1, which no later step reads (the solve
  // starts at i_mysta and the recalculation zeroes it), so it is not made.
  // nu_t enters the viscous coefficient as in the interior (rei + nu_t; zero
  // for laminar cases).
  void outlet_rhs(Level<R>& G) const {
    const int im = G.im, jm = G.jm, km = G.km, I = im;
    auto P = [&](int j, int k) { return G.id(I, j, k); };
    auto pl = [&](int j, int k) { return (long)(j - 1) + (long)jm * (k - 1); };
    const long NP = (long)jm * km;
    const R rei = R(1) / R(c.ren), one_fourth = R(0.25);
    const R de = G.de, dz = G.dz, de4 = R(0.25) * de, dz4 = R(0.25) * dz;
    const R de2 = R(0.5) * de, dz2 = R(0.5) * dz;
    const std::vector<R>* Q = G.q;
    auto ret = [&](long l) { return rei + G.nut[l]; };
    std::vector<R> ucn[3];
    for (int d = 0; d < 3; ++d) ucn[d].assign(G.N, R(0));
    contra_j(G, ucn);
    // ---- brhs_viscous: visc(1:3) on the plane
    std::vector<R> visc[3], fv[3];
    for (int m = 0; m < 3; ++m) { visc[m].assign(NP, R(0)); fv[m].assign(NP, R(0)); }
    auto face = [&](long l0, long l1, R ue, R ve, R we, R uz, R vz, R wz, bool eta_face, R* out) {
      R b1 = G.eta[0][l1] + G.eta[0][l0], b2 = G.eta[1][l1] + G.eta[1][l0], b3 = G.eta[2][l1] + G.eta[2][l0];
      R c1 = G.zet[0][l1] + G.zet[0][l0], c2 = G.zet[1][l1] + G.zet[1][l0], c3 = G.zet[2][l1] + G.zet[2][l0];
      R uu1 = b1 * ue + c1 * uz, vv1 = b1 * ve + c1 * vz, ww1 = b1 * we + c1 * wz;
      R uu2 = b2 * ue + c2 * uz, vv2 = b2 * ve + c2 * vz, ww2 = b2 * we + c2 * wz;
      R uu3 = b3 * ue + c3 * uz, vv3 = b3 * ve + c3 * vz, ww3 = b3 * we + c3 * wz;
      R vtj = one_fourth * (ret(l1) + ret(l0)) / (G.aj[l1] + G.aj[l0]);
      if (eta_face) {
        R c22 = b1 * b1 + b2 * b2 + b3 * b3, c23 = b1 * c1 + b2 * c2 + b3 * c3;
        out[0] = vtj * (b1 * uu1 + b2 * vv1 + b3 * ww1 + c22 * ue + c23 * uz);
        out[1] = vtj * (b1 * uu2 + b2 * vv2 + b3 * ww2 + c22 * ve + c23 * vz);
        out[2] = vtj * (b1 * uu3 + b2 * vv3 + b3 * ww3 + c22 * we + c23 * wz);
      } else {
        R c32 = c1 * b1 + c2 * b2 + c3 * b3, c33 = c1 * c1 + c2 * c2 + c3 * c3;
        out[0] = vtj * (c1 * uu1 + c2 * vv1 + c3 * ww1 + c32 * ue + c33 * uz);
        out[1] = vtj * (c1 * uu2 + c2 * vv2 + c3 * ww2 + c32 * ve + c33 * vz);
        out[2] = vtj * (c1 * uu3 + c2 * vv3 + c3 * ww3 + c32 * we + c33 * wz);
      }
    };
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 1; j <= jm - 1; ++j) {
        long l0 = P(j, k), l1 = P(j + 1, k);
        R d[3], z[3], o[3];
        for (int m = 0; m < 3; ++m) {
          const std::vector<R>& v = Q[m + 1];
          d[m] = de * (v[l1] - v[l0]);
          z[m] = dz4 * (v[P(j + 1, k + 1)] - v[P(j + 1, k - 1)] + v[P(j, k + 1)] - v[P(j, k - 1)]);
        }
        face(l0, l1, d[0], d[1], d[2], z[0], z[1], z[2], true, o);
        for (int m = 0; m < 3; ++m) fv[m][pl(j, k)] = o[m];
      }
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int m = 0; m < 3; ++m) visc[m][pl(j, k)] = de * (fv[m][pl(j, k)] - fv[m][pl(j - 1, k)]);
    for (int k = 1; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j) {
        long l0 = P(j, k), l1 = P(j, k + 1);
        R e[3], z[3], o[3];
        for (int m = 0; m < 3; ++m) {
          const std::vector<R>& v = Q[m + 1];
          e[m] = de4 * (v[P(j + 1, k + 1)] - v[P(j - 1, k + 1)] + v[P(j + 1, k)] - v[P(j - 1, k)]);
          z[m] = dz * (v[l1] - v[l0]);
        }
        face(l0, l1, e[0], e[1], e[2], z[0], z[1], z[2], false, o);
        for (int m = 0; m < 3; ++m) fv[m][pl(j, k)] = o[m];
      }
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int m = 0; m < 3; ++m)
          visc[m][pl(j, k)] = visc[m][pl(j, k)] + dz * (fv[m][pl(j, k)] - fv[m][pl(j, k - 1)]);
    // ---- brhs_diss_p: diss(1) on the plane
    std::vector<R> aux1(NP, R(0)), aux2(NP, R(0)), diss1(NP, R(0));
    const std::vector<R>& p = Q[0];
    const R desq = de * de, dzsq = dz * dz;
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j) {
        long l = P(j, k);
        R g2 = G.eta[0][l] * G.eta[0][l] + G.eta[1][l] * G.eta[1][l] + G.eta[2][l] * G.eta[2][l];
        aux1[pl(j, k)] = (g2 * G.dtau[l] / G.aj[l]) * (desq * (p[P(j + 1, k)] - R(2) * p[l] + p[P(j - 1, k)]));
        R g3 = G.zet[0][l] * G.zet[0][l] + G.zet[1][l] * G.zet[1][l] + G.zet[2][l] * G.zet[2][l];
        aux2[pl(j, k)] = (g3 * G.dtau[l] / G.aj[l]) * (dzsq * (p[P(j, k + 1)] - R(2) * p[l] + p[P(j, k - 1)]));
      }
    for (int k = 1; k <= km; ++k) { aux1[pl(1, k)] = aux1[pl(2, k)]; aux1[pl(jm, k)] = aux1[pl(jm - 1, k)]; }
    for (int j = 1; j <= jm; ++j) { aux2[pl(j, 1)] = aux2[pl(j, 2)]; aux2[pl(j, km)] = aux2[pl(j, km - 1)]; }
    const R pd = R(c.pdiss_coef);
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        diss1[pl(j, k)] = pd * ((aux1[pl(j + 1, k)] - R(2) * aux1[pl(j, k)] + aux1[pl(j - 1, k)]) +
                                (aux2[pl(j, k + 1)] - R(2) * aux2[pl(j, k)] + aux2[pl(j, k - 1)]));
    // ---- brhs_flux_sans_convec, brhs_convec_quick(2), brhs_unst_visc_diss
    const R coef = R(0.125);
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j) {
        long l = P(j, k), jp = P(j + 1, k), jn = P(j - 1, k), kp = P(j, k + 1), kn = P(j, k - 1);
        R r[4];
        for (int d = 0; d < 3; ++d) {
          R v = de2 * (p[jp] / G.aj[jp] * G.eta[d][jp] - p[jn] / G.aj[jn] * G.eta[d][jn]);
          r[d + 1] = v + dz2 * (p[kp] / G.aj[kp] * G.zet[d][kp] - p[kn] / G.aj[kn] * G.zet[d][kn]);
        }
        r[0] = R(0) + de2 * (ucn[1][jp] - ucn[1][jn]) + dz2 * (ucn[2][kp] - ucn[2][kn]);
        const int pos[2] = {j, k}, ext[2] = {jm, km};
        const long st[2] = {(long)im, (long)im * jm};
        const R h[2] = {de, dz};
        for (int d = 0; d < 2; ++d) {
          R ucon = R(0.5) * ucn[d + 1][l];
          R up = ucon + std::fabs(ucon), um = ucon - std::fabs(ucon);
          bool first = pos[d] == 2 || pos[d] == ext[d] - 1;
          const long s = st[d];
          for (int m = 0; m < 3; ++m) {
            const std::vector<R>& v = Q[m + 1];
            R f;
            if (first) f = h[d] * (up * (v[l] - v[l - s]) + um * (v[l + s] - v[l]));
            else
              f = coef * h[d] * (up * (R(3) * v[l + s] + R(3) * v[l] - R(7) * v[l - s] + v[l - 2 * s]) +
                                 um * (-R(3) * v[l - s] - R(3) * v[l] + R(7) * v[l + s] - v[l + 2 * s]));
            r[m + 1] = r[m + 1] + f;
          }
        }
        R dtaj = R(2) * R(c.delti) * G.aj[l];
        r[0] = r[0] + diss1[pl(j, k)];
        for (int m = 1; m < 4; ++m) {
          R dq = es * (R(3) * Q[m][l] - R(4) * G.qn[m][l] + G.qnm1[m][l]) / dtaj;
          r[m] = r[m] + R(0) + dq - visc[m - 1][pl(j, k)];
        }
        // ---- nonreflect_ibc, inout = 2: L_max of the general LODI vector
        R u = Q[1][l], v = Q[2][l], w = Q[3][l];
        R ucon = ucn[0][l] * G.aj[l];
        R c1 = G.csi[0][l], c2 = G.csi[1][l], c3 = G.csi[2][l];
        R gjj = c1 * c1 + c2 * c2 + c3 * c3;
        R sg = std::sqrt(gjj);
        R cj = std::sqrt(ucon * ucon + gjj);
        long lw = G.id(I - 1, j, k);
        R dq[4];
        for (int m = 0; m < 4; ++m) dq[m] = Q[m][l] - Q[m][lw];
        R lam1 = ucon - cj, lam2 = ucon + cj, lam3 = ucon, lam4 = ucon;
        R kj = c1 + c2 + c3;
        R d1 = (c2 - c1 + lam1 * (v - u)) / kj, d2 = (c2 - c1 + lam2 * (v - u)) / kj;
        R d3 = (c3 - c1 + lam1 * (w - u)) / kj, d4 = (c3 - c1 + lam2 * (w - u)) / kj;
        R d5 = (c2 - c1 + lam3 * (v - u)) / kj * R(2), d6 = (c3 - c1 + lam4 * (w - u)) / kj * R(2);
        R cc = R(2) * cj * cj / kj;
        R si[4][4] = {{-lam2, c1, c2, c3},
                      {-lam1, c1, c2, c3},
                      {lam2 * d1 + lam1 * d2, -cc - c1 * d5, cc - c2 * d5, -c3 * d5},
                      {lam2 * d3 + lam1 * d4, -cc - c1 * d6, -c2 * d6, cc - c3 * d6}};
        R den = R(2) * cj * cj;
        R lg[4];
        for (int a = 0; a < 4; ++a) {
          R s = R(0);
          for (int b = 0; b < 4; ++b) s = s + si[a][b] * sg / den * dq[b];
          lg[a] = s;
        }
        lg[0] = lam1 * lg[0]; lg[1] = lam2 * lg[1]; lg[2] = lam3 * lg[2]; lg[3] = lam4 * lg[3];
        R L1 = 0, L2 = lg[1], L3 = 0, L4 = 0;
        if (!(ucon < R(0))) { L3 = lg[2]; L4 = lg[3]; }
        R rh1 = (-cj * L1 + cj * L2) / sg;
        R rh2 = ((c1 + u * lam1) * L1 + (c1 + u * lam2) * L2 - c2 * L3 - c3 * L4) / sg;
        R rh3 = ((c2 + v * lam1) * L1 + (c2 + v * lam2) * L2 + (c1 + c3) * L3 - c3 * L4) / sg;
        R rh4 = ((c3 + w * lam1) * L1 + (c3 + w * lam2) * L2 - c2 * L3 + (c1 + c2) * L4) / sg;
        G.rh[0][l] = r[0] + rh1 / G.aj[l];
        G.rh[1][l] = r[1] + rh2 / G.aj[l];
        G.rh[2][l] = r[2] + rh3 / G.aj[l];
        G.rh[3][l] = r[3] + rh4 / G.aj[l];
      }
  }

  // ----------------------------------------------------------- DAF solve
  // Modal quantities of one node (src/rhs_modal_matrices.F90:50-268); each
  // stage of the diagonal solver builds the matrix it needs.
  inline void sigma_theta(const Level<R>& G, long l, R& sigma, R& theta) const {
    const R beta = R(c.beta);
    R alpha = R(1) + es * R(1.5) * G.dtau[l] / R(c.delti);
    sigma = std::sqrt(beta * alpha);
    theta = std::sqrt(beta / alpha);
  }
  M4<R> mat_mai(const Level<R>& G, long l) const {
    R s, t; sigma_theta(G, l, s, t);
    M4<R> a, ai; modal_pair(G.csi[0][l], G.csi[1][l], G.csi[2][l], s, a, ai);
    return ai;
  }
  M4<R> mat_n1i(const Level<R>& G, long l) const {  // Mb^-1 Ma
    R s, t; sigma_theta(G, l, s, t);
    M4<R> ma, mai, mb, mbi;
    modal_pair(G.csi[0][l], G.csi[1][l], G.csi[2][l], s, ma, mai);
    modal_pair(G.eta[0][l], G.eta[1][l], G.eta[2][l], s, mb, mbi);
    return mm4(mbi, ma);
  }
  M4<R> mat_n2i(const Level<R>& G, long l) const {  // Mc^-1 Mb
    R s, t; sigma_theta(G, l, s, t);
    M4<R> mb, mbi, mc, mci;
    modal_pair(G.eta[0][l], G.eta[1][l], G.eta[2][l], s, mb, mbi);
    modal_pair(G.zet[0][l], G.zet[1][l], G.zet[2][l], s, mc, mci);
    return mm4(mci, mb);
  }
  M4<R> mat_mc(const Level<R>& G, long l) const {
    R s, t; sigma_theta(G, l, s, t);
    M4<R> mc, mci; modal_pair(G.zet[0][l], G.zet[1][l], G.zet[2][l], s, mc, mci);
    return mc;
  }
  void spectral_radii(const Level<R>& G, std::vector<R>* spr) const {
    for (int d = 0; d < 3; ++d) spr[d].assign(G.N, R(0));
    ORC_PARFOR
    for (long l = 0; l < G.N; ++l) {
      R s, t; sigma_theta(G, l, s, t);
      R c1 = G.csi[0][l], c2 = G.csi[1][l], c3 = G.csi[2][l];
      R e1 = G.eta[0][l], e2 = G.eta[1][l], e3 = G.eta[2][l];
      R z1 = G.zet[0][l], z2 = G.zet[1][l], z3 = G.zet[2][l];
      spr[0][l] = t * std::sqrt(c1 * c1 + c2 * c2 + c3 * c3);
      spr[1][l] = t * std::sqrt(e1 * e1 + e2 * e2 + e3 * e3);
      spr[2][l] = t * std::sqrt(z1 * z1 + z2 * z2 + z3 * z3);
    }
  }

  // rhs_diag_solver (src/rhs_diag_solver.F90:44-633).  On entry rh holds the
  // residual; on exit the update dq on interior nodes.
  void diag_solver(Level<R>& G, int n) {
    auto t0 = std::chrono::steady_clock::now();
    const int im = G.im, jm = G.jm, km = G.km;
    const R beta = R(c.beta);
    const R dh[3] = {R(0.5) * G.dc, R(0.5) * G.de, R(0.5) * G.dz};
    const R dsq[3] = {G.dc * G.dc, G.de * G.de, G.dz * G.dz};
    const R lam[4] = {0, 0, 1, -1};
    const bool fine = (n == 0);
    std::vector<R> spr[3];
    spectral_radii(G, spr);
    // r <- S * (-dtau * rh * J) (src/rhs_diag_solver.F90:53-72)
    const R alpha_mult = es * R(1.5) / R(c.delti);
    // idend (src/solver_daf.F90:371-373): the fine level's characteristics
    // outlet plane i = im is solved with the interior
    const int ie = (n == 0 && c.btype[1] == 5) ? im : im - 1;
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= ie; ++i) {
          long l = G.id(i, j, k);
          R alpha = R(1) + alpha_mult * G.dtau[l];
          R s[4] = {beta, R(1) / alpha, R(1) / alpha, R(1) / alpha};
          for (int m = 0; m < 4; ++m) G.rh[m][l] = s[m] * (-G.dtau[l] * G.rh[m][l] * G.aj[l]);
        }
    // one line of one direction: ids = interior node ids along the line,
    // lprev / lnext = the boundary nodes before and after it; bw / be = the
    // semi-explicit boundary vectors (brh) or null.  Scratch is per call, so
    // lines may be solved concurrently.
    // With outrow the last node is the characteristics outlet node i = im
    // and its row is (src/rhs_diag_solver.F90:207-221): ap = 1, 1,
    // 1 + dtau dc spr, 1; aw = 0, 0, -dtau(im-1) dc spr(im-1), 0.
    auto sweep_line = [&](int dir, const std::vector<long>& ids, long lprev, long lnext, const R* bw, const R* be,
                          bool outrow = false) {
      int len = (int)ids.size();
      std::vector<R> aw(len, 0), ap(len, 0), ae(len, 0), aq(len, 0), dl, du;
      long piv = 0;
      const R epd = R(c.ep[0][dir]);
      for (int m = 0; m < 4; ++m) {
        for (int p = 0; p < len; ++p) {
          long l = ids[p];
          long lw = p == 0 ? lprev : ids[p - 1];
          long le = p == len - 1 ? lnext : ids[p + 1];
          R dtc = R(1);
          if (G.dtau[l] == R(0)) dtc = R(0);
          R tmp = G.dtau[l] * epd * spr[dir][l] * dsq[dir];
          ap[p] = R(1) + R(2) * tmp;
          R ddsw = dtc * G.dtau[lw] * dh[dir] * spr[dir][lw];
          R ddse = dtc * G.dtau[le] * dh[dir] * spr[dir][le];
          aw[p] = (m < 2) ? -tmp : (-ddsw * lam[m] - tmp);
          ae[p] = (m < 2) ? -tmp : (ddse * lam[m] - tmp);
          aq[p] = G.rh[m][l];
        }
        if (outrow) {
          const int p = len - 1;
          const long l = ids[p], lw = ids[p - 1];
          R dds = G.dtau[l] * G.dc * spr[0][l];
          ap[p] = m == 2 ? R(1) + dds * lam[2] : R(1);
          R ddw = G.dtau[lw] * G.dc * spr[0][lw];
          aw[p] = m == 2 ? -ddw * lam[2] : R(0);
        }
        if (bw) aq[0] = aq[0] - aw[0] * bw[m];
        if (be) aq[len - 1] = aq[len - 1] - ae[len - 1] * be[m];
        dl.assign(aw.begin() + 1, aw.end());
        du.assign(ae.begin(), ae.end() - 1);
        gtsv(len, 1, dl.data(), ap.data(), du.data(), aq.data(), len, &piv);
        for (int p = 0; p < len; ++p) G.rh[m][ids[p]] = aq[p];
      }
      if (piv) {
#ifdef _OPENMP
#pragma omp atomic
#endif
        pivots += piv;
      }
    };
    auto sabc = [&](int b, const R* r1, const R* r2, R* out) {
      for (int m = 0; m < 4; ++m) out[m] = sa[m][b] * r1[m] + sb[m][b] * r2[m];
    };
    auto getr = [&](long l, R* r) { for (int m = 0; m < 4; ++m) r[m] = G.rh[m][l]; };
    auto putr = [&](long l, const R* r) { for (int m = 0; m < 4; ++m) G.rh[m][l] = r[m]; };
    auto xform = [&](long l, const M4<R>& A) { R r[4], rp[4]; getr(l, r); mv4(A, r, rp); putr(l, rp); };
    auto xvec = [&](R* b, const M4<R>& A) { R rp[4]; mv4(A, b, rp); for (int m = 0; m < 4; ++m) b[m] = rp[m]; };
    // ---- csi sweep (src/rhs_diag_solver.F90:79-258).  The front face's brh
    // is never set on one rank (the guard at :102 reads myfront /=
    // mpi_proc_null), so only the back face contributes.
    {
      std::vector<R> brh((long)4 * jm * km, R(0));
      bool bback = fine && c.btype[0] != 5;
      auto bo = [&](int j, int k) { return (long)4 * ((j - 1) + (long)jm * (k - 1)); };
      if (bback)
        for (int k = 2; k <= km - 1; ++k)
          for (int j = 2; j <= jm - 1; ++j) {
            R r1[4], r2[4];
            getr(G.id(2, j, k), r1); getr(G.id(3, j, k), r2);
            sabc(0, r1, r2, &brh[bo(j, k)]);
          }
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= ie; ++i) { long l = G.id(i, j, k); xform(l, mat_mai(G, l)); }
      if (bback)
        for (int k = 2; k <= km - 1; ++k)
          for (int j = 2; j <= jm - 1; ++j) xvec(&brh[bo(j, k)], mat_mai(G, G.id(1, j, k)));
ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j) {
          std::vector<long> ids(ie - 1);
          for (int i = 2; i <= ie; ++i) ids[i - 2] = G.id(i, j, k);
          sweep_line(0, ids, G.id(1, j, k), G.id(im, j, k), bback ? &brh[bo(j, k)] : nullptr, nullptr, ie == im);
        }
    }
    // ---- eta sweep (src/rhs_diag_solver.F90:265-434)
    {
      std::vector<R> b1((long)4 * im * km, R(0)), b2((long)4 * im * km, R(0));
      bool bl = fine && c.btype[2] != 5, br = fine && c.btype[3] != 5;
      auto bo = [&](int i, int k) { return (long)4 * ((i - 1) + (long)im * (k - 1)); };
      for (int k = 2; k <= km - 1; ++k)
        for (int i = 2; i <= ie; ++i) {
          R r1[4], r2[4];
          if (bl) { getr(G.id(i, 2, k), r1); getr(G.id(i, 3, k), r2); sabc(2, r1, r2, &b1[bo(i, k)]); }
          if (br) { getr(G.id(i, jm - 1, k), r1); getr(G.id(i, jm - 2, k), r2); sabc(3, r1, r2, &b2[bo(i, k)]); }
        }
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= ie; ++i) { long l = G.id(i, j, k); xform(l, mat_n1i(G, l)); }
      for (int k = 2; k <= km - 1; ++k)
        for (int i = 2; i <= ie; ++i) {
          if (bl) xvec(&b1[bo(i, k)], mat_n1i(G, G.id(i, 1, k)));
          if (br) xvec(&b2[bo(i, k)], mat_n1i(G, G.id(i, jm, k)));
        }
ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int i = 2; i <= ie; ++i) {
          std::vector<long> ids(jm - 2);
          for (int j = 2; j <= jm - 1; ++j) ids[j - 2] = G.id(i, j, k);
          sweep_line(1, ids, G.id(i, 1, k), G.id(i, jm, k), bl ? &b1[bo(i, k)] : nullptr, br ? &b2[bo(i, k)] : nullptr);
        }
    }
    // ---- zeta sweep (src/rhs_diag_solver.F90:441-612).  The up face is set
    // up only if btype(6) /= 6 (:467) and used only if btype(6) /= 5
    // (:504, :571).
    {
      std::vector<R> b1((long)4 * im * jm, R(0)), b2((long)4 * im * jm, R(0));
      bool bd = fine && c.btype[4] != 5;
      bool bu_set = fine && c.btype[5] != 6, bu_use = fine && c.btype[5] != 5;
      auto bo = [&](int i, int j) { return (long)4 * ((i - 1) + (long)im * (j - 1)); };
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= ie; ++i) {
          R r1[4], r2[4];
          if (bd) { getr(G.id(i, j, 2), r1); getr(G.id(i, j, 3), r2); sabc(4, r1, r2, &b1[bo(i, j)]); }
          if (bu_set) { getr(G.id(i, j, km - 1), r1); getr(G.id(i, j, km - 2), r2); sabc(5, r1, r2, &b2[bo(i, j)]); }
        }
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= ie; ++i) { long l = G.id(i, j, k); xform(l, mat_n2i(G, l)); }
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= ie; ++i) {
          if (bd) xvec(&b1[bo(i, j)], mat_n2i(G, G.id(i, j, 1)));
          if (bu_use) xvec(&b2[bo(i, j)], mat_n2i(G, G.id(i, j, km)));
        }
ORC_PARFOR
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= ie; ++i) {
          std::vector<long> ids(km - 2);
          for (int k = 2; k <= km - 1; ++k) ids[k - 2] = G.id(i, j, k);
          sweep_line(2, ids, G.id(i, j, 1), G.id(i, j, km), bd ? &b1[bo(i, j)] : nullptr, bu_use ? &b2[bo(i, j)] : nullptr);
        }
    }
    // dq = Mc * r (src/rhs_diag_solver.F90:624-633)
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= ie; ++i) { long l = G.id(i, j, k); xform(l, mat_mc(G, l)); }
    phase_s[1] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // bcond_fm (src/bcond_fm.F90:60-322) on the fine level.  i_mysta = 1 and
  // i_myend = im here (boundary nodes included, :60-66).
  void bcond_fm() {
    auto t0 = std::chrono::steady_clock::now();
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    auto Q = [&](int m, int i, int j, int k) -> R& { return G.q[m][G.id(i, j, k)]; };
    // i faces
    for (int side = 0; side < 2; ++side) {
      int b = side, i = side == 0 ? 1 : im, s = side == 0 ? 1 : -1;
      int bt = c.btype[b];
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
          if (bt >= 1 && bt <= 3) {
            for (int m = 0; m < 4; ++m) Q(m, i, j, k) = sa[m][b] * Q(m, i + s, j, k) + sb[m][b] * Q(m, i + 2 * s, j, k);
          } else if (bt == 4) {
            R r = ratv(b, j, k);
            Q(0, i, j, k) = (R(1) + r) * Q(0, i + s, j, k) - r * Q(0, i + 2 * s, j, k);
          } else if (bt == 8 && side == 1) {
            for (int m = 0; m < 4; ++m) Q(m, i, j, k) = Q(m, i - 1, j, k);
          }
          // btype 6 in i: commented out in the reference (:105-110, :153-158)
        }
    }
    // j faces
    for (int side = 0; side < 2; ++side) {
      int b = 2 + side, j = side == 0 ? 1 : jm, s = side == 0 ? 1 : -1;
      int bt = c.btype[b];
      for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) {
          if (bt >= 1 && bt <= 3) {
            for (int m = 0; m < 4; ++m) Q(m, i, j, k) = sa[m][b] * Q(m, i, j + s, k) + sb[m][b] * Q(m, i, j + 2 * s, k);
          } else if (bt == 4) {
            R r = ratv(b, i, k);
            Q(0, i, j, k) = (R(1) + r) * Q(0, i, j + s, k) - r * Q(0, i, j + 2 * s, k);
          } else if (bt == 6) {
            int jo = side == 0 ? jm : 1;  // j_myend / j_mysta are the boundary nodes here
            for (int m = 0; m < 4; ++m) Q(m, i, j, k) = Q(m, i, jo, k);
          }
        }
    }
    // k faces
    for (int side = 0; side < 2; ++side) {
      int b = 4 + side, k = side == 0 ? 1 : km, s = side == 0 ? 1 : -1;
      int bt = c.btype[b];
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          if (bt >= 1 && bt <= 3) {
            for (int m = 0; m < 4; ++m) Q(m, i, j, k) = sa[m][b] * Q(m, i, j, k + s) + sb[m][b] * Q(m, i, j, k + 2 * s);
          } else if (bt == 4) {
            R r = ratv(b, i, j);
            Q(0, i, j, k) = (R(1) + r) * Q(0, i, j, k + s) - r * Q(0, i, j, k + 2 * s);
          } else if (bt == 6) {
            int ko = side == 0 ? km : 1;
            for (int m = 0; m < 4; ++m) Q(m, i, j, k) = Q(m, i, j, ko);
          }
        }
    }
    // pressure fix over the full range (:310-322)
    R pfix = Q(0, c.ifix, c.jfix, c.kfix);
    for (long l = 0; l < G.N; ++l) G.q[0][l] = G.q[0][l] - pfix;
    phase_s[2] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // ------------------------------------------------- actuator-line forcing
  // Airfoil polar lookup of src/rhs_lines.F90:241-281: a linear scan for the
  // interval [angle1, angle2] holding AOA, stopping unassigned when AOA is at
  // or below an interval's start or the end marker (-999) is reached; an
  // unassigned lookup leaves the caller's previous values.
  bool polar_lookup(int p, R aoa, R& cl, R& cd) const {
    const R* rows = polar_rows.data() + 3 * polar_off[p];
    int idx = 0, counter = 1;
    R angle1 = 1000, angle2 = 1000, cl1 = 0, cd1 = 0, cl2 = 0, cd2 = 0;
    while (angle2 != R(-999)) {
      if (counter == 1) { angle1 = rows[3 * idx]; cl1 = rows[3 * idx + 1]; cd1 = rows[3 * idx + 2]; ++idx; }
      else { angle1 = angle2; cl1 = cl2; cd1 = cd2; }
      angle2 = rows[3 * idx]; cl2 = rows[3 * idx + 1]; cd2 = rows[3 * idx + 2]; ++idx;
      if (aoa <= angle1) {
        angle2 = R(-999);
      } else if (angle2 == R(-999)) {
      } else if (aoa <= angle2 && aoa >= angle1) {
        R m = (cl2 - cl1) / (angle2 - angle1);
        cl = m * (aoa - angle1) + cl1;
        m = (cd2 - cd1) / (angle2 - angle1);
        cd = m * (aoa - angle1) + cd1;
        return true;
      } else {
        ++counter;
      }
    }
    return false;
  }

  // rhs_lines (src/rhs_lines.F90:47-483) on the fine level: element forces
  // from the interpolated velocity and the polars, then their Gaussian
  // projection onto each turbine's kernel nodes, added to rh(2:4).
  void rhs_lines(Level<R>& G) {
    const R pi = R(3.141592653589793);  // src/precision.F90:43
    const R rho = R(1178.62);
    const R ls = alm_length_scale;
    const R vel_scale = R(c.ren) * R(10E-7) / ls;
    for (int d = 0; d < 3; ++d) falm[d].assign(G.N, R(0));
    size_t nel = 0;
    for (auto& T : alm) nel += size_t(T.nblades) * T.nelems;
    forces_lines.assign(6 * nel, R(0));
    // the lookups' outputs persist from element to element within a call
    R cl_b = 0, cd_b = 0, cl_a = 0, cd_a = 0;
    size_t base = 0;
    for (auto& T : alm) {
      const R omega = (alm_vel_infty * T.tsr) / T.tur_rad;
      const R dth = R(2) * pi / R(T.nangles);
      for (int bld = 1; bld <= T.nblades; ++bld) {
        R angle_aux = T.angle + R(bld - 1) * R(2) * pi / R(T.nblades);
        if (angle_aux > R(2) * pi) angle_aux = angle_aux - R(2) * pi;
        int nang = int(std::lround(double(angle_aux / dth))) + 1;
        if (nang > T.nangles) nang -= T.nangles;  // the reference reads one bin past its table here
        for (int elem = 1; elem <= T.nelems; ++elem) {
          const long e = long(nang - 1) * T.nelems + (elem - 1);
          const int i = T.node_index[3 * e], j = T.node_index[3 * e + 1], k = T.node_index[3 * e + 2];
          // only cells whose lower corner is in the rank's interior (src/rhs_lines.F90:166-167)
          if (i < 2 || i > G.im - 1 || j < 2 || j > G.jm - 1 || k < 2 || k > G.km - 1) continue;
          const R* P = T.node_pos.data() + 27 * e;
          // node_indexes_pos(...,1:27): xf, yf, zf, then corners 000 100 110 010 001 101 111 011
          const R xf = P[0], yf = P[1], zf = P[2];
          const R x000 = P[3], z000 = P[5], x100 = P[6], y100 = P[7], y110 = P[10];
          const R x001 = P[15], z001 = P[17], x101 = P[18], y101 = P[19], y111 = P[22];
          const long jk = (long)(j - 1) + (long)G.jm * (k - 1);
          const R* D = T.disk_dat.data() + 8 * jk;
          const R radius = D[0] * ls, chord = D[4], twist = D[5], inter = D[6];
          auto q = [&](int m, int ii, int jj, int kk) { return G.q[m][G.id(ii, jj, kk)]; };
          R v[3];
          for (int m = 1; m <= 3; ++m) {  // src/rhs_lines.F90:192-214
            const R down = R(1) / ((x100 - x000) * (y110 - y100)) *
                           ((x100 - xf) * ((y110 - yf) * (q(m, i, j, k) + q(m, i, j + 1, k))) +
                            (xf - x000) * ((yf - y100) * (q(m, i + 1, j, k) + q(m, i + 1, j + 1, k))));
            const R up = R(1) / ((x101 - x001) * (y111 - y101)) *
                         ((x101 - xf) * ((y111 - yf) * (q(m, i, j, k + 1) + q(m, i, j + 1, k + 1))) +
                          (xf - x001) * ((yf - y101) * (q(m, i + 1, j, k + 1) + q(m, i + 1, j + 1, k + 1))));
            v[m - 1] = down + (up - down) / (z001 - z000) * (zf - z000);
          }
          const R u_x = v[0] * vel_scale, u_y = v[1] * vel_scale, u_z = v[2] * vel_scale;
          const R u_theta = omega * radius + u_y * std::sin(angle_aux) - u_z * std::cos(angle_aux);
          const R phi = std::atan2(u_x, u_theta);
          const R aoa = phi * R(180.0) / pi - twist;
          polar_lookup(T.polar_b[jk], aoa, cl_b, cd_b);
          polar_lookup(T.polar_a[jk], aoa, cl_a, cd_a);
          const R cl = (cl_a - cl_b) * inter + cl_b;
          const R cd = (cd_a - cd_b) * inter + cd_b;
          const R urel = std::sqrt(u_theta * u_theta + u_x * u_x);
          const R fl = R(0.5) * cl * rho * (urel * urel) * chord;
          const R fd = R(0.5) * cd * rho * (urel * urel) * chord;
          R* F = forces_lines.data() + 6 * (base + size_t(bld - 1) * T.nelems + (elem - 1));
          F[0] = xf; F[1] = yf; F[2] = zf;
          F[3] = fl * std::cos(phi) + fd * std::sin(phi);
          F[4] = fl * std::sin(angle_aux) * std::sin(phi) - fd * std::sin(angle_aux) * std::sin(phi);
          F[5] = fl * std::cos(angle_aux) * std::sin(phi) - fd * std::cos(angle_aux) * std::cos(phi);
        }
      }
      // projection (src/rhs_lines.F90:382-448)
      const R deltar = std::abs(T.tur_rad - T.hub_rad) / R(T.nelems);
      const size_t ne = size_t(T.nblades) * T.nelems;
      for (int n = 0; n < T.nker; ++n) {
        const int* I = T.ker_index.data() + 3 * n;
        if (I[0] < 2 || I[0] > G.im - 1 || I[1] < 2 || I[1] > G.jm - 1 || I[2] < 2 || I[2] > G.km - 1) continue;
        const R radius = T.ker_dat[4 * n] * ls;
        const R dV = T.ker_dat[4 * n + 3] * (ls * ls * ls);
        if (!(radius > T.hub_rad)) continue;
        const R xk = T.ker_pos[3 * n], yk = T.ker_pos[3 * n + 1], zk = T.ker_pos[3 * n + 2];
        R fx = 0, fy = 0, fz = 0;
        for (size_t e = 0; e < ne; ++e) {
          const R* F = forces_lines.data() + 6 * (base + e);
          const R rdis =
              std::sqrt((xk - F[0]) * (xk - F[0]) + (yk - F[1]) * (yk - F[1]) + (zk - F[2]) * (zk - F[2])) * ls;
          const R eps = R(2) * std::pow(dV, R(1.0) / R(3.0));
          const R ker =
              R(1) / ((eps * eps * eps) * std::pow(pi, R(3.0) / R(2.0))) * std::exp(-(rdis * rdis) / (eps * eps));
          fx = fx + ker * F[3] * deltar;
          fy = fy + ker * F[4] * deltar;
          fz = fz + ker * F[5] * deltar;
        }
        const long l = G.id(T.ker_index[3 * n], T.ker_index[3 * n + 1], T.ker_index[3 * n + 2]);
        const R sc = (ls / (rho * vel_scale * vel_scale)) * (R(1) / G.aj[l]);
        const R d[3] = {fx * sc, fy * sc, fz * sc};
        for (int m = 0; m < 3; ++m) {
          G.rh[m + 1][l] = G.rh[m + 1][l] + d[m];
          falm[m][l] = falm[m][l] + d[m];
        }
      }
      base += ne;
    }
  }

  // solver_daf (src/solver_daf.F90:138-488) on level index n (0 = fine).
  void solver_daf(int n, int recalc, int itr) {
    Level<R>& G = L[n];
    const int im = G.im, jm = G.jm, km = G.km;
    for (int m = 0; m < 4; ++m) std::fill(G.rh[m].begin(), G.rh[m].end(), R(0));
    residual(G, n, true, itr == 1 ? 1 : 0);
    const bool outlet = n == 0 && c.btype[1] == 5;
    if (outlet) outlet_rhs(G);
    if (n == 0 && alm_on) rhs_lines(G);  // src/solver_daf.F90:378-381
    diag_solver(G, n);
    // q <- qold_af + rh up to idend (src/solver_daf.F90:409-418)
    const int ie = outlet ? im : im - 1;
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= ie; ++i) {
          long l = G.id(i, j, k);
          for (int m = 0; m < 4; ++m) G.q[m][l] = G.q[m][l] + G.rh[m][l];
        }
    if (n == 0) bcond_fm();
    if (recalc == 1) residual(G, n, false, 0);
  }

  // mg_nlevel (src/mg_nlevel.F90:19-146) followed by mg_zero_pk_boundary
  // (src/mg_driver.F90:134,407-466); n = coarse level index.
  void mg_nlevel(int n) {
    auto t0 = std::chrono::steady_clock::now();
    Level<R>& C = L[n]; Level<R>& F = L[n - 1];
    auto fid = [&](int i, int j, int k, int& ii, int& jj, int& kk) {
      kk = (1 << c.kcrs) * k - c.kcrs; jj = (1 << c.jcrs) * j - c.jcrs; ii = (1 << c.icrs) * i - c.icrs;
    };
    for (int k = 1; k <= C.km; ++k)
      for (int j = 1; j <= C.jm; ++j)
        for (int i = 1; i <= C.im; ++i) {
          int ii, jj, kk; fid(i, j, k, ii, jj, kk);
          long l = C.id(i, j, k), ll = F.id(ii, jj, kk);
          for (int m = 0; m < 4; ++m) C.q[m][l] = F.q[m][ll];
          C.nut[l] = F.nut[ll];
        }
    for (int m = 0; m < 4; ++m) C.qold[m] = C.q[m];
    const long ic = 1, ie = F.im, iz = (long)F.im * F.jm;
    const R p25 = R(0.25), p5 = R(0.5), two = R(2), s16 = R(1) / R(16);
    ORC_PARFOR
    for (int k = 1; k <= C.km; ++k)
      for (int j = 1; j <= C.jm; ++j)
        for (int i = 1; i <= C.im; ++i) {
          long l = C.id(i, j, k);
          bool bnd = i == 1 || i == C.im || j == 1 || j == C.jm || k == 1 || k == C.km;
          if (bnd) { for (int m = 0; m < 4; ++m) C.pk[m][l] = R(0); continue; }  // zeroed by mg_zero_pk_boundary
          int ii, jj, kk; fid(i, j, k, ii, jj, kk);
          long ll = F.id(ii, jj, kk);
          for (int m = 0; m < 4; ++m) {
            const std::vector<R>& r = F.rh[m];
            R s = p25 * r[ll + ic + ie + iz];
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
            C.pk[m][l] = s * s16;
          }
        }
    phase_s[3] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // mg_prolong (src/mg_prolong.F90:56-277) from level n+1 to level n, with
  // rsmooth/rs_sweep (src/rsmooth.F90:65-95, src/rs_sweep.F90:146-284).
  void mg_prolong(int n) {
    auto t0 = std::chrono::steady_clock::now();
    Level<R>& F = L[n]; Level<R>& C = L[n + 1];
    const int im = F.im, jm = F.jm, km = F.km;
    std::vector<R> dq[4];
    for (int m = 0; m < 4; ++m) dq[m].assign(F.N, R(0));
    ORC_PARFOR
    for (int k = 1; k <= C.km; ++k)
      for (int j = 1; j <= C.jm; ++j)
        for (int i = 1; i <= C.im; ++i) {
          int kk = (1 << c.kcrs) * k - c.kcrs, jj = (1 << c.jcrs) * j - c.jcrs, ii = (1 << c.icrs) * i - c.icrs;
          long ll = F.id(ii, jj, kk), l = C.id(i, j, k);
          for (int m = 0; m < 4; ++m) dq[m][ll] = C.q[m][l] - C.qold[m][l];
        }
    const R cp = R(0.5), cm = R(0.5);
    const long ie = im, iz = (long)im * jm;
    if (c.kcrs == 1)
ORC_PARFOR
      for (int k = 2; k <= km - 1; k += 2)
        for (int j = 1; j <= jm; j += (1 << c.jcrs))
          for (int i = 1; i <= im; i += (1 << c.icrs)) {
            long l = F.id(i, j, k);
            for (int m = 0; m < 4; ++m) dq[m][l] = cp * dq[m][l + iz] + cm * dq[m][l - iz];
          }
    if (c.jcrs == 1)
ORC_PARFOR
      for (int k = 1; k <= km; ++k)
        for (int j = 2; j <= jm - 1; j += 2)
          for (int i = 1; i <= im; i += (1 << c.icrs)) {
            long l = F.id(i, j, k);
            for (int m = 0; m < 4; ++m) dq[m][l] = cp * dq[m][l + ie] + cm * dq[m][l - ie];
          }
    if (c.icrs == 1)
ORC_PARFOR
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
          for (int i = 2; i <= im - 1; i += 2) {
            long l = F.id(i, j, k);
            for (int m = 0; m < 4; ++m) dq[m][l] = cp * dq[m][l + 1] + cm * dq[m][l - 1];
          }
    // implicit residual smoothing with ep(2, :) on interior lines
    const int ext[3] = {im, jm, km};
    for (int dir = 0; dir < 3; ++dir) {
      const R e = R(c.ep[1][dir]);
      int len = ext[dir] - 2;
      if (len <= 0) continue;
      int a1 = dir == 0 ? jm : im, a2 = dir == 2 ? jm : km;
ORC_PARFOR
      for (int q2 = 2; q2 <= a2 - 1; ++q2)
        for (int q1 = 2; q1 <= a1 - 1; ++q1) {
          std::vector<R> ax(len), bx(len), cx(len), dx((long)4 * len);
          std::vector<long> ids(len);
          for (int p = 0; p < len; ++p) {
            int t = p + 2;
            ids[p] = dir == 0 ? F.id(t, q1, q2) : (dir == 1 ? F.id(q1, t, q2) : F.id(q1, q2, t));
          }
          for (int p = 0; p < len; ++p) {
            ax[p] = -e; bx[p] = R(1) + R(2) * e; cx[p] = -e;
            for (int m = 0; m < 4; ++m) dx[(long)m * len + p] = dq[m][ids[p]];
          }
          std::vector<R> dl(ax.begin() + 1, ax.end()), du(cx.begin(), cx.end() - 1);
          gtsv(len, 4, dl.data(), bx.data(), du.data(), dx.data(), len, nullptr);
          for (int p = 0; p < len; ++p)
            for (int m = 0; m < 4; ++m) dq[m][ids[p]] = dx[(long)m * len + p];
        }
    }
    // dq = 0 on the domain boundary, then q += dq over the whole level
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i)
          if (i == 1 || i == im || j == 1 || j == jm || k == 1 || k == km)
            for (int m = 0; m < 4; ++m) dq[m][F.id(i, j, k)] = R(0);
    for (int m = 0; m < 4; ++m)
      for (long l = 0; l < F.N; ++l) F.q[m][l] = F.q[m][l] + dq[m][l];
    phase_s[3] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // mg_residual (src/mg_residual.F90:32-84): log10 of the mean |q - qold|.
  void mg_residual(int n, double* out) {
    auto t0 = std::chrono::steady_clock::now();
    Level<R>& G = L[n];
    R tnu = R((long)(G.im - 2) * (G.jm - 2) * (G.km - 2));
    R resd[5] = {0, 0, 0, 0, 0};
    for (int k = 2; k <= G.km - 1; ++k)
      for (int j = 2; j <= G.jm - 1; ++j)
        for (int i = 2; i <= G.im - 1; ++i) {
          long l = G.id(i, j, k);
          for (int m = 0; m < 5; ++m) resd[m] = resd[m] + std::fabs(G.q[m][l] - G.qold[m][l]);
        }
    for (int m = 0; m < 5; ++m) out[m] = (double)std::log10(resd[m] / tnu);
    phase_s[5] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // ------------------------------------------------------------- SA model
  // des_eddy (src/des_eddy.F90:109-297) on the fine level.
  void des_eddy() {
    auto t0 = std::chrono::steady_clock::now();
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    const R cb1 = R(0.1355), cb2 = R(0.622), sig = R(2.0) / R(3.0), capa = R(0.41);
    const R cw1 = R(3.23906782), cw2 = R(0.3), cw3h = R(64.0), cv1c = R(357.911), cv2 = R(5.0);
    const R rei = R(1) / R(c.ren);
    const R one = 1, two = 2, pt5 = R(0.5), zero = 0;
    const R dc = G.dc, de = G.de, dz = G.dz;
    const R dc2 = pt5 * dc, de2 = pt5 * de, dz2 = pt5 * dz;
    const R dc4 = R(0.25) * dc, de4 = R(0.25) * de, dz4 = R(0.25) * dz;
    std::vector<R>& q5 = G.q[4];
    std::vector<R> qold(q5), ucn[3], wo(G.N, R(0)), dnu(G.N, R(0)), psa(G.N, R(0)), visc(G.N, R(0)), rh(G.N, R(0)), fv(G.N, R(0));
    for (int d = 0; d < 3; ++d) ucn[d].assign(G.N, R(0));
    contra_j(G, ucn);
    auto id = [&](int i, int j, int k) { return G.id(i, j, k); };
    // rhs_sa_source (src/rhs_sa_source.F90:35-95): interior only
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = id(i, j, k);
          R g[3][3];  // g[var][dir]
          for (int m = 0; m < 3; ++m) {
            const std::vector<R>& v = G.q[m + 1];
            g[m][0] = dc2 * (v[id(i + 1, j, k)] - v[id(i - 1, j, k)]);
            g[m][1] = de2 * (v[id(i, j + 1, k)] - v[id(i, j - 1, k)]);
            g[m][2] = dz2 * (v[id(i, j, k + 1)] - v[id(i, j, k - 1)]);
          }
          R d[3][3];  // d[var][x]
          for (int m = 0; m < 3; ++m)
            for (int x = 0; x < 3; ++x) d[m][x] = g[m][0] * G.csi[x][l] + g[m][1] * G.eta[x][l] + g[m][2] * G.zet[x][l];
          R w12 = pt5 * (d[0][1] - d[1][0]);
          R w13 = pt5 * (d[0][2] - d[2][0]);
          R w23 = pt5 * (d[1][2] - d[2][1]);
          wo[l] = two * (w12 * w12 + w13 * w13 + w23 * w23);
        }
    for (int iterk = 1; iterk <= c.itk; ++iterk) {
      // rhs_sa_grdnu (src/rhs_sa_grdnu.F90:22-60)
      std::vector<R> q5j(G.N);
      for (long l = 0; l < G.N; ++l) q5j[l] = q5[l] / G.aj[l];
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = id(i, j, k);
            long ip = id(i + 1, j, k), imn = id(i - 1, j, k), jp = id(i, j + 1, k), jmn = id(i, j - 1, k);
            long kp = id(i, j, k + 1), kmn = id(i, j, k - 1);
            R dn[3];
            for (int x = 0; x < 3; ++x) {
              R v = dc2 * (q5j[ip] * G.csi[x][ip] - q5j[imn] * G.csi[x][imn]);
              v = v + de2 * (q5j[jp] * G.eta[x][jp] - q5j[jmn] * G.eta[x][jmn]);
              v = v + dz2 * (q5j[kp] * G.zet[x][kp] - q5j[kmn] * G.zet[x][kmn]);
              dn[x] = v;
            }
            R aj2 = G.aj[l] * G.aj[l];
            dnu[l] = aj2 * (dn[0] * dn[0] + dn[1] * dn[1] + dn[2] * dn[2]);
          }
      // rhs_sa_prod (src/rhs_sa_prod.F90:32-100)
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = id(i, j, k);
            if (G.wd[l] == zero) { psa[l] = zero; continue; }
            R chi = q5[l] / rei;
            R chic = chi * chi * chi;
            R fv1 = chic / (chic + cv1c);
            R t = one + chi / cv2;
            R fv2 = one / (t * t * t);
            R fv3 = ((one + chi * fv1) * (one - fv2)) / chi;
            R vtcm = std::sqrt(two * wo[l]);
            R cawd = capa * capa * G.wd[l] * G.wd[l];
            R vtc = fv3 * vtcm + q5[l] * fv2 / cawd;
            vtc = std::max(vtc, R(0.00001));
            R p = cb1 * vtc * q5[l];
            R rr = q5[l] / (vtc * cawd);
            R rr6 = rr * rr * rr * rr * rr * rr;
            R grr = rr + cw2 * (rr6 - rr);
            grr = std::max(zero, grr);
            R grr6 = grr * grr * grr * grr * grr * grr;
            R fw = grr * std::pow((one + cw3h) / (grr6 + cw3h), one / R(6));
            R vwd = q5[l] / G.wd[l];
            p = p - cw1 * fw * vwd * vwd;
            p = p + cb2 * dnu[l] / sig;
            psa[l] = p;
          }
      // rhs_sa_viscous (src/rhs_sa_viscous.F90:48-188)
      auto ret = [&](long l) { return (rei + q5[l]) / sig; };
      auto vflux = [&](long l0, long l1, int dir, R vcs, R vet, R vze) {
        R a1 = G.csi[0][l1] + G.csi[0][l0], a2 = G.csi[1][l1] + G.csi[1][l0], a3 = G.csi[2][l1] + G.csi[2][l0];
        R b1 = G.eta[0][l1] + G.eta[0][l0], b2 = G.eta[1][l1] + G.eta[1][l0], b3 = G.eta[2][l1] + G.eta[2][l0];
        R c1 = G.zet[0][l1] + G.zet[0][l0], c2 = G.zet[1][l1] + G.zet[1][l0], c3 = G.zet[2][l1] + G.zet[2][l0];
        R k1, k2, k3;
        if (dir == 0) { k1 = a1 * a1 + a2 * a2 + a3 * a3; k2 = a1 * b1 + a2 * b2 + a3 * b3; k3 = a1 * c1 + a2 * c2 + a3 * c3; }
        else if (dir == 1) { k1 = b1 * a1 + b2 * a2 + b3 * a3; k2 = b1 * b1 + b2 * b2 + b3 * b3; k3 = b1 * c1 + b2 * c2 + b3 * c3; }
        else { k1 = c1 * a1 + c2 * a2 + c3 * a3; k2 = c1 * b1 + c2 * b2 + c3 * b3; k3 = c1 * c1 + c2 * c2 + c3 * c3; }
        R vtj = R(0.25) * (ret(l1) + ret(l0)) / (G.aj[l1] + G.aj[l0]);
        return vtj * (k1 * vcs + k2 * vet + k3 * vze);
      };
      std::fill(fv.begin(), fv.end(), R(0));
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 1; i <= im - 1; ++i) {
            R vcs = dc * (q5[id(i + 1, j, k)] - q5[id(i, j, k)]);
            R vet = de4 * (q5[id(i + 1, j + 1, k)] - q5[id(i + 1, j - 1, k)] + q5[id(i, j + 1, k)] - q5[id(i, j - 1, k)]);
            R vze = dz4 * (q5[id(i + 1, j, k + 1)] - q5[id(i + 1, j, k - 1)] + q5[id(i, j, k + 1)] - q5[id(i, j, k - 1)]);
            fv[id(i, j, k)] = vflux(id(i, j, k), id(i + 1, j, k), 0, vcs, vet, vze);
          }
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) visc[id(i, j, k)] = fv[id(i, j, k)] - fv[id(i - 1, j, k)];
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 1; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            R vcs = dc4 * (q5[id(i + 1, j + 1, k)] - q5[id(i - 1, j + 1, k)] + q5[id(i + 1, j, k)] - q5[id(i - 1, j, k)]);
            R vet = de * (q5[id(i, j + 1, k)] - q5[id(i, j, k)]);
            R vze = dz4 * (q5[id(i, j + 1, k + 1)] - q5[id(i, j + 1, k - 1)] + q5[id(i, j, k + 1)] - q5[id(i, j, k - 1)]);
            fv[id(i, j, k)] = vflux(id(i, j, k), id(i, j + 1, k), 1, vcs, vet, vze);
          }
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) visc[id(i, j, k)] = visc[id(i, j, k)] + fv[id(i, j, k)] - fv[id(i, j - 1, k)];
      ORC_PARFOR
      for (int k = 1; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            R vcs = dc4 * (q5[id(i + 1, j, k + 1)] - q5[id(i - 1, j, k + 1)] + q5[id(i + 1, j, k)] - q5[id(i - 1, j, k)]);
            R vet = de4 * (q5[id(i, j + 1, k + 1)] - q5[id(i, j - 1, k + 1)] + q5[id(i, j + 1, k)] - q5[id(i, j - 1, k)]);
            R vze = dz * (q5[id(i, j, k + 1)] - q5[id(i, j, k)]);
            fv[id(i, j, k)] = vflux(id(i, j, k), id(i, j, k + 1), 2, vcs, vet, vze);
          }
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) visc[id(i, j, k)] = visc[id(i, j, k)] + fv[id(i, j, k)] - fv[id(i, j, k - 1)];
      // rhs_sa_flux (src/rhs_sa_flux.F90:32-109)
      const long st[3] = {1, (long)im, (long)im * jm};
      for (int dir = 0; dir < 3; ++dir) {
        std::fill(fv.begin(), fv.end(), R(0));
        ORC_PARFOR
        for (int k = (dir == 2 ? 1 : 2); k <= km - 1; ++k)
          for (int j = (dir == 1 ? 1 : 2); j <= jm - 1; ++j)
            for (int i = (dir == 0 ? 1 : 2); i <= im - 1; ++i) {
              long l = id(i, j, k), lp = l + st[dir];
              R eigh = pt5 * std::fabs(ucn[dir][lp] + ucn[dir][l]);
              fv[l] = pt5 * (q5[lp] * ucn[dir][lp] + q5[l] * ucn[dir][l] - eigh * (q5[lp] - q5[l]));
            }
        for (int k = 2; k <= km - 1; ++k)
          for (int j = 2; j <= jm - 1; ++j)
            for (int i = 2; i <= im - 1; ++i) {
              long l = id(i, j, k);
              if (dir == 0) rh[l] = fv[l] - fv[l - st[0]];
              else rh[l] = rh[l] + fv[l] - fv[l - st[dir]];
            }
      }
      // rhs_sa_unst_visc (src/rhs_sa_unst_visc.F90:18-30) and
      // rhs_sa_implicit_source (src/rhs_sa_implicit_source.F90:41-53); the
      // boundary values of rh are then zeroed (src/des_eddy.F90:231-236).
      ORC_PARFOR
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j)
          for (int i = 1; i <= im; ++i) {
            long l = id(i, j, k);
            bool interior = i > 1 && i < im && j > 1 && j < jm && k > 1 && k < km;
            if (!interior) { rh[l] = zero; continue; }
            R dtj = two * R(c.delti) * G.aj[l];
            R dq5dt = es * (R(3) * q5[l] - R(4) * G.qn[4][l] + G.qnm1[4][l]) / dtj;
            R r = rh[l] + dq5dt - visc[l] - psa[l] / G.aj[l];
            rh[l] = -G.dtev[l] * G.aj[l] * r;
          }
      // rhs_sa_adi_solver (src/rhs_sa_adi_solver.F90:40-244)
      const int ext[3] = {im, jm, km};
      const std::vector<R>* met[3] = {G.csi, G.eta, G.zet};
      for (int dir = 0; dir < 3; ++dir) {
        int len = ext[dir] - 2;
        int a1 = dir == 0 ? jm : im, a2 = dir == 2 ? jm : km;
ORC_PARFOR
        for (int p2 = 2; p2 <= a2 - 1; ++p2)
          for (int p1 = 2; p1 <= a1 - 1; ++p1) {
            std::vector<R> av(len + 1), aw(len), ap(len), ae(len), aq(len);
            auto node = [&](int t) { return dir == 0 ? id(t, p1, p2) : (dir == 1 ? id(p1, t, p2) : id(p1, p2, t)); };
            for (int t = 1; t <= ext[dir] - 1; ++t) {  // av(t) on the face t+1/2
              long l0 = node(t), l1 = node(t + 1);
              R gx = met[dir][0][l1] + met[dir][0][l0];
              R gy = met[dir][1][l1] + met[dir][1][l0];
              R gz = met[dir][2][l1] + met[dir][2][l0];
              R ev = (rei + pt5 * (q5[l1] + q5[l0])) / sig;
              R ucna = pt5 * std::fabs(ucn[dir][l1] + ucn[dir][l0]);
              av[t - 1] = ucna + ev * (gx * gx + gy * gy + gz * gz) / (G.aj[l1] + G.aj[l0]);
            }
            for (int t = 2; t <= ext[dir] - 1; ++t) {
              long l = node(t);
              R dtj = pt5 * G.dtev[l] * G.aj[l];
              int p = t - 2;
              aw[p] = -dtj * (ucn[dir][node(t - 1)] + av[t - 2]);
              ap[p] = one + dtj * (av[t - 2] + av[t - 1]);
              ae[p] = dtj * (ucn[dir][node(t + 1)] - av[t - 1]);
              aq[p] = rh[l];
            }
            std::vector<R> dl(aw.begin() + 1, aw.end()), du(ae.begin(), ae.end() - 1);
            long piv = 0;
            gtsv(len, 1, dl.data(), ap.data(), du.data(), aq.data(), len, &piv);
            if (piv) {
#ifdef _OPENMP
#pragma omp atomic
#endif
              pivots += piv;
            }
            for (int t = 2; t <= ext[dir] - 1; ++t) rh[node(t)] = aq[t - 2];
          }
      }
      // update (src/des_eddy.F90:260-272)
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = id(i, j, k);
            R qe5 = qold[l] + rh[l];
            R dum = one + R(1.5) * es * G.dtev[l] / R(c.delti);
            q5[l] = q5[l] + (-q5[l] + qe5) / dum;
          }
      sa_bcond();
      qold = q5;
    }
    phase_s[4] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // rhs_sa_bcond (src/rhs_sa_bcond.F90:22-291).  Interior ranges here are
  // 2..m-1; the face loops run over 1..m (ista = i_mysta - 1 etc.).
  void sa_bcond() {
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    std::vector<R>& q5 = G.q[4];
    auto Q = [&](int i, int j, int k) -> R& { return q5[G.id(i, j, k)]; };
    const R one = 1, zero = 0;
    for (int side = 0; side < 2; ++side) {
      int b = side, i = side ? im : 1, s = side ? -1 : 1;
      int bt = c.btype[b];
      for (int k = 1; k <= km; ++k)
        for (int j = 1; j <= jm; ++j) {
          if (bt == 1) Q(i, j, k) = zero;
          else if (bt == 2 || bt == 3) Q(i, j, k) = sa[0][b] * Q(i + s, j, k) + sb[0][b] * Q(i + 2 * s, j, k);
          else if (bt == 5) Q(i, j, k) = (one + ratv(b, j, k)) * Q(i + s, j, k) - ratv(b, j, k) * Q(i + 2 * s, j, k);
          else if (bt == 6) Q(i, j, k) = Q(side ? 2 : im - 1, j, k);
          else if (bt == 8 && side == 1) Q(i, j, k) = Q(i - 1, j, k);
        }
    }
    for (int side = 0; side < 2; ++side) {
      int b = 2 + side, j = side ? jm : 1, s = side ? -1 : 1;
      int bt = c.btype[b];
      for (int k = 1; k <= km; ++k)
        for (int i = 1; i <= im; ++i) {
          if (bt == 1) Q(i, j, k) = zero;
          else if (bt == 2 || bt == 3) Q(i, j, k) = sa[0][b] * Q(i, j + s, k) + sb[0][b] * Q(i, j + 2 * s, k);
          else if (bt == 5) Q(i, j, k) = (one + ratv(b, i, k)) * Q(i, j + s, k) - ratv(b, i, k) * Q(i, j + 2 * s, k);
          else if (bt == 6) Q(i, j, k) = Q(i, side ? 2 : jm - 1, k);
        }
    }
    for (int side = 0; side < 2; ++side) {
      int b = 4 + side, k = side ? km : 1, s = side ? -1 : 1;
      int bt = c.btype[b];
      for (int j = 1; j <= jm; ++j)
        for (int i = 1; i <= im; ++i) {
          if (bt == 1) Q(i, j, k) = zero;
          else if (bt == 2 || bt == 3) Q(i, j, k) = sa[0][b] * Q(i, j, k + s) + sb[0][b] * Q(i, j, k + 2 * s);
          else if (bt == 5) Q(i, j, k) = (one + ratv(b, i, j)) * Q(i, j, k + s) - ratv(b, i, j) * Q(i, j, k + 2 * s);
          else if (bt == 6) Q(i, j, k) = Q(i, j, side ? 2 : km - 1);
        }
    }
    const R rei = one / R(c.ren), cv1c = R(357.911);
    for (long l = 0; l < G.N; ++l) {
      q5[l] = std::max(R(1.0E-07), q5[l]);
      R chi = q5[l] / rei;
      R chic = chi * chi * chi;
      R fv1 = chic / (chic + cv1c);
      G.nut[l] = q5[l] * fv1;
    }
  }

  // ---------------------------------------------------------- k-omega model
  // Wilcox's (1994) low-Reynolds-number k-omega model of kw_eddy
  // (src/kw_eddy.F90:2-296), on the fine level: k is q(5) (the field SA
  // uses for nu_tilde) and omega q(6), held here in om / omn / omnm1 (the
  // reference's q(6), qn(2), qnm1(2)).  The reference builds none of this
  // (kw_eddy.F90 is not in src/makefile, no routine calls it, and its ADI
  // file rhs_kw_adi_solver_ijk.F90 does not exist), so this restatement is
  // parity unpinned.  Its parts:
  //   rhs_kw_ptke (src/rhs_kw_ptke.F90:42-96, nlinc = .false.), once per call;
  //   rhs_kw_coef (src/rhs_kw_coef.F90:41-54) on every node;
  //   per sub-iteration rhs_kw_prod (src/rhs_kw_prod.F90:18-31),
  //   rhs_kw_viscous (src/rhs_kw_viscous.F90:39-243), rhs_kw_flux
  //   (src/rhs_kw_flux.F90:20-166), rhs_kw_unst_visc
  //   (src/rhs_kw_unst_visc.F90:23-37), rhs_kw_implicit_source
  //   (src/rhs_kw_implicit_source.F90:41-53), the ADI, the update
  //   (src/kw_eddy.F90:247-266) and rhs_kw_bcond.
  // The ADI is restated from the SA model's (src/rhs_sa_adi_solver.F90:
  // 50-244) for each of k and omega: its rows divide by the implicit-source
  // factor dk (dw for omega) and the i sweep's right-hand side does too, as
  // there; the face diffusivity is the one rhs_kw_viscous uses,
  // 1/Re + (nu_t(l1) + nu_t(l0)) / (2 sigma).
  std::vector<R> om, omn, omnm1;
  R ckin = R(1.0e-10), cein = R(1.0e-6);

  // rhs_kw_coef (src/rhs_kw_coef.F90:41-54) on every node
  void kw_coef(std::vector<R>& As, std::vector<R>& Ac, std::vector<R>& Bs) const {
    const Level<R>& G = L[0];
    const std::vector<R>& k5 = G.q[4];
    ORC_PARFOR
    for (long l = 0; l < G.N; ++l) {
      R Rt = R(c.ren) * k5[l] / om[l];
      R Rt4 = Rt * Rt * Rt * Rt;
      As[l] = (R(0.15) + Rt) / (R(6) + Rt);
      Ac[l] = ((R(0.27) + Rt) / (R(2.70) + Rt)) * R(0.5555) / As[l];
      Bs[l] = ((R(1137.77) + Rt4) / (R(4096.00) + Rt4)) * R(0.09);
    }
  }

  void kw_eddy() {
    auto t0 = std::chrono::steady_clock::now();
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    const R cw2 = R(0.075), sk = R(2), sw = R(2);
    const R rei = R(1) / R(c.ren);
    const R one = 1, two = 2, pt5 = R(0.5), pt25 = R(0.25);
    const R dc = G.dc, de = G.de, dz = G.dz;
    const R dc2 = pt5 * dc, de2 = pt5 * de, dz2 = pt5 * dz;
    const R dc4 = pt25 * dc, de4 = pt25 * de, dz4 = pt25 * dz;
    std::vector<R>& k5 = G.q[4];
    std::vector<R> qold1(k5), qold2(om), ucn[3], ptke(G.N, R(0)), As(G.N), Ac(G.N), Bs(G.N);
    std::vector<R> pk1(G.N, R(0)), pk2(G.N, R(0)), v1(G.N, R(0)), v2(G.N, R(0)), r1(G.N, R(0)), r2(G.N, R(0));
    std::vector<R> f1(G.N, R(0)), f2(G.N, R(0)), dk(G.N, R(1)), dw(G.N, R(1));
    for (int d = 0; d < 3; ++d) ucn[d].assign(G.N, R(0));
    auto id = [&](int i, int j, int k) { return G.id(i, j, k); };
    contra_j(G, ucn);
    // rhs_kw_ptke, interior
    ORC_PARFOR
    for (int k = 2; k <= km - 1; ++k)
      for (int j = 2; j <= jm - 1; ++j)
        for (int i = 2; i <= im - 1; ++i) {
          long l = id(i, j, k);
          R g[3][3];  // g[var][dir]
          for (int m = 0; m < 3; ++m) {
            const std::vector<R>& v = G.q[m + 1];
            g[m][0] = dc2 * (v[id(i + 1, j, k)] - v[id(i - 1, j, k)]);
            g[m][1] = de2 * (v[id(i, j + 1, k)] - v[id(i, j - 1, k)]);
            g[m][2] = dz2 * (v[id(i, j, k + 1)] - v[id(i, j, k - 1)]);
          }
          R d[3][3];  // d[var][x]: du_var / dx_x
          for (int m = 0; m < 3; ++m)
            for (int x = 0; x < 3; ++x) d[m][x] = g[m][0] * G.csi[x][l] + g[m][1] * G.eta[x][l] + g[m][2] * G.zet[x][l];
          ptke[l] = G.nut[l] * (two * (d[0][0] * d[0][0] + d[1][1] * d[1][1] + d[2][2] * d[2][2]) +
                                (d[0][1] + d[1][0]) * (d[0][1] + d[1][0]) +
                                (d[0][2] + d[2][0]) * (d[0][2] + d[2][0]) +
                                (d[1][2] + d[2][1]) * (d[1][2] + d[2][1]));
        }
    kw_coef(As, Ac, Bs);
    const long st[3] = {1, (long)im, (long)im * jm};
    const std::vector<R>* met[3] = {G.csi, G.eta, G.zet};
    for (int iterk = 1; iterk <= c.itk; ++iterk) {
      // rhs_kw_prod
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = id(i, j, k);
            R pkw1a = Bs[l] * om[l] * k5[l];
            pk1[l] = (-ptke[l] + pkw1a) / G.aj[l];
            R pkw2a = -Ac[l] * om[l] * ptke[l] / k5[l];
            R pkw2b = cw2 * om[l] * om[l];
            pk2[l] = (pkw2a + pkw2b) / G.aj[l];
          }
      // rhs_kw_viscous: ret(1:2) on every node, then the face loops
      std::vector<R> ret1(G.N), ret2(G.N);
      for (long l = 0; l < G.N; ++l) { ret1[l] = rei + G.nut[l] / sk; ret2[l] = rei + G.nut[l] / sw; }
      for (int dir = 0; dir < 3; ++dir) {
        ORC_PARFOR
        for (int k = (dir == 2 ? 1 : 2); k <= km - 1; ++k)
          for (int j = (dir == 1 ? 1 : 2); j <= jm - 1; ++j)
            for (int i = (dir == 0 ? 1 : 2); i <= im - 1; ++i) {
              long l0 = id(i, j, k), l1 = l0 + st[dir];
              R g1[3], g2[3];  // derivatives of k and omega along csi, eta, zeta on the face
              for (int s = 0; s < 2; ++s) {
                const std::vector<R>& v = s == 0 ? k5 : om;
                R* g = s == 0 ? g1 : g2;
                if (dir == 0) {
                  g[0] = dc * (v[l1] - v[l0]);
                  g[1] = de4 * (v[l1 + st[1]] - v[l1 - st[1]] + v[l0 + st[1]] - v[l0 - st[1]]);
                  g[2] = dz4 * (v[l1 + st[2]] - v[l1 - st[2]] + v[l0 + st[2]] - v[l0 - st[2]]);
                } else if (dir == 1) {
                  g[0] = dc4 * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
                  g[1] = de * (v[l1] - v[l0]);
                  g[2] = dz4 * (v[l1 + st[2]] - v[l1 - st[2]] + v[l0 + st[2]] - v[l0 - st[2]]);
                } else {
                  g[0] = dc4 * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
                  g[1] = de4 * (v[l1 + st[1]] - v[l1 - st[1]] + v[l0 + st[1]] - v[l0 - st[1]]);
                  g[2] = dz * (v[l1] - v[l0]);
                }
              }
              R a1 = G.csi[0][l1] + G.csi[0][l0], a2 = G.csi[1][l1] + G.csi[1][l0], a3 = G.csi[2][l1] + G.csi[2][l0];
              R b1 = G.eta[0][l1] + G.eta[0][l0], b2 = G.eta[1][l1] + G.eta[1][l0], b3 = G.eta[2][l1] + G.eta[2][l0];
              R c1 = G.zet[0][l1] + G.zet[0][l0], c2 = G.zet[1][l1] + G.zet[1][l0], c3 = G.zet[2][l1] + G.zet[2][l0];
              R cc1, cc2, cc3;
              if (dir == 0) { cc1 = a1 * a1 + a2 * a2 + a3 * a3; cc2 = a1 * b1 + a2 * b2 + a3 * b3; cc3 = a1 * c1 + a2 * c2 + a3 * c3; }
              else if (dir == 1) { cc1 = b1 * a1 + b2 * a2 + b3 * a3; cc2 = b1 * b1 + b2 * b2 + b3 * b3; cc3 = b1 * c1 + b2 * c2 + b3 * c3; }
              else { cc1 = c1 * a1 + c2 * a2 + c3 * a3; cc2 = c1 * b1 + c2 * b2 + c3 * b3; cc3 = c1 * c1 + c2 * c2 + c3 * c3; }
              R vtj1 = pt25 * (ret1[l1] + ret1[l0]) / (G.aj[l1] + G.aj[l0]);
              R vtj2 = pt25 * (ret2[l1] + ret2[l0]) / (G.aj[l1] + G.aj[l0]);
              f1[l0] = vtj1 * (cc1 * g1[0] + cc2 * g1[1] + cc3 * g1[2]);
              f2[l0] = vtj2 * (cc1 * g2[0] + cc2 * g2[1] + cc3 * g2[2]);
            }
        ORC_PARFOR
        for (int k = 2; k <= km - 1; ++k)
          for (int j = 2; j <= jm - 1; ++j)
            for (int i = 2; i <= im - 1; ++i) {
              long l = id(i, j, k);
              if (dir == 0) { v1[l] = f1[l] - f1[l - 1]; v2[l] = f2[l] - f2[l - 1]; }
              else { v1[l] = v1[l] + f1[l] - f1[l - st[dir]]; v2[l] = v2[l] + f2[l] - f2[l - st[dir]]; }
            }
      }
      // rhs_kw_flux: first-order flux-difference upwinding
      for (int dir = 0; dir < 3; ++dir) {
        ORC_PARFOR
        for (int k = (dir == 2 ? 1 : 2); k <= km - 1; ++k)
          for (int j = (dir == 1 ? 1 : 2); j <= jm - 1; ++j)
            for (int i = (dir == 0 ? 1 : 2); i <= im - 1; ++i) {
              long l0 = id(i, j, k), l1 = l0 + st[dir];
              R gcu = (met[dir][0][l1] + met[dir][0][l0]) * (G.q[1][l1] + G.q[1][l0]);
              R gev = (met[dir][1][l1] + met[dir][1][l0]) * (G.q[2][l1] + G.q[2][l0]);
              R gzw = (met[dir][2][l1] + met[dir][2][l0]) * (G.q[3][l1] + G.q[3][l0]);
              R eigh = pt5 * std::fabs((gcu + gev + gzw) / (G.aj[l1] + G.aj[l0]));
              f1[l0] = pt5 * (k5[l1] * ucn[dir][l1] + k5[l0] * ucn[dir][l0] - eigh * (k5[l1] - k5[l0]));
              f2[l0] = pt5 * (om[l1] * ucn[dir][l1] + om[l0] * ucn[dir][l0] - eigh * (om[l1] - om[l0]));
            }
        ORC_PARFOR
        for (int k = 2; k <= km - 1; ++k)
          for (int j = 2; j <= jm - 1; ++j)
            for (int i = 2; i <= im - 1; ++i) {
              long l = id(i, j, k);
              if (dir == 0) { r1[l] = f1[l] - f1[l - 1]; r2[l] = f2[l] - f2[l - 1]; }
              else { r1[l] = r1[l] + f1[l] - f1[l - st[dir]]; r2[l] = r2[l] + f2[l] - f2[l - st[dir]]; }
            }
      }
      // rhs_kw_unst_visc and rhs_kw_implicit_source (interior; the boundary
      // rows are not read by the line solves)
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = id(i, j, k);
            R dtj = two * R(c.delti) * G.aj[l];
            R dq5dt = es * (R(3) * k5[l] - R(4) * G.qn[4][l] + G.qnm1[4][l]) / dtj;
            R dq6dt = es * (R(3) * om[l] - R(4) * omn[l] + omnm1[l]) / dtj;
            r1[l] = r1[l] + dq5dt - v1[l] + pk1[l];
            r2[l] = r2[l] + dq6dt - v2[l] + pk2[l];
            dk[l] = one + Bs[l] * G.dtev[l] * om[l];
            dw[l] = one + cw2 * G.dtev[l] * om[l];
            r1[l] = -G.dtev[l] * G.aj[l] * r1[l];
            r2[l] = -G.dtev[l] * G.aj[l] * r2[l];
          }
      // the ADI of each scalar (restated from src/rhs_sa_adi_solver.F90:50-244)
      const int ext[3] = {im, jm, km};
      for (int s = 0; s < 2; ++s) {
        std::vector<R>& rh = s == 0 ? r1 : r2;
        const std::vector<R>& df = s == 0 ? dk : dw;
        const R sig = s == 0 ? sk : sw;
        for (int dir = 0; dir < 3; ++dir) {
          int len = ext[dir] - 2;
          int a1 = dir == 0 ? jm : im, a2 = dir == 2 ? jm : km;
          ORC_PARFOR
          for (int p2 = 2; p2 <= a2 - 1; ++p2)
            for (int p1 = 2; p1 <= a1 - 1; ++p1) {
              std::vector<R> av(len + 1), aw(len), ap(len), ae(len), aq(len);
              auto node = [&](int t) { return dir == 0 ? id(t, p1, p2) : (dir == 1 ? id(p1, t, p2) : id(p1, p2, t)); };
              for (int t = 1; t <= ext[dir] - 1; ++t) {  // av(t) on the face t+1/2
                long l0 = node(t), l1 = node(t + 1);
                R gx = met[dir][0][l1] + met[dir][0][l0];
                R gy = met[dir][1][l1] + met[dir][1][l0];
                R gz = met[dir][2][l1] + met[dir][2][l0];
                R ev = rei + pt5 * (G.nut[l1] + G.nut[l0]) / sig;
                R ucna = pt5 * std::fabs(ucn[dir][l1] + ucn[dir][l0]);
                av[t - 1] = ucna + ev * (gx * gx + gy * gy + gz * gz) / (G.aj[l1] + G.aj[l0]);
              }
              for (int t = 2; t <= ext[dir] - 1; ++t) {
                long l = node(t);
                R dtj = pt5 * G.dtev[l] * G.aj[l] / df[l];
                int p = t - 2;
                aw[p] = -dtj * (ucn[dir][node(t - 1)] + av[t - 2]);
                ap[p] = one + dtj * (av[t - 2] + av[t - 1]);
                ae[p] = dtj * (ucn[dir][node(t + 1)] - av[t - 1]);
                aq[p] = dir == 0 ? rh[l] / df[l] : rh[l];
              }
              std::vector<R> dl(aw.begin() + 1, aw.end()), du(ae.begin(), ae.end() - 1);
              long piv = 0;
              gtsv(len, 1, dl.data(), ap.data(), du.data(), aq.data(), len, &piv);
              if (piv) {
#ifdef _OPENMP
#pragma omp atomic
#endif
                pivots += piv;
              }
              for (int t = 2; t <= ext[dir] - 1; ++t) rh[node(t)] = aq[t - 2];
            }
        }
      }
      // update (src/kw_eddy.F90:247-266)
      ORC_PARFOR
      for (int k = 2; k <= km - 1; ++k)
        for (int j = 2; j <= jm - 1; ++j)
          for (int i = 2; i <= im - 1; ++i) {
            long l = id(i, j, k);
            R qe5 = qold1[l] + r1[l];
            R qe6 = qold2[l] + r2[l];
            R dum = one + R(1.5) * es * G.dtev[l] / R(c.delti);
            k5[l] = k5[l] + (-k5[l] + qe5) / dum;
            om[l] = om[l] + (-om[l] + qe6) / dum;
          }
      kw_bcond(As, Ac, Bs);
      qold1 = k5;
      qold2 = om;
    }
    phase_s[4] += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }

  // rhs_kw_bcond (src/rhs_kw_bcond.F90:22-519).  Face loops cover the
  // face's interior plus the edges toward non-wall faces (ista = i_mysta - 1
  // where btype(1) /= 1, :44-49); a wall face gets k = 0 and omega =
  // 60 / (Re 0.075 yd^2) from the adjacent node's wall distance; then As,
  // Ac, Bs and nu_t = As k / omega on every node (:477-491, nlinc =
  // .false.); then omega on each edge where two wall faces meet is the mean
  // of its two face neighbours, edges in the reference's order (:493-519;
  // its first condition's ".and btype(3)" read as ".and. btype(3)").
  void kw_bcond(std::vector<R>& As, std::vector<R>& Ac, std::vector<R>& Bs) {
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    std::vector<R>& k5 = G.q[4];
    auto K = [&](int i, int j, int k) -> R& { return k5[G.id(i, j, k)]; };
    auto W = [&](int i, int j, int k) -> R& { return om[G.id(i, j, k)]; };
    const R srenp = R(60) / R(c.ren) / R(0.075), one = 1, pt5 = R(0.5);
    const int ista = c.btype[0] != 1 ? 1 : 2, iend = c.btype[1] != 1 ? im : im - 1;
    const int jsta = c.btype[2] != 1 ? 1 : 2, jend = c.btype[3] != 1 ? jm : jm - 1;
    const int ksta = c.btype[4] != 1 ? 1 : 2, kend = c.btype[5] != 1 ? km : km - 1;
    // one boundary node (i, j, k) of face b, its inward neighbours (i1..), (i2..)
    auto face = [&](int b, int i, int j, int k, int i1, int j1, int k1, int i2, int j2, int k2, int ip, int jp, int kp, R r) {
      const int bt = c.btype[b];
      if (bt == 1) {
        R yd = G.wd[G.id(i1, j1, k1)];
        W(i, j, k) = srenp / yd / yd;
        K(i, j, k) = 0;
      } else if (bt == 2 || bt == 3) {
        K(i, j, k) = sa[0][b] * K(i1, j1, k1) + sb[0][b] * K(i2, j2, k2);
        W(i, j, k) = sa[0][b] * W(i1, j1, k1) + sb[0][b] * W(i2, j2, k2);
        K(i, j, k) = std::max(ckin, K(i, j, k));
        W(i, j, k) = std::max(cein, W(i, j, k));
      } else if (bt == 5) {
        K(i, j, k) = (one + r) * K(i1, j1, k1) - r * K(i2, j2, k2);
        W(i, j, k) = (one + r) * W(i1, j1, k1) - r * W(i2, j2, k2);
        K(i, j, k) = std::max(ckin, K(i, j, k));
        W(i, j, k) = std::max(cein, W(i, j, k));
      } else if (bt == 6) {
        K(i, j, k) = K(ip, jp, kp);
        W(i, j, k) = W(ip, jp, kp);
        K(i, j, k) = std::max(ckin, K(i, j, k));
        W(i, j, k) = std::max(cein, W(i, j, k));
      }
    };
    for (int k = ksta; k <= kend; ++k)
      for (int j = jsta; j <= jend; ++j) face(0, 1, j, k, 2, j, k, 3, j, k, im - 1, j, k, ratv(0, j, k));
    for (int k = ksta; k <= kend; ++k)
      for (int j = jsta; j <= jend; ++j) face(1, im, j, k, im - 1, j, k, im - 2, j, k, 2, j, k, ratv(1, j, k));
    for (int k = ksta; k <= kend; ++k)
      for (int i = ista; i <= iend; ++i) face(2, i, 1, k, i, 2, k, i, 3, k, i, jm - 1, k, ratv(2, i, k));
    for (int k = ksta; k <= kend; ++k)
      for (int i = ista; i <= iend; ++i) face(3, i, jm, k, i, jm - 1, k, i, jm - 2, k, i, 2, k, ratv(3, i, k));
    for (int j = jsta; j <= jend; ++j)
      for (int i = ista; i <= iend; ++i) face(4, i, j, 1, i, j, 2, i, j, 3, i, j, km - 1, ratv(4, i, j));
    for (int j = jsta; j <= jend; ++j)
      for (int i = ista; i <= iend; ++i) face(5, i, j, km, i, j, km - 1, i, j, km - 2, i, j, 2, ratv(5, i, j));
    kw_coef(As, Ac, Bs);
    for (long l = 0; l < G.N; ++l) G.nut[l] = As[l] * k5[l] / om[l];
    const int* bt = c.btype;
    if (bt[0] == 1 && bt[2] == 1) for (int k = 1; k <= km; ++k) W(1, 1, k) = pt5 * (W(2, 1, k) + W(1, 2, k));
    if (bt[0] == 1 && bt[3] == 1) for (int k = 1; k <= km; ++k) W(1, jm, k) = pt5 * (W(2, jm, k) + W(1, jm - 1, k));
    if (bt[0] == 1 && bt[4] == 1) for (int j = 1; j <= jm; ++j) W(1, j, 1) = pt5 * (W(2, j, 1) + W(1, j, 2));
    if (bt[0] == 1 && bt[5] == 1) for (int j = 1; j <= jm; ++j) W(1, j, km) = pt5 * (W(2, j, km) + W(1, j, km - 1));
    if (bt[1] == 1 && bt[2] == 1) for (int k = 1; k <= km; ++k) W(im, 1, k) = pt5 * (W(im - 1, 1, k) + W(im, 2, k));
    if (bt[1] == 1 && bt[3] == 1) for (int k = 1; k <= km; ++k) W(im, jm, k) = pt5 * (W(im - 1, jm, k) + W(im, jm - 1, k));
    if (bt[1] == 1 && bt[4] == 1) for (int j = 1; j <= jm; ++j) W(im, j, 1) = pt5 * (W(im - 1, j, 1) + W(im, j, 2));
    if (bt[1] == 1 && bt[5] == 1) for (int j = 1; j <= jm; ++j) W(im, j, km) = pt5 * (W(im - 1, j, km) + W(im, j, km - 1));
    if (bt[2] == 1 && bt[4] == 1) for (int i = 1; i <= im; ++i) W(i, 1, 1) = pt5 * (W(i, 2, 1) + W(i, 1, 2));
    if (bt[2] == 1 && bt[5] == 1) for (int i = 1; i <= im; ++i) W(i, 1, km) = pt5 * (W(i, 2, km) + W(i, 1, km - 1));
    if (bt[3] == 1 && bt[4] == 1) for (int i = 1; i <= im; ++i) W(i, jm, 1) = pt5 * (W(i, jm - 1, 1) + W(i, jm, 2));
    if (bt[3] == 1 && bt[5] == 1) for (int i = 1; i <= im; ++i) W(i, jm, km) = pt5 * (W(i, jm - 1, km) + W(i, jm, km - 1));
  }

  // Friction velocity u_tau of the wall law the reference solves
  // (funcv, src/wf_mpi.F90:602-628, ks = 0): with c = Re y,
  //   c u_tau^2 = u0                          when c u_tau <= 11.3,
  //   u_tau (ln(c u_tau) / kappa + B) = u0    when c u_tau > 11.3,
  // and funcv's zero band at c u_tau = 11.3 (:627) taken as the root where
  // u0 falls in the jump between the two branches.  The reference finds it
  // with a third-party Newton / line-search driver stopped at |F| < 1e-4
  // (:640); this restatement solves the equation to full precision: the
  // linear branch in closed form, the log branch (convex, increasing) by
  // Newton's method from the branch point, whose first step lands right of
  // the root and whose later steps decrease monotonically onto it.
  static R wf_utau(R u0, R c) {
    const R kapa = R(0.41), blog = R(5.45), yk = R(11.3);
    if (!(c > R(0)) || !(u0 > R(0))) return R(0);
    if (c * u0 <= yk * yk) return std::sqrt(u0 / c);
    const R us = yk / c;
    if (us * (std::log(yk) / kapa + blog) >= u0) return us;
    R ut = us;
    for (int it = 0; it < 100; ++it) {
      const R lg = std::log(c * ut);
      const R g = ut * (lg / kapa + blog) - u0;
      const R dg = lg / kapa + blog + R(1) / kapa;
      const R nx = ut - g / dg;
      const bool done = std::fabs(nx - ut) <= R(4) * std::numeric_limits<R>::epsilon() * nx;
      ut = nx;
      if (done) break;
    }
    return ut;
  }

  // wf_eta(jb) (src/wf_mpi.F90:246-413) on the fine level, jb = 1 (j = 1
  // wall, layers j = 2, 3) and jb = 2 (j = jm wall, layers jm-1, jm-2); the
  // driver calls both after every fine solver_daf (src/mg_driver.F90:
  // 221-224).  u_tau comes from the wall-parallel speed at layer 3 and its
  // wall distance; the velocity at layer 2 is set to the wall law's speed at
  // layer 2's wall distance, in the direction of layer 3's velocity resolved
  // along the wall's csi and zeta lines; nu_tilde there to kappa y+ / Re.
  // Interior (i, k) only.  A wall-parallel speed whose square root argument
  // rounds below zero is taken as zero (the reference's sqrt would return
  // NaN there).
  void wall_functions() {
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    const R kapa = R(0.41), blog = R(5.45), yplm = R(11.3), qmin = R(1.0E-08);
    const R ren = R(c.ren), half = R(0.5);
    std::vector<R>* Q = G.q;
    for (int jb = 1; jb <= 2; ++jb) {
      const int j = jb == 1 ? 1 : jm, j1 = jb == 1 ? 2 : jm - 1, j2 = jb == 1 ? 3 : jm - 2;
      std::vector<R> ut0((long)im * km, R(0));
      auto uo = [&](int i, int k) -> R& { return ut0[(long)(i - 1) + (long)im * (k - 1)]; };
      for (int k = 2; k <= km - 1; ++k)
        for (int i = 2; i <= im - 1; ++i) {
          long l = G.id(i, j, k), l2 = G.id(i, j2, k);
          R vmod = std::sqrt(G.eta[0][l] * G.eta[0][l] + G.eta[1][l] * G.eta[1][l] + G.eta[2][l] * G.eta[2][l]);
          R qnor = (Q[1][l2] * G.eta[0][l] + Q[2][l2] * G.eta[1][l] + Q[3][l2] * G.eta[2][l]) / vmod;
          R qpar = Q[1][l2] * Q[1][l2] + Q[2][l2] * Q[2][l2] + Q[3][l2] * Q[3][l2];
          qpar = std::sqrt(std::max(qpar - qnor * qnor, R(0)));
          uo(i, k) = wf_utau(qpar, ren * G.wd[l2]);
        }
      for (int k = 2; k <= km - 1; ++k)
        for (int i = 2; i <= im - 1; ++i) {
          long l1 = G.id(i, j1, k), l2 = G.id(i, j2, k);
          R qsq = Q[1][l2] * Q[1][l2] + Q[2][l2] * Q[2][l2] + Q[3][l2] * Q[3][l2];
          if (qsq > qmin) {
            const R ut = uo(i, k);
            R yplus = G.wd[l1] * ren * ut;
            R q2 = yplus > yplm ? (std::log(yplus) / kapa + blog) * ut : yplus * ut;
            long lu = G.id(i + 1, j, k), ld = G.id(i - 1, j, k);
            R xc = half * (G.x[lu] - G.x[ld]), yc = half * (G.y[lu] - G.y[ld]), zc = half * (G.z[lu] - G.z[ld]);
            lu = G.id(i, j, k + 1); ld = G.id(i, j, k - 1);
            R xz = half * (G.x[lu] - G.x[ld]), yz = half * (G.y[lu] - G.y[ld]), zz = half * (G.z[lu] - G.z[ld]);
            R sg11 = std::sqrt(xc * xc + yc * yc + zc * zc);
            R sg33 = std::sqrt(xz * xz + yz * yz + zz * zz);
            R qc1 = (G.csi[0][l2] * Q[1][l2] + G.csi[1][l2] * Q[2][l2] + G.csi[2][l2] * Q[3][l2]) * sg11;
            R qc2 = (G.zet[0][l2] * Q[1][l2] + G.zet[1][l2] * Q[2][l2] + G.zet[2][l2] * Q[3][l2]) * sg33;
            R cgama = (xc * xz + yc * yz + zc * zz) / (sg11 * sg33);
            R fb = std::sqrt(qc1 * qc1 + qc2 * qc2 + R(2) * qc1 * qc2 * cgama);
            fb = (qc1 + qc2 * cgama) / fb;
            fb = std::min(fb, R(1));
            fb = std::max(fb, R(-1));
            R fbeta = qc2 > R(0) ? std::acos(fb) : -std::acos(fb);
            R qstar = q2;
            R c2 = qstar * std::sin(fbeta) / std::sin(std::acos(cgama));
            R c1 = qstar * std::cos(fbeta) - c2 * cgama;
            Q[1][l1] = c1 * xc / sg11 + c2 * xz / sg33;
            Q[2][l1] = c1 * yc / sg11 + c2 * yz / sg33;
            Q[3][l1] = c1 * zc / sg11 + c2 * zz / sg33;
            Q[4][l1] = kapa * yplus / ren;
          } else {
            Q[1][l1] = Q[2][l1] = Q[3][l1] = R(0);
            Q[4][l1] = R(0.1) / ren;
          }
        }
    }
  }

  // conservation (src/conservation.F90:64-160): on one rank the first and
  // last i planes are the domain's inflow and outflow planes.
  void conservation() {
    Level<R>& G = L[0];
    const int im = G.im, jm = G.jm, km = G.km;
    std::vector<R> ucn[3];
    for (int d = 0; d < 3; ++d) ucn[d].assign(G.N, R(0));
    contra_j(G, ucn);
    R fin = 0, fout = 0;
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j) fin = fin + ucn[0][G.id(1, j, k)];
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j) fout = fout + ucn[0][G.id(im, j, k)];
    R delta_e = fin - fout;
    for (int k = 1; k <= km; ++k)
      for (int j = 1; j <= jm; ++j) {
        long l = G.id(im, j, k);
        R u1 = ucn[0][l] + delta_e * ucn[0][l] / fout;
        R a = G.aj[l];
        G.q[1][l] = a * (u1 * G.xc[l] + ucn[1][l] * G.xe[l] + ucn[2][l] * G.xz[l]);
        G.q[2][l] = a * (u1 * G.yc[l] + ucn[1][l] * G.ye[l] + ucn[2][l] * G.yz[l]);
        G.q[3][l] = a * (u1 * G.zc[l] + ucn[1][l] * G.ze[l] + ucn[2][l] * G.zz[l]);
      }
  }

  // ---------------------------------------------------------- the driver
  void save_qold() {
    for (int m = 0; m < 5; ++m) L[0].qold[m] = L[0].q[m];
  }

  // History shift, coarse injection and initial guess (src/mg_driver.F90:42-75).
  void begin_step() {
    Level<R>& F = L[0];
    for (int m = 0; m < 5; ++m) { F.qnm1[m] = F.qn[m]; F.qn[m] = F.q[m]; }
    if (c.turbulence == 2) { omnm1 = omn; omn = om; }
    if (c.predictor == DESALM_PRED_LINEAR) {
      for (int m = 0; m < 5; ++m)
        for (long l = 0; l < F.N; ++l) F.q[m][l] = R(2) * F.qn[m][l] - F.qnm1[m][l];
      if (c.turbulence == 2)
        for (long l = 0; l < F.N; ++l) om[l] = R(2) * omn[l] - omnm1[l];
    }
    for (int m = 0; m < 5; ++m) { inject_arr(&Level<R>::qn, m); inject_arr(&Level<R>::qnm1, m); }
    if (c.conservation) conservation();
    itc = 0;
  }

  // One pseudo-time iteration (src/mg_driver.F90:81-316).  Returns converged.
  bool pseudo_iteration(double* res) {
    itc++;
    save_qold();
    int recalc = 0;
    for (int n = 0; n < ng; ++n) {
      if (n > 0) mg_nlevel(n);
      for (int itr = 1; itr <= c.iter[n]; ++itr) {
        if (n != ng - 1) recalc = (itr != c.iter[n]) ? 0 : 1;  // kept at n = ng (Q5)
        if (c.turbulence == 1 && n == 0) des_eddy();
        if (c.turbulence == 2 && n == 0) kw_eddy();
        solver_daf(n, recalc, itr);
        if (c.wall_functions && n == 0) wall_functions();  // src/mg_driver.F90:221-224
      }
    }
    for (int n = ng - 2; n >= 0; --n) mg_prolong(n);
    bcond_fm();
    mg_residual(0, res);
    // mg_ck_conver (src/mg_driver.F90:372-398)
    if (itc == 1) for (int m = 0; m < 5; ++m) init_resd[m] = R(res[m]);
    R eomax = std::max(R(res[1]), std::max(R(res[2]), R(res[3])));
    R ermax = std::max(R(res[1]) - init_resd[1], std::max(R(res[2]) - init_resd[2], R(res[3]) - init_resd[3]));
    bool conv = false;
    if (itc > c.it_min && ermax < R(c.er_min)) conv = true;
    if (itc > c.it_min && eomax < R(c.eo_min)) conv = true;
    return conv;
  }
};

}  // namespace orc
