// sa.cuh -- Spalart-Allmaras sub-iterations on the fine level (des_eddy,
// src/des_eddy.F90:109-297) and the outlet mass-flux fix (conservation,
// src/conservation.F90:64-160).  nu_tilde, nu_t and the residual terms are
// FP64 in every precision mode; the ADI rows and line solves run in the
// sweep precision SW (FP32 in MIXED mode).
#pragma once
#include "common.cuh"
#include "sweep.cuh"

namespace desalm {

// fine-level FP64 work arrays of the SA model
struct SaWork {
  static const int NARR = 14;
  double* a[NARR];  // wo, rh5, the ADI coefficients aw, ap, ae of the i, j, k lines, U/J V/J W/J
};

// SW: type of the ADI work arrays and arithmetic (double in FP64 mode,
// float in MIXED mode, where the ADI is the FP32 preconditioner of an FP64
// residual); nu_tilde, nu_t and the residual terms stay FP64.
template <class SW>
struct SaT {
  int im, jm, km, N, sj, sk;
  double* q[5];
  const double* qn5;
  const double* qnm1_5;
  const double* csi[3];
  const double* eta[3];
  const double* zet[3];
  const double* aj;
  const double* rj;  // 1/aj
  const double* wd;
  const double* dtev;
  double* nut;
  double* wo;
  SW* rh;
  SW* co[9];        // co[3 d + 0..2] = aw, ap, ae of the direction-d line through each interior node
  double* uc[3];  // contravariant U/J of each direction on every node, for the current velocities
  double* upd;    // the scalar the last (k) sweep updates: nu_tilde (q[4]) for SA; k or omega for k-omega
  SW* gs;         // line-solve scratch of k_sa_gsweep: 4 arrays gss elements apart
  int gss;
  int* flags;
  double ren, delti, es;
  double sa1[6], sb1[6];  // pressure-row extrapolation coefficients, sa(1,b), sb(1,b)
  int btype[6];
  const double* rat;      // extrapolation ratios rat(:,:,b), [6][ratdim][ratdim]
  int ratdim;
};

using Sa = SaT<double>;

template <class SW>
DESALM_DEV double sa_ucn(const SaT<SW>& S, int d, int l) {
  const double* const* m = d == 0 ? S.csi : (d == 1 ? S.eta : S.zet);
  double tmp = S.rj[l];
  return tmp * (m[0][l] * S.q[1][l] + m[1][l] * S.q[2][l] + m[2][l] * S.q[3][l]);
}

// U/J of the three directions on every node (src/rhs_contra_j.F90:14-29), once
// per pseudo-iteration: the velocities do not change during the SA
// sub-iterations.
template <class SW>
__global__ void k_sa_ucn(SaT<SW> S) {
  pdl_wait();
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= S.N) return;
#pragma unroll
  for (int d = 0; d < 3; ++d) S.uc[d][l] = sa_ucn(S, d, l);
}

// vorticity magnitude wo = 2 |W|^2 on interior nodes (src/rhs_sa_source.F90:44-93)
template <class SW>
__global__ void k_sa_source(SaT<SW> S) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z + 1;
  if (i > S.im - 2 || j > S.jm - 2) return;
  const int l = i + S.sj * j + S.sk * k;
  double g[3][3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const double* v = S.q[m + 1];
    g[m][0] = 0.5 * (v[l + 1] - v[l - 1]);
    g[m][1] = 0.5 * (v[l + S.sj] - v[l - S.sj]);
    g[m][2] = 0.5 * (v[l + S.sk] - v[l - S.sk]);
  }
  double d[3][3];
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int x = 0; x < 3; ++x) d[m][x] = g[m][0] * S.csi[x][l] + g[m][1] * S.eta[x][l] + g[m][2] * S.zet[x][l];
  double w12 = 0.5 * (d[0][1] - d[1][0]);
  double w13 = 0.5 * (d[0][2] - d[2][0]);
  double w23 = 0.5 * (d[1][2] - d[2][1]);
  S.wo[l] = 2.0 * (w12 * w12 + w13 * w13 + w23 * w23);
}

// viscous flux of nu_tilde through the face l0 -> l0 + st[dir]
// (src/rhs_sa_viscous.F90:58-175)
template <class SW>
DESALM_DEV double sa_visc_face(const SaT<SW>& S, int dir, int l0, double rei, double rsig, double* gvt = nullptr) {
  const int sj = S.sj, sk = S.sk;
  const double* v = S.q[4];
  int l1;
  double vcs, vet, vze;
  if (dir == 0) {
    l1 = l0 + 1;
    vcs = v[l1] - v[l0];
    vet = 0.25 * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
    vze = 0.25 * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
  } else if (dir == 1) {
    l1 = l0 + sj;
    vcs = 0.25 * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
    vet = v[l1] - v[l0];
    vze = 0.25 * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
  } else {
    l1 = l0 + sk;
    vcs = 0.25 * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
    vet = 0.25 * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
    vze = v[l1] - v[l0];
  }
  double a1 = S.csi[0][l1] + S.csi[0][l0], a2 = S.csi[1][l1] + S.csi[1][l0], a3 = S.csi[2][l1] + S.csi[2][l0];
  double b1 = S.eta[0][l1] + S.eta[0][l0], b2 = S.eta[1][l1] + S.eta[1][l0], b3 = S.eta[2][l1] + S.eta[2][l0];
  double c1 = S.zet[0][l1] + S.zet[0][l0], c2 = S.zet[1][l1] + S.zet[1][l0], c3 = S.zet[2][l1] + S.zet[2][l0];
  double k1, k2, k3;
  if (dir == 0) { k1 = a1 * a1 + a2 * a2 + a3 * a3; k2 = a1 * b1 + a2 * b2 + a3 * b3; k3 = a1 * c1 + a2 * c2 + a3 * c3; }
  else if (dir == 1) { k1 = b1 * a1 + b2 * a2 + b3 * a3; k2 = b1 * b1 + b2 * b2 + b3 * b3; k3 = b1 * c1 + b2 * c2 + b3 * c3; }
  else { k1 = c1 * a1 + c2 * a2 + c3 * a3; k2 = c1 * b1 + c2 * b2 + c3 * b3; k3 = c1 * c1 + c2 * c2 + c3 * c3; }
  double vtj = 0.25 * ((rei + v[l1]) * rsig + (rei + v[l0]) * rsig) / (S.aj[l1] + S.aj[l0]);
  // the face's diffusive ADI coefficient ((1/Re + (nu1 + nu0) / 2) / sigma)
  // |g_dir|^2 / (J1 + J0) with the summed metrics, which is 2 vtj times the
  // direction's own product (k1, k2 or k3)
  if (gvt) *gvt = 2.0 * vtj * (dir == 0 ? k1 : (dir == 1 ? k2 : k3));
  return vtj * (k1 * vcs + k2 * vet + k3 * vze);
}

// first-order flux-difference upwind flux of nu_tilde through the face
// l0 -> l0 + st (src/rhs_sa_flux.F90:32-109)
template <class SW>
DESALM_DEV double sa_conv_face(const SaT<SW>& S, int dir, int l0, int st, double* ucf = nullptr) {
  const int l1 = l0 + st;
  const double u1 = S.uc[dir][l1], u0 = S.uc[dir][l0];
  if (ucf) { ucf[0] = u0; ucf[1] = u1; }
  const double* v = S.q[4];
  double eigh = 0.5 * fabs(u1 + u0);
  return 0.5 * (v[l1] * u1 + v[l0] * u0 - eigh * (v[l1] - v[l0]));
}

// Tridiagonal row (aw, ap, ae) of the scalar ADI for nu_tilde at interior
// node l along direction d (src/rhs_sa_adi_solver.F90:50-244): first-order
// upwind convection plus the face diffusivity, scaled by dtev J / 2, stored per
// node so that the three sweeps read three coefficients.  It is formed from
// the two faces the residual has just computed: av = |U/J| on the face + the
// face's diffusive coefficient gm (face (l - s, l)) or gp (face (l, l + s));
// um, up are the faces' U/J pairs.
template <class SW>
DESALM_DEV void sa_adi_row(const SaT<SW>& S, int l, int d, double gm, double gp, const double um[2],
                           const double up[2]) {
  const double av0 = 0.5 * fabs(um[1] + um[0]) + gm;
  const double av1 = 0.5 * fabs(up[1] + up[0]) + gp;
  const double dtj = 0.5 * S.dtev[l] * S.aj[l];
  S.co[3 * d + 0][l] = SW(-dtj * (um[0] + av0));
  S.co[3 * d + 1][l] = SW(1.0 + dtj * (av0 + av1));
  S.co[3 * d + 2][l] = SW(dtj * (up[1] - av1));
}

// One fused pass of rhs_sa_grdnu, rhs_sa_prod, rhs_sa_viscous, rhs_sa_flux,
// rhs_sa_unst_visc and rhs_sa_implicit_source on interior nodes
// (src/des_eddy.F90:164-223), plus the ADI rows; boundary values of rh stay
// zero.  Divisions by J and by sigma_SA are multiplications by 1/J and 1.5,
// U/J comes from k_sa_ucn, and f_w's sixth root is cbrt(sqrt(x)); the results
// equal the reference's expressions up to rounding.
// Minimum resident CTAs per SM requested for k_sa_rhs (128 threads each); a
// build-time tuning knob.  5 (96 registers, 96 B of spills) against 4 (127
// registers): 0.477 against 0.492 s per MIXED channel step on one box.
#ifndef DESALM_SA_MINBLOCKS
#define DESALM_SA_MINBLOCKS 5
#endif
template <class SW>
__global__ void __launch_bounds__(128, DESALM_SA_MINBLOCKS) k_sa_rhs(SaT<SW> S) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int k = blockIdx.z * blockDim.z + threadIdx.z + 1;
  if (i > S.im - 2 || j > S.jm - 2 || k > S.km - 2) return;
  const int sj = S.sj, sk = S.sk;
  const int l = i + sj * j + sk * k;
  const double cb1 = 0.1355, cb2 = 0.622, rsig = 1.5, capa = 0.41;  // rsig = 1 / sigma_SA
  const double cw1 = 3.23906782, cw2 = 0.3, cw3h = 64.0, cv1c = 357.911, cv2 = 5.0;
  const double rei = 1.0 / S.ren;
  const double* q5 = S.q[4];
  const int st[3] = {1, sj, sk};
  const double* const* mt[3] = {S.csi, S.eta, S.zet};
  // gradient of nu_tilde (src/rhs_sa_grdnu.F90:22-60)
  double dn[3];
  {
    double qp[3], qm[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      qp[d] = q5[l + st[d]] * S.rj[l + st[d]];
      qm[d] = q5[l - st[d]] * S.rj[l - st[d]];
    }
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      double v = 0.5 * (qp[0] * mt[0][x][l + 1] - qm[0] * mt[0][x][l - 1]);
      v = v + 0.5 * (qp[1] * mt[1][x][l + sj] - qm[1] * mt[1][x][l - sj]);
      v = v + 0.5 * (qp[2] * mt[2][x][l + sk] - qm[2] * mt[2][x][l - sk]);
      dn[x] = v;
    }
  }
  double aj2 = S.aj[l] * S.aj[l];
  double dnu = aj2 * (dn[0] * dn[0] + dn[1] * dn[1] + dn[2] * dn[2]);
  // production, destruction, diffusion (src/rhs_sa_prod.F90:32-100)
  double psa;
  const double w = S.wd[l];
  if (w == 0.0) {
    psa = 0.0;
  } else {
    double nt = q5[l];
    double chi = nt * S.ren;
    double chic = chi * chi * chi;
    double fv1 = chic / (chic + cv1c);
    double t = 1.0 + chi / cv2;
    double fv2 = 1.0 / (t * t * t);
    double fv3 = ((1.0 + chi * fv1) * (1.0 - fv2)) / chi;
    double vtcm = sqrt(2.0 * S.wo[l]);
    double cawd = capa * capa * w * w;
    double vtc = fv3 * vtcm + nt * fv2 / cawd;
    vtc = vtc > 0.00001 ? vtc : 0.00001;
    double p = cb1 * vtc * nt;
    double rr = nt / (vtc * cawd);
    double rr6 = rr * rr * rr * rr * rr * rr;
    double grr = rr + cw2 * (rr6 - rr);
    grr = grr > 0.0 ? grr : 0.0;
    double grr6 = grr * grr * grr * grr * grr * grr;
    double fw = grr * cbrt(sqrt((1.0 + cw3h) / (grr6 + cw3h)));  // x^(1/6)
    double vwd = nt / w;
    p = p - cw1 * fw * vwd * vwd;
    p = p + cb2 * dnu * rsig;
    psa = p;
  }
  // viscous terms and convective flux; each face also gives what the ADI
  // rows of its direction need (diffusive coefficient, U/J pair)
  double gdm[3], gdp[3], ucm[3][2], ucp[3][2];
  double visc = sa_visc_face(S, 0, l, rei, rsig, &gdp[0]) - sa_visc_face(S, 0, l - 1, rei, rsig, &gdm[0]);
  visc = visc + sa_visc_face(S, 1, l, rei, rsig, &gdp[1]) - sa_visc_face(S, 1, l - sj, rei, rsig, &gdm[1]);
  visc = visc + sa_visc_face(S, 2, l, rei, rsig, &gdp[2]) - sa_visc_face(S, 2, l - sk, rei, rsig, &gdm[2]);
  double rh = sa_conv_face(S, 0, l, 1, ucp[0]) - sa_conv_face(S, 0, l - 1, 1, ucm[0]);
  rh = rh + sa_conv_face(S, 1, l, sj, ucp[1]) - sa_conv_face(S, 1, l - sj, sj, ucm[1]);
  rh = rh + sa_conv_face(S, 2, l, sk, ucp[2]) - sa_conv_face(S, 2, l - sk, sk, ucm[2]);
  // unsteady term and implicit source scaling
  double rdtj = 1.0 / (2.0 * S.delti * S.aj[l]);
  double dq5dt = S.es * (3.0 * q5[l] - 4.0 * S.qn5[l] + S.qnm1_5[l]) * rdtj;
  double r = rh + dq5dt - visc - psa * S.rj[l];
  S.rh[l] = SW(-S.dtev[l] * S.aj[l] * r);
  // ADI rows of the three directions for this nu_tilde (its values change
  // only at the end of the k sweep)
#pragma unroll
  for (int d = 0; d < 3; ++d) sa_adi_row<SW>(S, l, d, gdm[d], gdp[d], ucm[d], ucp[d]);
}

// Scalar ADI sweep of nu_tilde along one direction
// (src/rhs_sa_adi_solver.F90:50-244) on the stored rows, as a shared-memory
// slab: a CTA owns NL lines of one plane (kSlabThreads threads).
//   phase 0  the rows (aw, ap, ae) and the right-hand side of the slab are
//            copied into shared memory (cp.async, all in flight, coalesced
//            along the fastest global index), laid out [node][line];
//   phase 1  thread (line, half) eliminates the upper half of its line
//            top-down (SGTSV's no-interchange order; a would-swap row is
//            counted in flags[0]) or the lower half bottom-up, the reciprocal
//            of the eliminated diagonal replacing ap; the halves meet in a 2x2
//            solve and back-substitute;
//   phase 2  the solution goes back to rh, or, after the k sweep, into the
//            update nu <- nu + (-nu + (nu_old + dnu)) / (1 + 1.5 dtev / dt)
//            (src/des_eddy.F90:260-272).
// Shared memory: 4 fields of slab_fs(n, NL + 1) elements of SW.
template <class SW, int DIR, int NL>
__global__ void __launch_bounds__(kSlabThreads) k_sa_sweep4(SaT<SW> S) {
  pdl_wait();
  constexpr int NT = kSlabThreads, NLP = NL + 1;
  extern __shared__ __align__(16) unsigned char sa_slab[];
  __shared__ SW m_d[NL], m_c[NL], m_b[NL], n_d[NL], n_c[NL], n_b[NL];
  __shared__ int s_ndom[NL];  // columns of the line's matrix that are not diagonally dominant
  const int tid = threadIdx.x;
  const int a0 = blockIdx.x * NL + 1;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa, base;
  if (DIR == 0) { amax = S.jm - 2; n = S.im - 2; st = 1; sa = S.sj; base = S.sk * b; }
  else if (DIR == 1) { amax = S.im - 2; n = S.jm - 2; st = S.sj; sa = 1; base = S.sk * b; }
  else { amax = S.im - 2; n = S.km - 2; st = S.sk; sa = 1; base = S.sj * b; }
  const int nl = min(NL, amax - a0 + 1);
  const int fs = slab_fs(n, NLP);  // row p (node p + 1) at p * NLP + line
  SW* s_aw = reinterpret_cast<SW*>(sa_slab);
  SW* s_ap = s_aw + fs;
  SW* s_ae = s_aw + 2 * fs;
  SW* s_rh = s_aw + 3 * fs;
  const int total = nl * n;
  auto node = [&](int t, int& li, int& p) {
    if (DIR == 0) { li = t / n; p = t - li * n; }
    else { p = t / nl; li = t - p * nl; }
    return base + (a0 + li) * sa + (p + 1) * st;
  };

  // ---- phase 0
  if (tid < NL) s_ndom[tid] = 0;
  for (int t = tid; t < total; t += NT) {
    int li, p;
    const int l = node(t, li, p);
    const int so = p * NLP + li;
    cp_async_elem(s_aw + so, S.co[3 * DIR + 0] + l);
    cp_async_elem(s_ap + so, S.co[3 * DIR + 1] + l);
    cp_async_elem(s_ae + so, S.co[3 * DIR + 2] + l);
    cp_async_elem(s_rh + so, S.rh + l);
  }
  cp_async_wait_all();
  __syncthreads();

  // ---- phase 1 (1/d replaces ap, so that back-substitution multiplies)
  const int li = tid % NL, half = tid / NL;
  const bool act = tid < 2 * NL && li < nl;  // solver threads
  const int h = n / 2;
  auto at = [&](int p) { return p * NLP + li; };
  constexpr int R = 4;  // rows read ahead of the elimination chain
  // column checks, |ap_p| >= |ae_{p-1}| + |aw_{p+1}| (no interchange under
  // partial pivoting when every column passes): the previous row's ap and the
  // ae before it (top half), or the next row's ap and the aw after it
  // (bottom half)
  int ndom = 0;
  SW apc = 0, aec2 = 0;
  if (act && half == 0) {
    SW dprev = 0, rdprev = 0, duprev = 0, bprev = 0;
    for (int p0 = 0; p0 < h; p0 += R) {
      SW baw[R], bap[R], bae[R], brr[R];
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (p0 + u < h) { baw[u] = s_aw[at(p0 + u)]; bap[u] = s_ap[at(p0 + u)]; bae[u] = s_ae[at(p0 + u)]; brr[u] = s_rh[at(p0 + u)]; }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p < h) {
          SW d;
          if (p == 0) { d = bap[u]; bprev = brr[u]; }
          else {
            ndom += dabs(apc) < dabs(aec2) + dabs(baw[u]);
            const SW f = mulw(baw[u], rdprev);
            d = fmaw(-f, duprev, bap[u]);
            bprev = fmaw(-f, bprev, brr[u]);
          }
          aec2 = duprev; apc = bap[u];
          rdprev = sweep_rcp(d);
          s_ap[at(p)] = rdprev; s_rh[at(p)] = bprev;
          dprev = d; duprev = bae[u];
        }
      }
    }
    m_d[li] = dprev; m_c[li] = duprev; m_b[li] = bprev;
  } else if (act && half == 1) {
    SW dprev = 0, rdprev = 0, awprev = 0, bprev = 0;
    for (int p0 = n - 1; p0 >= h; p0 -= R) {
      SW baw[R], bap[R], bae[R], brr[R];
#pragma unroll
      for (int u = 0; u < R; ++u)
        if (p0 - u >= h) { baw[u] = s_aw[at(p0 - u)]; bap[u] = s_ap[at(p0 - u)]; bae[u] = s_ae[at(p0 - u)]; brr[u] = s_rh[at(p0 - u)]; }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 - u;
        if (p >= h) {
          SW d;
          if (p == n - 1) { d = bap[u]; bprev = brr[u]; }
          else {
            ndom += dabs(apc) < dabs(bae[u]) + dabs(aec2);
            const SW f = mulw(bae[u], rdprev);
            d = fmaw(-f, awprev, bap[u]);
            bprev = fmaw(-f, bprev, brr[u]);
          }
          aec2 = awprev; apc = bap[u];
          rdprev = sweep_rcp(d);
          s_ap[at(p)] = rdprev; s_rh[at(p)] = bprev;
          dprev = d; awprev = baw[u];
        }
      }
    }
    n_d[li] = dprev; n_c[li] = awprev; n_b[li] = bprev;
  }
  __syncthreads();
  if (act) {
    const SW d1 = m_d[li], u1 = m_c[li], b1 = m_b[li];
    const SW d2 = n_d[li], l2 = n_c[li], b2 = n_b[li];
    const SW det = fms2(d1, d2, u1, l2);
    // the middle columns h - 1 (needs the bottom half's aw_h, l2) and h
    // (needs the top half's ae_{h-1}, u1)
    if (half == 0) ndom += dabs(apc) < dabs(aec2) + dabs(l2);
    else ndom += dabs(apc) < dabs(u1) + dabs(aec2);
    if (ndom) atomicAdd(&s_ndom[li], ndom);
    if (half == 0) {
      SW x = fms2(b1, d2, u1, b2) / det;
      s_rh[at(h - 1)] = x;
      for (int p0 = h - 2; p0 >= 0; p0 -= R) {
        SW bae[R], brr[R], brd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 - u >= 0) { bae[u] = s_ae[at(p0 - u)]; brr[u] = s_rh[at(p0 - u)]; brd[u] = s_ap[at(p0 - u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 - u >= 0) { x = mulw(fmaw(-bae[u], x, brr[u]), brd[u]); s_rh[at(p0 - u)] = x; }
      }
    } else {
      SW x = fms2(d1, b2, l2, b1) / det;
      s_rh[at(h)] = x;
      for (int p0 = h + 1; p0 < n; p0 += R) {
        SW baw[R], brr[R], brd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 + u < n) { baw[u] = s_aw[at(p0 + u)]; brr[u] = s_rh[at(p0 + u)]; brd[u] = s_ap[at(p0 + u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 + u < n) { x = mulw(fmaw(-baw[u], x, brr[u]), brd[u]); s_rh[at(p0 + u)] = x; }
      }
    }
  }
  __syncthreads();

  // ---- a line whose matrix has a column that is not dominant: solved again
  // from its original rows by SGTSV's elimination with partial pivoting
  // (src/sgtsv.f:107-162, 232-257), one thread per line, in the line's own
  // columns: ap and the right-hand side are reloaded, aw (dl, with the
  // fill-in of a swap) and ae (du) are modified in place.  Interchanges are
  // counted in flags[0], zero pivots in flags[1], the lines solved this way
  // in flags[2].
  if (tid < nl && s_ndom[tid]) {
    const int lf = tid;
    auto fat = [&](int p) { return p * NLP + lf; };
    const int l0 = base + (a0 + lf) * sa + st;   // node of row 0
    for (int p = 0; p < n; ++p) {
      s_ap[fat(p)] = S.co[3 * DIR + 1][l0 + p * st];
      s_rh[fat(p)] = S.rh[l0 + p * st];
    }
    int nsw = 0;
    bool sing = false;
    for (int i = 0; i <= n - 2 && !sing; ++i) {
      const SW dli = s_aw[fat(i + 1)];
      if (dabs(s_ap[fat(i)]) >= dabs(dli)) {
        if (s_ap[fat(i)] != SW(0)) {
          const SW fact = dli / s_ap[fat(i)];
          s_ap[fat(i + 1)] = fmaw(-fact, s_ae[fat(i)], s_ap[fat(i + 1)]);
          s_rh[fat(i + 1)] = fmaw(-fact, s_rh[fat(i)], s_rh[fat(i + 1)]);
        } else {
          sing = true;
        }
        s_aw[fat(i + 1)] = SW(0);
      } else {
        ++nsw;
        const SW fact = s_ap[fat(i)] / dli;
        s_ap[fat(i)] = dli;
        const SW temp = s_ap[fat(i + 1)];
        s_ap[fat(i + 1)] = fmaw(-fact, temp, s_ae[fat(i)]);
        if (i <= n - 3) {
          s_aw[fat(i + 1)] = s_ae[fat(i + 1)];        // du2(i), the fill-in
          s_ae[fat(i + 1)] = -fact * s_aw[fat(i + 1)];
        }
        s_ae[fat(i)] = temp;
        const SW tb = s_rh[fat(i)];
        s_rh[fat(i)] = s_rh[fat(i + 1)];
        s_rh[fat(i + 1)] = fmaw(-fact, s_rh[fat(i + 1)], tb);
      }
    }
    if (sing || s_ap[fat(n - 1)] == SW(0)) {
      atomicAdd(&S.flags[1], 1);
    } else {
      s_rh[fat(n - 1)] = s_rh[fat(n - 1)] / s_ap[fat(n - 1)];
      if (n > 1) s_rh[fat(n - 2)] = fmaw(-s_ae[fat(n - 2)], s_rh[fat(n - 1)], s_rh[fat(n - 2)]) / s_ap[fat(n - 2)];
      for (int i = n - 3; i >= 0; --i)
        s_rh[fat(i)] = fmaw(-s_aw[fat(i + 1)], s_rh[fat(i + 2)], fmaw(-s_ae[fat(i)], s_rh[fat(i + 1)], s_rh[fat(i)])) / s_ap[fat(i)];
    }
    if (nsw) atomicAdd(&S.flags[0], nsw);
    atomicAdd(&S.flags[2], 1);
  }
  __syncthreads();

  // ---- phase 2
  if (DIR < 2) {
    for (int t = tid; t < total; t += NT) {
      int lq, p;
      const int l = node(t, lq, p);
      S.rh[l] = s_rh[p * NLP + lq];
    }
  } else {
    const double dmul = 1.5 * S.es;
    constexpr int U = 4;
    for (int t0 = tid; t0 < total; t0 += NT * U) {
      int ln[U], so[U];
      double nt[U], dt[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int t = t0 + u * NT;
        ln[u] = -1;
        so[u] = 0;
        if (t < total) {
          int lq, p;
          ln[u] = node(t, lq, p);
          so[u] = p * NLP + lq;
          nt[u] = S.upd[ln[u]];
          dt[u] = __ldg(S.dtev + ln[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (ln[u] < 0) continue;
        const double qe5 = nt[u] + double(s_rh[so[u]]);
        const double dum = 1.0 + dmul * dt[u] / S.delti;
        S.upd[ln[u]] = nt[u] + (-nt[u] + qe5) / dum;
      }
    }
  }
}

// A second scalar solved in the same launch as S (blockIdx.z = 1): the
// rows of the sweep's direction, the right-hand side and the field the k
// sweep updates (k-omega's omega beside k: the two line solves share
// nothing, and one launch puts twice the lines in flight).
template <class SW>
struct SaPair {
  const SW* co[3];
  SW* rh;
  double* upd;
};

// The same scalar ADI sweep with the lines in the lanes: a warp owns 32
// neighbouring lines of one plane and one half of each, a CTA 2 x 32 lines
// (four warps).  The rows are read from global memory as the elimination
// proceeds (rows of the j and k sweeps are coalesced across the lanes; the
// i sweep's through L1 sectors), and the eliminated row of each node
// (1/d, b') goes to a scratch laid out [row][line], coalesced across the
// lanes, from which the back-substitution reads it.  No slab is staged, so
// occupancy is set by registers alone and every line runs at once instead of
// a few per SM.  The elimination is k_sa_sweep4's: the same operations in
// the same order (two-ended, no interchange where every column is
// diagonally dominant, SGTSV's pivoting elimination otherwise), so the two
// kernels give the same values.  The back-substitution drops the scratch rows
// it has read from L2 without write-back (lines of a plane padded to a
// multiple of 32: a warp's row is one 128-byte line, two in FP64), unless a
// lane of the warp takes the pivoting path, which reuses them.
// Scratch (S.gs, arrays S.gss apart): 1/d, b', and for the pivoting
// elimination du and dl (arrays 4..7 for the second scalar); row p of line
// (a, b) at p nln + (a - 1) + amaxp (b - 1), amaxp = amax rounded up to 32.
// Build-time tuning knobs of k_sa_gsweep (as for k_gsweep).
#ifndef DESALM_SAGS_MINBLOCKS
#define DESALM_SAGS_MINBLOCKS 4
#endif
#ifndef DESALM_SAGS_ROWS
#define DESALM_SAGS_ROWS 8
#endif
template <class SW, int DIR>
__global__ void __launch_bounds__(128, DESALM_SAGS_MINBLOCKS) k_sa_gsweep(SaT<SW> S, SaPair<SW> B) {
  pdl_wait();
  constexpr int LG = 2;                       // line groups of 32 per CTA
  constexpr int R = sizeof(SW) == 4 ? DESALM_SAGS_ROWS : DESALM_SAGS_ROWS / 2;  // rows loaded one block ahead
  __shared__ SW m_d[LG][32], m_c[LG][32], m_b[LG][32], n_d[LG][32], n_c[LG][32], n_b[LG][32];
  __shared__ int s_ndom[LG][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = w >> 1, half = w & 1;
  const int b = blockIdx.y + 1;
  int amax, n, st, sa, base;
  if (DIR == 0) { amax = S.jm - 2; n = S.im - 2; st = 1; sa = S.sj; base = S.sk * b; }
  else if (DIR == 1) { amax = S.im - 2; n = S.jm - 2; st = S.sj; sa = 1; base = S.sk * b; }
  else { amax = S.im - 2; n = S.km - 2; st = S.sk; sa = 1; base = S.sj * b; }
  const int a = blockIdx.x * (32 * LG) + g * 32 + lane + 1;
  const bool act = a <= amax;
  const int amaxp = (amax + 31) & ~31;
  const int nln = amaxp * (int)gridDim.y;           // padded lines of the sweep
  const int line = (a - 1) + amaxp * (b - 1);
  const int line0 = line - lane;                    // the warp's first line
  const unsigned wact = __ballot_sync(0xffffffffu, act);
  const int l0 = base + a * sa + st;                 // node of row 0
  // blockIdx.z = 1: the second scalar of B (its rows, right-hand side,
  // field and scratch arrays 4..7)
  const bool second = blockIdx.z == 1;
  const SW* __restrict__ caw = second ? B.co[0] : S.co[3 * DIR + 0];
  const SW* __restrict__ cap = second ? B.co[1] : S.co[3 * DIR + 1];
  const SW* __restrict__ cae = second ? B.co[2] : S.co[3 * DIR + 2];
  SW* __restrict__ rhs = second ? B.rh : S.rh;
  double* __restrict__ upd = second ? B.upd : S.upd;
  SW* __restrict__ gs = S.gs + (second ? 4 * (size_t)S.gss : 0);
  SW* __restrict__ gd = gs;
  SW* __restrict__ gb = gs + S.gss;
  auto sc = [&](int p) { return p * nln + line; };
  if (half == 0) s_ndom[g][lane] = 0;
  const int h = n / 2;
  int ndom = 0;
  SW apc = 0, aec2 = 0;
  if (act && half == 0) {
    SW dprev = 0, rdprev = 0, duprev = 0, bprev = 0;
    SW caw_[R], cap_[R], cae_[R], crr_[R];
#pragma unroll
    for (int u = 0; u < R; ++u)
      if (u < h) { const int l = l0 + u * st; caw_[u] = __ldg(caw + l); cap_[u] = __ldg(cap + l); cae_[u] = __ldg(cae + l); crr_[u] = rhs[l]; }
    for (int p0 = 0; p0 < h; p0 += R) {
      SW naw[R], nap[R], nae[R], nrr[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        naw[u] = nap[u] = nae[u] = nrr[u] = SW(0);
        if (p0 + R + u < h) { const int l = l0 + (p0 + R + u) * st; naw[u] = __ldg(caw + l); nap[u] = __ldg(cap + l); nae[u] = __ldg(cae + l); nrr[u] = rhs[l]; }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 + u;
        if (p < h) {
          SW d;
          if (p == 0) { d = cap_[u]; bprev = crr_[u]; }
          else {
            ndom += dabs(apc) < dabs(aec2) + dabs(caw_[u]);
            const SW f = mulw(caw_[u], rdprev);
            d = fmaw(-f, duprev, cap_[u]);
            bprev = fmaw(-f, bprev, crr_[u]);
          }
          aec2 = duprev; apc = cap_[u];
          rdprev = sweep_rcp(d);
          gd[sc(p)] = rdprev; gb[sc(p)] = bprev;
          dprev = d; duprev = cae_[u];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) { caw_[u] = naw[u]; cap_[u] = nap[u]; cae_[u] = nae[u]; crr_[u] = nrr[u]; }
    }
    m_d[g][lane] = dprev; m_c[g][lane] = duprev; m_b[g][lane] = bprev;
  } else if (act && half == 1) {
    SW dprev = 0, rdprev = 0, awprev = 0, bprev = 0;
    SW caw_[R], cap_[R], cae_[R], crr_[R];
#pragma unroll
    for (int u = 0; u < R; ++u)
      if (n - 1 - u >= h) { const int l = l0 + (n - 1 - u) * st; caw_[u] = __ldg(caw + l); cap_[u] = __ldg(cap + l); cae_[u] = __ldg(cae + l); crr_[u] = rhs[l]; }
    for (int p0 = n - 1; p0 >= h; p0 -= R) {
      SW naw[R], nap[R], nae[R], nrr[R];
#pragma unroll
      for (int u = 0; u < R; ++u) {
        naw[u] = nap[u] = nae[u] = nrr[u] = SW(0);
        if (p0 - R - u >= h) { const int l = l0 + (p0 - R - u) * st; naw[u] = __ldg(caw + l); nap[u] = __ldg(cap + l); nae[u] = __ldg(cae + l); nrr[u] = rhs[l]; }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) {
        const int p = p0 - u;
        if (p >= h) {
          SW d;
          if (p == n - 1) { d = cap_[u]; bprev = crr_[u]; }
          else {
            ndom += dabs(apc) < dabs(cae_[u]) + dabs(aec2);
            const SW f = mulw(cae_[u], rdprev);
            d = fmaw(-f, awprev, cap_[u]);
            bprev = fmaw(-f, bprev, crr_[u]);
          }
          aec2 = awprev; apc = cap_[u];
          rdprev = sweep_rcp(d);
          gd[sc(p)] = rdprev; gb[sc(p)] = bprev;
          dprev = d; awprev = caw_[u];
        }
      }
#pragma unroll
      for (int u = 0; u < R; ++u) { caw_[u] = naw[u]; cap_[u] = nap[u]; cae_[u] = nae[u]; crr_[u] = nrr[u]; }
    }
    n_d[g][lane] = dprev; n_c[g][lane] = awprev; n_b[g][lane] = bprev;
  }
  __syncthreads();
  SW d1 = 0, u1 = 0, b1 = 0, d2 = 0, l2 = 0, b2 = 0, det = 0;
  if (act) {
    d1 = m_d[g][lane]; u1 = m_c[g][lane]; b1 = m_b[g][lane];
    d2 = n_d[g][lane]; l2 = n_c[g][lane]; b2 = n_b[g][lane];
    det = fms2(d1, d2, u1, l2);
    if (half == 0) ndom += dabs(apc) < dabs(aec2) + dabs(l2);
    else ndom += dabs(apc) < dabs(u1) + dabs(aec2);
    if (ndom) atomicAdd(&s_ndom[g][lane], ndom);
  }
  __syncthreads();
  const bool wdisc = __all_sync(0xffffffffu, !act || !s_ndom[g][lane]);
  if (!act) return;
  // rows pb, pb + dir, ... (R of them, those in [lo, hi]) of the warp's 32
  // lines read for the last time: lane t < 2 R SEG drops one 128-byte line
  auto drop = [&](int pb, int dir, int lo, int hi) {
    if (!wdisc) return;
    __syncwarp(wact);
    constexpr int SEG = 32 * (int)sizeof(SW) / 128;
    static_assert(R * 2 * SEG <= 32, "one 128-byte line per lane");
    if (lane < R * 2 * SEG) {
      const int u = lane / (2 * SEG), col = (lane / SEG) & 1, piece = lane % SEG;
      const int p = pb + dir * u;
      if (p >= lo && p <= hi) l2_discard((col ? gd : gb) + p * nln + line0 + piece * (128 / (int)sizeof(SW)));
    }
  };
  const double dmul = 1.5 * S.es;
  // the solution of row p: into rh, or after the k sweep into the update
  // nu <- nu + (-nu + (nu_old + dnu)) / (1 + 1.5 dtev / dt)
  auto put = [&](int p, SW x) {
    const int l = l0 + p * st;
    if (DIR < 2) {
      rhs[l] = x;
    } else {
      const double nt = upd[l];
      const double qe5 = nt + double(x);
      const double dum = 1.0 + dmul * __ldg(S.dtev + l) / S.delti;
      upd[l] = nt + (-nt + qe5) / dum;
    }
  };
  if (!s_ndom[g][lane]) {
    if (half == 0) {
      SW x = fms2(b1, d2, u1, b2) / det;
      put(h - 1, x);
      drop(h - 1, 1, h - 1, h - 1);     // the middle row is not read back
      for (int p0 = h - 2; p0 >= 0; p0 -= R) {
        SW bae[R], brr[R], brd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 - u >= 0) { bae[u] = __ldg(cae + l0 + (p0 - u) * st); brr[u] = gb[sc(p0 - u)]; brd[u] = gd[sc(p0 - u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 - u >= 0) { x = mulw(fmaw(-bae[u], x, brr[u]), brd[u]); put(p0 - u, x); }
        drop(p0, -1, 0, h - 2);
      }
    } else {
      SW x = fms2(d1, b2, l2, b1) / det;
      put(h, x);
      drop(h, 1, h, h);
      for (int p0 = h + 1; p0 < n; p0 += R) {
        SW baw[R], brr[R], brd[R];
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 + u < n) { baw[u] = __ldg(caw + l0 + (p0 + u) * st); brr[u] = gb[sc(p0 + u)]; brd[u] = gd[sc(p0 + u)]; }
#pragma unroll
        for (int u = 0; u < R; ++u)
          if (p0 + u < n) { x = mulw(fmaw(-baw[u], x, brr[u]), brd[u]); put(p0 + u, x); }
        drop(p0, 1, h + 1, n - 1);
      }
    }
    return;
  }
  if (half != 0) return;
  // ---- a line with a column that is not dominant: SGTSV's elimination with
  // partial pivoting (src/sgtsv.f:107-162, 232-257) from the original rows,
  // in the line's scratch: d (gd), b (gb), du (gu) and dl (gl, with the
  // fill-in of a swap)
  SW* __restrict__ gu = gs + 2 * (size_t)S.gss;
  SW* __restrict__ gl = gs + 3 * (size_t)S.gss;
  for (int p = 0; p < n; ++p) {
    const int l = l0 + p * st;
    gd[sc(p)] = cap[l];
    gb[sc(p)] = rhs[l];
    gu[sc(p)] = cae[l];
    gl[sc(p)] = caw[l];
  }
  int nsw = 0;
  bool sing = false;
  for (int i = 0; i <= n - 2 && !sing; ++i) {
    const SW dli = gl[sc(i + 1)];
    const SW di = gd[sc(i)];
    if (dabs(di) >= dabs(dli)) {
      if (di != SW(0)) {
        const SW fact = dli / di;
        gd[sc(i + 1)] = fmaw(-fact, gu[sc(i)], gd[sc(i + 1)]);
        gb[sc(i + 1)] = fmaw(-fact, gb[sc(i)], gb[sc(i + 1)]);
      } else {
        sing = true;
      }
      gl[sc(i + 1)] = SW(0);
    } else {
      ++nsw;
      const SW fact = di / dli;
      gd[sc(i)] = dli;
      const SW temp = gd[sc(i + 1)];
      gd[sc(i + 1)] = fmaw(-fact, temp, gu[sc(i)]);
      if (i <= n - 3) {
        gl[sc(i + 1)] = gu[sc(i + 1)];               // du2(i), the fill-in
        gu[sc(i + 1)] = -fact * gl[sc(i + 1)];
      }
      gu[sc(i)] = temp;
      const SW tb = gb[sc(i)];
      gb[sc(i)] = gb[sc(i + 1)];
      gb[sc(i + 1)] = fmaw(-fact, gb[sc(i + 1)], tb);
    }
  }
  if (sing || gd[sc(n - 1)] == SW(0)) {
    atomicAdd(&S.flags[1], 1);
  } else {
    gb[sc(n - 1)] = gb[sc(n - 1)] / gd[sc(n - 1)];
    if (n > 1) gb[sc(n - 2)] = fmaw(-gu[sc(n - 2)], gb[sc(n - 1)], gb[sc(n - 2)]) / gd[sc(n - 2)];
    for (int i = n - 3; i >= 0; --i)
      gb[sc(i)] = fmaw(-gl[sc(i + 1)], gb[sc(i + 2)], fmaw(-gu[sc(i)], gb[sc(i + 1)], gb[sc(i)])) / gd[sc(i)];
    for (int p = 0; p < n; ++p) put(p, gb[sc(p)]);
  }
  if (nsw) atomicAdd(&S.flags[0], nsw);
  atomicAdd(&S.flags[2], 1);
}

// boundary values of nu_tilde (src/rhs_sa_bcond.F90:40-269): one kernel per
// face pair in the order i, j, k; full transverse ranges.
template <class SW, int DIR>
__global__ void k_sa_bc(SaT<SW> S) {
  pdl_wait();
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  int amax, n, st, lb;
  if (DIR == 0) { amax = S.jm; n = S.im; st = 1; lb = S.sj * a + S.sk * b; }
  else if (DIR == 1) { amax = S.im; n = S.jm; st = S.sj; lb = a + S.sk * b; }
  else { amax = S.im; n = S.km; st = S.sk; lb = a + S.sj * b; }
  if (a >= amax) return;
  double* q5 = S.q[4];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int bi = 2 * DIR + side;
    const int bt = S.btype[bi];
    const int l = side == 0 ? lb : lb + (n - 1) * st;
    const int s = side == 0 ? st : -st;
    if (bt == 1) q5[l] = 0.0;
    else if (bt == 2 || bt == 3) q5[l] = S.sa1[bi] * q5[l + s] + S.sb1[bi] * q5[l + 2 * s];
    else if (bt == 5) {
      const double r = S.rat[(size_t)bi * S.ratdim * S.ratdim + a + (size_t)S.ratdim * b];
      q5[l] = (1.0 + r) * q5[l + s] - r * q5[l + 2 * s];
    } else if (bt == 6) q5[l] = side == 0 ? q5[lb + (n - 2) * st] : q5[lb + st];
    else if (bt == 8 && DIR == 0 && side == 1) q5[l] = q5[l - 1];
  }
}

// nu_tilde >= 1e-7 and nu_t = nu_tilde f_v1 on every node (src/rhs_sa_bcond.F90:279-291)
template <class SW>
__global__ void k_sa_clamp(SaT<SW> S) {
  pdl_wait();
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= S.N) return;
  double v = S.q[4][l];
  v = v > 1.0E-07 ? v : 1.0E-07;
  S.q[4][l] = v;
  double chi = v / (1.0 / S.ren);
  double chic = chi * chi * chi;
  S.nut[l] = v * (chic / (chic + 357.911));
}

// ---------------------------------------------------------------- conservation
// Sums of U/J over the first and last i planes (all j, k), into acc[0..1].
__global__ void k_cons_sum(Sa S, double* acc) {
  pdl_wait();
  __shared__ double sh[2][256];
  double a0 = 0, a1 = 0;
  const int P = S.jm * S.km;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < P; t += gridDim.x * blockDim.x) {
    const int j = t % S.jm, k = t / S.jm;
    a0 += sa_ucn(S, 0, S.sj * j + S.sk * k);
    a1 += sa_ucn(S, 0, (S.im - 1) + S.sj * j + S.sk * k);
  }
  sh[0][threadIdx.x] = a0;
  sh[1][threadIdx.x] = a1;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) { sh[0][threadIdx.x] += sh[0][threadIdx.x + s]; sh[1][threadIdx.x] += sh[1][threadIdx.x + s]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) { acc[0] = sh[0][0]; acc[1] = sh[1][0]; }
}

// Rescale the outlet plane's U/J by fin/fout and return to Cartesian
// velocities with the covariant metrics (src/conservation.F90:137-157).
__global__ void k_cons_apply(Sa S, const double* acc, double* const* cov) {
  pdl_wait();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= S.jm * S.km) return;
  const int j = t % S.jm, k = t / S.jm;
  const int l = (S.im - 1) + S.sj * j + S.sk * k;
  const double fin = acc[0], fout = acc[1];
  const double delta_e = fin - fout;
  double u1 = sa_ucn(S, 0, l), u2 = sa_ucn(S, 1, l), u3 = sa_ucn(S, 2, l);
  u1 = u1 + delta_e * u1 / fout;
  const double a = S.aj[l];
  S.q[1][l] = a * (u1 * cov[0][l] + u2 * cov[1][l] + u3 * cov[2][l]);
  S.q[2][l] = a * (u1 * cov[3][l] + u2 * cov[4][l] + u3 * cov[5][l]);
  S.q[3][l] = a * (u1 * cov[6][l] + u2 * cov[7][l] + u3 * cov[8][l]);
}

}  // namespace desalm
