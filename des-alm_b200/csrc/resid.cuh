// resid.cuh -- K_R: the momentum/continuity residual of one level, fused.
//
// One thread per interior node computes, in registers:
//   U/J at the neighbours            src/rhs_contra_j.F90:14-29
//   viscous face fluxes and visc     src/rhs_viscous.F90:103-329
//   pressure dissipation diss(1)     src/rhs_diss_p.F90:33-203   (first pass)
//   pressure gradient + divergence   src/rhs_flux_sans_convec.F90:44-136
//   QUICK / first-order convection   src/rhs_convec_quick.F90:53-425
//   BDF2 + assembly                  src/rhs_unst_visc_diss.F90:35-50
//   FAS forcing (coarse levels)      src/rhs_pk.F90:35-67
// and then either stores the raw residual (recalculation pass,
// src/solver_daf.F90:432-477) or applies r = S (-dtau J rh) and r <- Ma^-1 r
// (src/rhs_diag_solver.F90:53-122) and stores the transformed residual for
// the line sweeps, with sigma and the row coefficients of every direction.
// Divisions by J are multiplications by the stored 1/J, and the BDF2 and
// alpha denominators are inverted once per node; the results equal the
// reference's expressions up to rounding.
#pragma once
#include "modal.cuh"

namespace desalm {

// U/J of direction d at node l
template <class T, class W>
DESALM_DEV T ucn(const Lv<T, W>& L, int d, int l) {
  const T* const* m = d == 0 ? L.csi : (d == 1 ? L.eta : L.zet);
  T tmp = L.rj[l];
  return tmp * (m[0][l] * L.q[1][l] + m[1][l] * L.q[2][l] + m[2][l] * L.q[3][l]);
}

// Viscous flux through the face between l0 and l0 + st[dir]
// (src/rhs_viscous.F90:112-163 for dir 0, :189-240 dir 1, :263-313 dir 2).
template <class T, class W>
DESALM_DEV void visc_face(const Lv<T, W>& L, int dir, int l0, T rei, T out[3]) {
  const int sj = L.sj, sk = L.sk;
  const T dc = L.dc, de = L.de, dz = L.dz;
  const T q4 = T(0.25);
  int l1;
  T U[3], E[3], Z[3];
  if (dir == 0) {
    l1 = l0 + 1;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const T* v = L.q[m + 1];
      U[m] = dc * (v[l1] - v[l0]);
      E[m] = (q4 * de) * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
      Z[m] = (q4 * dz) * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
    }
  } else if (dir == 1) {
    l1 = l0 + sj;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const T* v = L.q[m + 1];
      U[m] = (q4 * dc) * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
      E[m] = de * (v[l1] - v[l0]);
      Z[m] = (q4 * dz) * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
    }
  } else {
    l1 = l0 + sk;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const T* v = L.q[m + 1];
      U[m] = (q4 * dc) * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
      E[m] = (q4 * de) * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
      Z[m] = dz * (v[l1] - v[l0]);
    }
  }
  T a1 = L.csi[0][l1] + L.csi[0][l0], a2 = L.csi[1][l1] + L.csi[1][l0], a3 = L.csi[2][l1] + L.csi[2][l0];
  T b1 = L.eta[0][l1] + L.eta[0][l0], b2 = L.eta[1][l1] + L.eta[1][l0], b3 = L.eta[2][l1] + L.eta[2][l0];
  T c1 = L.zet[0][l1] + L.zet[0][l0], c2 = L.zet[1][l1] + L.zet[1][l0], c3 = L.zet[2][l1] + L.zet[2][l0];
  T uu1 = a1 * U[0] + b1 * E[0] + c1 * Z[0], vv1 = a1 * U[1] + b1 * E[1] + c1 * Z[1], ww1 = a1 * U[2] + b1 * E[2] + c1 * Z[2];
  T uu2 = a2 * U[0] + b2 * E[0] + c2 * Z[0], vv2 = a2 * U[1] + b2 * E[1] + c2 * Z[1], ww2 = a2 * U[2] + b2 * E[2] + c2 * Z[2];
  T uu3 = a3 * U[0] + b3 * E[0] + c3 * Z[0], vv3 = a3 * U[1] + b3 * E[1] + c3 * Z[1], ww3 = a3 * U[2] + b3 * E[2] + c3 * Z[2];
  T n1, n2, n3, k1, k2, k3;
  if (dir == 0) {
    n1 = a1; n2 = a2; n3 = a3;
    k1 = a1 * a1 + a2 * a2 + a3 * a3; k2 = a1 * b1 + a2 * b2 + a3 * b3; k3 = a1 * c1 + a2 * c2 + a3 * c3;
  } else if (dir == 1) {
    n1 = b1; n2 = b2; n3 = b3;
    k1 = b1 * a1 + b2 * a2 + b3 * a3; k2 = b1 * b1 + b2 * b2 + b3 * b3; k3 = b1 * c1 + b2 * c2 + b3 * c3;
  } else {
    n1 = c1; n2 = c2; n3 = c3;
    k1 = c1 * a1 + c2 * a2 + c3 * a3; k2 = c1 * b1 + c2 * b2 + c3 * b3; k3 = c1 * c1 + c2 * c2 + c3 * c3;
  }
  T vtj = T(0.25) * ((rei + L.nut[l1]) + (rei + L.nut[l0])) / (L.aj[l1] + L.aj[l0]);
  // the flux is rounded here (mulw), so a node's difference of its two face
  // fluxes is the same whether the faces were formed in registers (k_resid)
  // or came from shared memory (k_resid_f)
  out[0] = mulw(vtj, n1 * uu1 + n2 * vv1 + n3 * ww1 + k1 * U[0] + k2 * E[0] + k3 * Z[0]);
  out[1] = mulw(vtj, n1 * uu2 + n2 * vv2 + n3 * ww2 + k1 * U[1] + k2 * E[1] + k3 * Z[1]);
  out[2] = mulw(vtj, n1 * uu3 + n2 * vv3 + n3 * ww3 + k1 * U[2] + k2 * E[2] + k3 * Z[2]);
}

// Second difference of the pressure scaled by g_dd dtau / J at node l
// (src/rhs_diss_p.F90:58-117).
template <class T, class W>
DESALM_DEV T diss_fv(const Lv<T, W>& L, int dir, int l, int st, T dsq) {
  const T* const* m = dir == 0 ? L.csi : (dir == 1 ? L.eta : L.zet);
  T g = m[0][l] * m[0][l] + m[1][l] * m[1][l] + m[2][l] * m[2][l];
  T tmp1 = g * L.dtau[l] * L.rj[l];
  const T* p = L.q[0];
  T tmp2 = dsq * (p[l + st] - T(2) * p[l] + p[l - st]);
  return tmp1 * tmp2;
}

// Minimum resident CTAs per SM requested from the register allocator for
// K_R (128 threads each); a build-time tuning knob.
#ifndef DESALM_KR_MINBLOCKS
#define DESALM_KR_MINBLOCKS 3
#endif
// CTA shape of K_R and of the SA residual (i extent 32; j x k = 4), another
// build-time knob: j rows and k planes per CTA.
#ifndef DESALM_KR_BY
#define DESALM_KR_BY 4
#endif
#define DESALM_KR_BZ (4 / DESALM_KR_BY)

// k planes a thread of K_R takes in turn (the CTA tile's k extent apart), so
// that the neighbour planes it has just read are still in L1 for the next;
// a build-time tuning knob.
#ifndef DESALM_KR_KLOOP
#define DESALM_KR_KLOOP 2
#endif

// The residual of interior node (i, j, k); MODE 0: first pass of a DAF step;
// MODE 1: recalculation for restriction.
// VGIVEN: the viscous terms come in vg (k_resid_f forms them from face
// fluxes computed once per face).
template <class T, class W, int MODE, bool VGIVEN = false>
DESALM_DEV void resid_node(const Lv<T, W>& L, const Par& P, int upwind, int calc_pk, int coarse, int bback, int i, int j, int k,
                           const T* vg = nullptr) {
  const int sj = L.sj, sk = L.sk;
  const int l = i + sj * j + sk * k;
  const T rei = T(1) / T(P.ren);
  const T dsp[3] = {L.dc, L.de, L.dz};
  const int st[3] = {1, sj, sk};
  const int pos[3] = {i, j, k};
  const int ext[3] = {L.im, L.jm, L.km};

  // ---- viscous terms
  T visc[3];
  if constexpr (VGIVEN) {
#pragma unroll
    for (int m = 0; m < 3; ++m) visc[m] = vg[m];
  } else {
    T fp[3], fm[3];
    visc_face(L, 0, l, rei, fp);
    visc_face(L, 0, l - 1, rei, fm);
#pragma unroll
    for (int m = 0; m < 3; ++m) visc[m] = mulw(L.dc, fp[m] - fm[m]);
    visc_face(L, 1, l, rei, fp);
    visc_face(L, 1, l - sj, rei, fm);
#pragma unroll
    for (int m = 0; m < 3; ++m) visc[m] = fmaw(L.de, fp[m] - fm[m], visc[m]);
    visc_face(L, 2, l, rei, fp);
    visc_face(L, 2, l - sk, rei, fm);
#pragma unroll
    for (int m = 0; m < 3; ++m) visc[m] = fmaw(L.dz, fp[m] - fm[m], visc[m]);
  }

  // ---- pressure dissipation (first pass only; the recalculation reuses it)
  T diss1;
  if (MODE == 0) {
    T acc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T dsq = dsp[d] * dsp[d];
      const int s = st[d];
      // boundary copies fv(1) = fv(2), fv(m) = fv(m-1) (src/rhs_diss_p.F90:124-129)
      T f0 = diss_fv(L, d, l, s, dsq);
      T fmi = pos[d] - 1 == 0 ? f0 : diss_fv(L, d, l - s, s, dsq);
      T fpl = pos[d] + 1 == ext[d] - 1 ? f0 : diss_fv(L, d, l + s, s, dsq);
      acc[d] = fpl - T(2) * f0 + fmi;
    }
    diss1 = T(P.pdiss) * (acc[0] + acc[1] + acc[2]);
  } else {
    diss1 = L.diss1[l];
  }

  // ---- pressure gradient and divergence
  T rh[4];
  {
    const T* p = L.q[0];
    const T dh[3] = {T(0.5) * L.dc, T(0.5) * L.de, T(0.5) * L.dz};
    const T* const* mt[3] = {L.csi, L.eta, L.zet};
    T pp[3], pm[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      pp[d] = p[l + st[d]] * L.rj[l + st[d]];
      pm[d] = p[l - st[d]] * L.rj[l - st[d]];
    }
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      T v = dh[0] * (pp[0] * mt[0][x][l + 1] - pm[0] * mt[0][x][l - 1]);
      v = v + dh[1] * (pp[1] * mt[1][x][l + sj] - pm[1] * mt[1][x][l - sj]);
      v = v + dh[2] * (pp[2] * mt[2][x][l + sk] - pm[2] * mt[2][x][l - sk]);
      rh[x + 1] = v;
    }
    T dudx = dh[0] * (ucn(L, 0, l + 1) - ucn(L, 0, l - 1));
    T dvdy = dh[1] * (ucn(L, 1, l + sj) - ucn(L, 1, l - sj));
    T dwdz = dh[2] * (ucn(L, 2, l + sk) - ucn(L, 2, l - sk));
    rh[0] = dudx + dvdy + dwdz;
  }

  // ---- convection
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int s = st[d];
    const T h = dsp[d];
    T ucon = T(0.5) * ucn(L, d, l);
    T up = ucon + dabs(ucon), um = ucon - dabs(ucon);
    bool first = (upwind == 1) || pos[d] == 1 || pos[d] == ext[d] - 2;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const T* v = L.q[m + 1];
      T f;
      if (first) {
        f = h * (up * (v[l] - v[l - s]) + um * (v[l + s] - v[l]));
      } else {
        f = T(0.125) * h * (up * (T(3) * v[l + s] + T(3) * v[l] - T(7) * v[l - s] + v[l - 2 * s]) +
                            um * (-T(3) * v[l - s] - T(3) * v[l] + T(7) * v[l + s] - v[l + 2 * s]));
      }
      rh[m + 1] = rh[m + 1] + f;
    }
  }

  // ---- unsteady terms, viscous and dissipation
  {
    const T rdtaj = T(1) / (T(2) * T(P.delti) * L.aj[l]);
    rh[0] = rh[0] + diss1;
#pragma unroll
    for (int m = 1; m < 4; ++m) {
      T dq = T(P.es) * (T(3) * L.q[m][l] - T(4) * L.qn[m][l] + L.qnm1[m][l]) * rdtaj;
      rh[m] = rh[m] + T(0) + dq - visc[m - 1];
    }
  }

  // ---- FAS forcing on coarse levels
  T pkn[4];
  if (coarse) {
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      T pk = L.pk[m][l];
      if (MODE == 0 && calc_pk) pk = pk - rh[m];
      pkn[m] = pk;
      rh[m] = rh[m] + pk;
    }
  }

  // actuator-line forcing, first pass only (src/solver_daf.F90:378-381)
  if (MODE == 0 && L.falm) {
    rh[1] = rh[1] + L.falm[l];
    rh[2] = rh[2] + L.falm[L.N + l];
    rh[3] = rh[3] + L.falm[2 * L.N + l];
  }

  if (MODE == 1) {
#pragma unroll
    for (int m = 0; m < 4; ++m) L.rh[m][l] = rh[m];
    return;
  }
  // Every store of the first pass is issued after the last load, so that no
  // store can force a metric or state value to be read again.

  // ---- r = S (-dtau rh J), then Ma^-1 r
  const T dtau = L.dtau[l];
  // sigma and theta of src/rhs_modal_matrices.F90:82-84 with one division
  const T alpha = T(1) + (T(P.es) * T(1.5) / T(P.delti)) * dtau;
  const T ra = T(1) / alpha;
  const T sg = sqrt(T(P.beta) * alpha), th = sqrt(T(P.beta) * ra);
  T s[4] = {T(P.beta), ra, ra, ra};
  T r[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) r[m] = s[m] * (-dtau * rh[m] * L.aj[l]);
  W rp[4];
  {
    // Ma^-1 in the sweep precision W (the preconditioner's precision)
    W rw[4] = {W(r[0]), W(r[1]), W(r[2]), W(r[3])};
    minv_apply<W>(W(L.csi[0][l]), W(L.csi[1][l]), W(L.csi[2][l]), W(sg), rw, rp);
  }

  // ---- line-sweep coefficients of every direction (src/rhs_diag_solver.F90:
  // 159-181): tmp = dtau ep spr dsq for the node's own row, and
  // h = dtau (dxi/2) spr, which the neighbouring rows multiply by lambda.
  // The boundary nodes before/after each line get their h too.
  const T* const* mt[3] = {L.csi, L.eta, L.zet};
  W tcv[3], hcv[3], hcb[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const T* const* m3 = mt[d];
    T g = m3[0][l] * m3[0][l] + m3[1][l] * m3[1][l] + m3[2][l] * m3[2][l];
    T spr = th * sqrt(g);
    T dq = dsp[d] * dsp[d];
    T dh = T(0.5) * dsp[d];
    tcv[d] = W(dtau * T(P.ep1[d]) * spr * dq);
    hcv[d] = W(dtau * dh * spr);
    hcb[d] = W(0);
    if (pos[d] == 1 || pos[d] == ext[d] - 2) {
      const int lb = pos[d] == 1 ? l - st[d] : l + st[d];
      T s2, t2;
      sigma_theta(L.dtau[lb], P, s2, t2);
      T g2 = m3[0][lb] * m3[0][lb] + m3[1][lb] * m3[1][lb] + m3[2][lb] * m3[2][lb];
      hcb[d] = W(L.dtau[lb] * dh * (t2 * sqrt(g2)));
    }
  }

  // ---- stores
  if (MODE == 0) L.diss1[l] = diss1;
  if (coarse && calc_pk) {
#pragma unroll
    for (int m = 0; m < 4; ++m) L.pk[m][l] = pkn[m];
  }
  if (bback && (i == 1 || i == 2)) {
    W* b = L.bi + (i - 1) * 4 * (L.jm * L.km);
    const int o = j + L.jm * k;
#pragma unroll
    for (int m = 0; m < 4; ++m) b[m * (L.jm * L.km) + o] = W(r[m]);
  }
#pragma unroll
  for (int m = 0; m < 4; ++m) L.wk[m][l] = rp[m];
  L.sig[l] = W(sg);
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    L.tc[d][l] = tcv[d];
    L.hc[d][l] = hcv[d];
    if (pos[d] == 1 || pos[d] == ext[d] - 2) L.hc[d][pos[d] == 1 ? l - st[d] : l + st[d]] = hcb[d];
  }
}

template <class T, class W, int MODE>
__global__ void __launch_bounds__(128, DESALM_KR_MINBLOCKS) k_resid(Lv<T, W> L, Par P, int upwind, int calc_pk, int coarse, int bback) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > L.im - 2 || j > L.jm - 2) return;
#pragma unroll 1
  for (int kk = 0; kk < DESALM_KR_KLOOP; ++kk) {
    const int k = (blockIdx.z * DESALM_KR_KLOOP + kk) * blockDim.z + threadIdx.z + 1;
    if (k > L.km - 2) return;
    resid_node<T, W, MODE>(L, P, upwind, calc_pk, coarse, bback, i, j, k);
  }
}

// K_R with every viscous face flux formed once (k_resid forms each twice,
// once for each of its nodes): a CTA of 32 x 4 x 2 threads covers 31 x 4 x 2
// nodes.  Phase 1: lane L of row y, plane z forms the i face between nodes
// i0 + L - 1 and i0 + L, and the tile's j faces (5 rows of 31, both planes)
// and k faces (3 planes of 4 x 31) are shared out over all threads, their
// three momentum fluxes into shared memory (component-major).  Phase 2:
// thread (L < 31, y, z) forms its node's viscous terms from its six faces in
// k_resid's order and finishes the node with resid_node.
constexpr int KRF_TX = 31, KRF_TY = 4, KRF_TZ = 2;
template <class T, class W, int MODE>
__global__ void __launch_bounds__(256, 2) k_resid_f(Lv<T, W> L, Par P, int upwind, int calc_pk, int coarse, int bback) {
  pdl_wait();
  __shared__ T s_fi[3][KRF_TZ][KRF_TY][32];
  __shared__ T s_fj[3][KRF_TZ][KRF_TY + 1][KRF_TX];
  __shared__ T s_fk[3][KRF_TZ + 1][KRF_TY][KRF_TX];
  const int Ln = threadIdx.x & 31, y = (threadIdx.x >> 5) & 3, z = threadIdx.x >> 7;
  const int i0 = blockIdx.x * KRF_TX + 1, j0 = blockIdx.y * KRF_TY + 1, k0 = blockIdx.z * KRF_TZ + 1;
  const int sj = L.sj, sk = L.sk;
  const int ni = L.im - 2, nj = L.jm - 2, nk = L.km - 2;
  const T rei = T(1) / T(P.ren);
  constexpr int CI = KRF_TZ * KRF_TY * 32, CJ = KRF_TZ * (KRF_TY + 1) * KRF_TX, CK = (KRF_TZ + 1) * KRF_TY * KRF_TX;
  auto face = [&](int dir, int l0, T* out, int cs) {
    T f[3];
    visc_face(L, dir, l0, rei, f);
    out[0] = f[0];
    out[cs] = f[1];
    out[2 * cs] = f[2];
  };
  {
    const int i = i0 + Ln - 1, j = j0 + y, k = k0 + z;
    if (i <= ni && j <= nj && k <= nk) face(0, i + sj * j + sk * k, &s_fi[0][z][y][Ln], CI);
  }
  for (int f = threadIdx.x; f < CJ + CK; f += 256) {
    if (f < CJ) {
      const int x = f % KRF_TX, r = f / KRF_TX, yy = r % (KRF_TY + 1), zz = r / (KRF_TY + 1);
      const int i = i0 + x, j = j0 + yy - 1, k = k0 + zz;
      if (i <= ni && j <= nj && k <= nk) face(1, i + sj * j + sk * k, &s_fj[0][zz][yy][x], CJ);
    } else {
      const int g = f - CJ;
      const int x = g % KRF_TX, r = g / KRF_TX, yy = r % KRF_TY, zz = r / KRF_TY;
      const int i = i0 + x, j = j0 + yy, k = k0 + zz - 1;
      if (i <= ni && j <= nj && k <= nk) face(2, i + sj * j + sk * k, &s_fk[0][zz][yy][x], CK);
    }
  }
  __syncthreads();
  if (Ln >= KRF_TX) return;
  const int i = i0 + Ln, j = j0 + y, k = k0 + z;
  if (i > ni || j > nj || k > nk) return;
  T visc[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) visc[m] = mulw(L.dc, s_fi[m][z][y][Ln + 1] - s_fi[m][z][y][Ln]);
#pragma unroll
  for (int m = 0; m < 3; ++m) visc[m] = fmaw(L.de, s_fj[m][z][y + 1][Ln] - s_fj[m][z][y][Ln], visc[m]);
#pragma unroll
  for (int m = 0; m < 3; ++m) visc[m] = fmaw(L.dz, s_fk[m][z + 1][y][Ln] - s_fk[m][z][y][Ln], visc[m]);
  resid_node<T, W, MODE, true>(L, P, upwind, calc_pk, coarse, bback, i, j, k, visc);
}

// dtau on every node (src/rhs_daf_dtau.F90:85-117): the smallest of the
// convective limits cfl / (|grad xi_d| dxi_d) and the viscous limits
// vnn / ((1/Re + nu_t) dxi_d^2 g_dd), formed as 1 / (the largest of their
// reciprocals) so that a node costs one division; equal to the reference's
// minimum up to rounding.  The metric parts change only with the grid:
// k_dtau_pre stores, per node, the largest convective reciprocal and the
// largest g_dd dxi_d^2 / vnn; k_dtau then needs nu_t and those two (1/Re +
// nu_t > 0, so the largest viscous reciprocal is (1/Re + nu_t) times the
// largest of the rest).
template <class T, class W>
__global__ void k_dtau_pre(Lv<T, W> L, Par P) {
  pdl_wait();
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L.N) return;
  const T rcfl = T(1) / T(P.cfl1), rvnn = T(1) / T(P.vnn1);
  const T dcsq = L.dc * L.dc, desq = L.de * L.de, dzsq = L.dz * L.dz;
  T g1 = L.csi[0][l] * L.csi[0][l] + L.csi[1][l] * L.csi[1][l] + L.csi[2][l] * L.csi[2][l];
  T g2 = L.eta[0][l] * L.eta[0][l] + L.eta[1][l] * L.eta[1][l] + L.eta[2][l] * L.eta[2][l];
  T g3 = L.zet[0][l] * L.zet[0][l] + L.zet[1][l] * L.zet[1][l] + L.zet[2][l] * L.zet[2][l];
  T c = sqrt(g1) * L.dc * rcfl;
  c = dmax(c, sqrt(g2) * L.de * rcfl);
  c = dmax(c, sqrt(g3) * L.dz * rcfl);
  T v = dcsq * g1 * rvnn;
  v = dmax(v, desq * g2 * rvnn);
  v = dmax(v, dzsq * g3 * rvnn);
  L.dtc[l] = c;
  L.dtv[l] = v;
}

template <class T, class W>
__global__ void k_dtau(Lv<T, W> L, Par P) {
  pdl_wait();
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= L.N) return;
  const T ret = T(1) / T(P.ren) + L.nut[l];
  L.dtau[l] = T(1) / dmax(L.dtc[l], ret * L.dtv[l]);
}

}  // namespace desalm
