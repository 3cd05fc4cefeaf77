// outlet.cuh -- K_O: the characteristics outlet (btype 5) on the front face
// i = im of the fine level (src/solver_daf.F90:318-373).
//
// One thread per interior node (j, k) of the plane i = im computes, in
// registers, the plane's residual from its eta and zeta derivatives alone
// (mg_brhs, src/mg_brhs.F90:58-97):
//   viscous face fluxes and visc     src/brhs_viscous.F90:40-160
//   pressure dissipation diss(1)     src/brhs_diss_p.F90:33-89
//   pressure gradient + divergence   src/brhs_flux_sans_convec.F90:45-86
//   QUICK convection (upwind = 2)    src/brhs_convec_quick.F90:41-205
//   BDF2 + assembly                  src/brhs_unst_visc_diss.F90:30-44
// then adds the locally one-dimensional inviscid (LODI) csi terms of
// nonreflect_ibc (src/nonreflect_ibc.F90:86-242, inout = 2): the outgoing
// part of the csi flux Jacobian applied to the one-sided difference
// q(im) - q(im-1), in the reference's closed form (rows of si are its left
// eigenvectors, the columns of calc_rh's matrix the right ones; the speeds
// ucon +- sqrt(ucon^2 + g11) are those of beta = 1).  The plane's node is
// then prepared for the csi line solve exactly as K_R prepares an interior
// node: r = S (-dtau rh J), r <- Ma^-1 r (src/rhs_diag_solver.F90:53-122,
// loops to idend), sigma, and the eta and zeta row coefficients (the csi
// row of the plane is special and built by the i sweep from hc).  Divisions
// by J are multiplications by the stored 1/J, as in K_R.
#pragma once
#include "resid.cuh"

namespace desalm {

// Viscous flux through the eta (dir 1) or zeta (dir 2) face between l0 and
// its neighbour on the plane, without csi derivatives (src/brhs_viscous.F90:
// 60-99 for dir 1, :109-148 for dir 2).
template <class T, class W>
DESALM_DEV void visc_face_plane(const Lv<T, W>& L, int dir, int l0, T rei, T out[3]) {
  const int sj = L.sj, sk = L.sk;
  const T q4 = T(0.25);
  const int l1 = dir == 1 ? l0 + sj : l0 + sk;
  T E[3], Z[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    const T* v = L.q[m + 1];
    if (dir == 1) {
      E[m] = L.de * (v[l1] - v[l0]);
      Z[m] = (q4 * L.dz) * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
    } else {
      E[m] = (q4 * L.de) * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
      Z[m] = L.dz * (v[l1] - v[l0]);
    }
  }
  T b1 = L.eta[0][l1] + L.eta[0][l0], b2 = L.eta[1][l1] + L.eta[1][l0], b3 = L.eta[2][l1] + L.eta[2][l0];
  T c1 = L.zet[0][l1] + L.zet[0][l0], c2 = L.zet[1][l1] + L.zet[1][l0], c3 = L.zet[2][l1] + L.zet[2][l0];
  T uu1 = b1 * E[0] + c1 * Z[0], vv1 = b1 * E[1] + c1 * Z[1], ww1 = b1 * E[2] + c1 * Z[2];
  T uu2 = b2 * E[0] + c2 * Z[0], vv2 = b2 * E[1] + c2 * Z[1], ww2 = b2 * E[2] + c2 * Z[2];
  T uu3 = b3 * E[0] + c3 * Z[0], vv3 = b3 * E[1] + c3 * Z[1], ww3 = b3 * E[2] + c3 * Z[2];
  T n1, n2, n3, k2, k3;
  if (dir == 1) {
    n1 = b1; n2 = b2; n3 = b3;
    k2 = b1 * b1 + b2 * b2 + b3 * b3; k3 = b1 * c1 + b2 * c2 + b3 * c3;
  } else {
    n1 = c1; n2 = c2; n3 = c3;
    k2 = c1 * b1 + c2 * b2 + c3 * b3; k3 = c1 * c1 + c2 * c2 + c3 * c3;
  }
  T vtj = T(0.25) * ((rei + L.nut[l1]) + (rei + L.nut[l0])) / (L.aj[l1] + L.aj[l0]);
  out[0] = vtj * (n1 * uu1 + n2 * vv1 + n3 * ww1 + k2 * E[0] + k3 * Z[0]);
  out[1] = vtj * (n1 * uu2 + n2 * vv2 + n3 * ww2 + k2 * E[1] + k3 * Z[1]);
  out[2] = vtj * (n1 * uu3 + n2 * vv3 + n3 * ww3 + k2 * E[2] + k3 * Z[2]);
}

template <class T, class W>
__global__ void __launch_bounds__(128) k_outlet(Lv<T, W> L, Par P) {
  pdl_wait();
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (j > L.jm - 2 || k > L.km - 2) return;
  const int sj = L.sj, sk = L.sk;
  const int l = (L.im - 1) + sj * j + sk * k;
  const T rei = T(1) / T(P.ren);
  const T dsp[3] = {L.dc, L.de, L.dz};
  const int st[3] = {1, sj, sk};
  const int pos[3] = {L.im - 1, j, k};
  const int ext[3] = {L.im, L.jm, L.km};

  // ---- viscous terms (eta, then zeta)
  T visc[3];
  {
    T fp[3], fm[3];
    visc_face_plane(L, 1, l, rei, fp);
    visc_face_plane(L, 1, l - sj, rei, fm);
#pragma unroll
    for (int m = 0; m < 3; ++m) visc[m] = L.de * (fp[m] - fm[m]);
    visc_face_plane(L, 2, l, rei, fp);
    visc_face_plane(L, 2, l - sk, rei, fm);
#pragma unroll
    for (int m = 0; m < 3; ++m) visc[m] = visc[m] + L.dz * (fp[m] - fm[m]);
  }

  // ---- pressure dissipation, with the boundary copies aux(j=1) = aux(j=2)
  // etc. (src/brhs_diss_p.F90:75-79)
  T acc[2];
#pragma unroll
  for (int d = 1; d < 3; ++d) {
    const T dsq = dsp[d] * dsp[d];
    const int s = st[d];
    T f0 = diss_fv(L, d, l, s, dsq);
    T fmi = pos[d] - 1 == 0 ? f0 : diss_fv(L, d, l - s, s, dsq);
    T fpl = pos[d] + 1 == ext[d] - 1 ? f0 : diss_fv(L, d, l + s, s, dsq);
    acc[d - 1] = fpl - T(2) * f0 + fmi;
  }
  const T diss1 = T(P.pdiss) * (acc[0] + acc[1]);

  // ---- pressure gradient and divergence (no csi terms: dudx = 0)
  T rh[4];
  {
    const T* p = L.q[0];
    const T dh1 = T(0.5) * L.de, dh2 = T(0.5) * L.dz;
    const T pp1 = p[l + sj] * L.rj[l + sj], pm1 = p[l - sj] * L.rj[l - sj];
    const T pp2 = p[l + sk] * L.rj[l + sk], pm2 = p[l - sk] * L.rj[l - sk];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      T v = dh1 * (pp1 * L.eta[x][l + sj] - pm1 * L.eta[x][l - sj]);
      rh[x + 1] = v + dh2 * (pp2 * L.zet[x][l + sk] - pm2 * L.zet[x][l - sk]);
    }
    rh[0] = dh1 * (ucn(L, 1, l + sj) - ucn(L, 1, l - sj)) + dh2 * (ucn(L, 2, l + sk) - ucn(L, 2, l - sk));
  }

  // ---- convection: QUICK, first-order upwind next to the plane's edges
#pragma unroll
  for (int d = 1; d < 3; ++d) {
    const int s = st[d];
    const T h = dsp[d];
    T ucon = T(0.5) * ucn(L, d, l);
    T up = ucon + dabs(ucon), um = ucon - dabs(ucon);
    bool first = pos[d] == 1 || pos[d] == ext[d] - 2;
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

  // ---- LODI csi terms, calc_L_general + calc_L_max + calc_rh.  L1 = 0 on
  // this side, so only rows 2..4 of si are formed.
  {
    const T u = L.q[1][l], v = L.q[2][l], w = L.q[3][l];
    const T ucon = ucn(L, 0, l) * L.aj[l];
    const T c1 = L.csi[0][l], c2 = L.csi[1][l], c3 = L.csi[2][l];
    const T gjj = c1 * c1 + c2 * c2 + c3 * c3;
    const T sg = sqrt(gjj);
    const T cj = sqrt(ucon * ucon + gjj);
    T dq[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) dq[m] = L.q[m][l] - L.q[m][l - 1];
    const T lam1 = ucon - cj, lam2 = ucon + cj;
    const T kj = c1 + c2 + c3;
    const T d1 = (c2 - c1 + lam1 * (v - u)) / kj, d2 = (c2 - c1 + lam2 * (v - u)) / kj;
    const T d3 = (c3 - c1 + lam1 * (w - u)) / kj, d4 = (c3 - c1 + lam2 * (w - u)) / kj;
    const T d5 = (c2 - c1 + ucon * (v - u)) / kj * T(2), d6 = (c3 - c1 + ucon * (w - u)) / kj * T(2);
    const T cc = T(2) * cj * cj / kj;
    const T sc = sg / (T(2) * cj * cj);
    const T g2 = sc * (-lam1 * dq[0] + c1 * dq[1] + c2 * dq[2] + c3 * dq[3]);
    const T g3 = sc * ((lam2 * d1 + lam1 * d2) * dq[0] + (-cc - c1 * d5) * dq[1] + (cc - c2 * d5) * dq[2] - c3 * d5 * dq[3]);
    const T g4 = sc * ((lam2 * d3 + lam1 * d4) * dq[0] + (-cc - c1 * d6) * dq[1] - c2 * d6 * dq[2] + (cc - c3 * d6) * dq[3]);
    const T L2 = lam2 * g2;
    const T L3 = ucon < T(0) ? T(0) : ucon * g3;
    const T L4 = ucon < T(0) ? T(0) : ucon * g4;
    const T rsg = T(1) / sg, rj = L.rj[l];
    rh[0] = rh[0] + (cj * L2) * rsg * rj;
    rh[1] = rh[1] + ((c1 + u * lam2) * L2 - c2 * L3 - c3 * L4) * rsg * rj;
    rh[2] = rh[2] + ((c2 + v * lam2) * L2 + (c1 + c3) * L3 - c3 * L4) * rsg * rj;
    rh[3] = rh[3] + ((c3 + w * lam2) * L2 - c2 * L3 + (c1 + c2) * L4) * rsg * rj;
  }

  // ---- r = S (-dtau rh J), then Ma^-1 r, as K_R
  const T dtau = L.dtau[l];
  const T alpha = T(1) + (T(P.es) * T(1.5) / T(P.delti)) * dtau;
  const T ra = T(1) / alpha;
  const T sg = sqrt(T(P.beta) * alpha), th = sqrt(T(P.beta) * ra);
  const T s[4] = {T(P.beta), ra, ra, ra};
  W rw[4], rp[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) rw[m] = W(s[m] * (-dtau * rh[m] * L.aj[l]));
  minv_apply<W>(W(L.csi[0][l]), W(L.csi[1][l]), W(L.csi[2][l]), W(sg), rw, rp);

  // ---- eta and zeta row coefficients of the node and of the boundary nodes
  // before/after its lines (src/rhs_diag_solver.F90:335-360, 511-536)
  const T* const* mt[3] = {L.csi, L.eta, L.zet};
#pragma unroll
  for (int d = 1; d < 3; ++d) {
    const T* const* m3 = mt[d];
    T g = m3[0][l] * m3[0][l] + m3[1][l] * m3[1][l] + m3[2][l] * m3[2][l];
    T spr = th * sqrt(g);
    T dh = T(0.5) * dsp[d];
    L.tc[d][l] = W(dtau * T(P.ep1[d]) * spr * (dsp[d] * dsp[d]));
    L.hc[d][l] = W(dtau * dh * spr);
    if (pos[d] == 1 || pos[d] == ext[d] - 2) {
      const int lb = pos[d] == 1 ? l - st[d] : l + st[d];
      T s2, t2;
      sigma_theta(L.dtau[lb], P, s2, t2);
      T gb = m3[0][lb] * m3[0][lb] + m3[1][lb] * m3[1][lb] + m3[2][lb] * m3[2][lb];
      L.hc[d][lb] = W(L.dtau[lb] * dh * (t2 * sqrt(gb)));
    }
  }
#pragma unroll
  for (int m = 0; m < 4; ++m) L.wk[m][l] = rp[m];
  L.sig[l] = W(sg);
}

}  // namespace desalm
