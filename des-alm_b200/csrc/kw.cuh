// kw.cuh -- Wilcox's (1994) low-Reynolds-number k-omega sub-iterations on the
// fine level (kw_eddy, src/kw_eddy.F90:2-296).  k is q(5), the field the SA
// model uses for nu_tilde; omega, the reference's q(6), is a separate array
// with its own time levels.  The reference compiles none of this (kw_eddy.F90
// is not in src/makefile and includes an ADI file that does not exist), so
// the ADI is restated from the SA model's (src/rhs_sa_adi_solver.F90:
// 50-244): one scalar system per line for each of k and omega, with the
// implicit-source factors dk and dw dividing the rows and the i sweep's
// right-hand side, and the face diffusivity of rhs_kw_viscous.
//
// Per kw_eddy call:
//   k_kw_pre       rhs_kw_ptke (interior, src/rhs_kw_ptke.F90:42-96) and
//                  rhs_kw_coef (every node, src/rhs_kw_coef.F90:41-54)
//   per sub-iteration:
//   k_kw_rhs       rhs_kw_prod, rhs_kw_viscous, rhs_kw_flux,
//                  rhs_kw_unst_visc, rhs_kw_implicit_source fused, plus the
//                  ADI rows of both scalars in all three directions
//   k_sa_sweep4    the line solves of k, then of omega (sa.cuh), the k sweep
//                  applying the update (src/kw_eddy.F90:247-266)
//   k_kw_bc<DIR>   rhs_kw_bcond's faces (src/rhs_kw_bcond.F90:22-475)
//   k_kw_nut       rhs_kw_coef again and nu_t = As k / omega (:477-491)
//   k_kw_edges     omega on edges where two walls meet (:493-519)
// Everything but the ADI rows and line solves is FP64 in every mode.
#pragma once
#include "sa.cuh"

namespace desalm {

// fine-level work arrays of the k-omega model: FP64 first, then the omega
// ADI rows and right-hand side in the sweep precision (allocated as FP64
// slots, used as SW)
struct KwWork {
  static const int NARR = 19;
  // om, omn, omnm1, As, Ac, Bs, ptke, (two spare) | co_w[9], rh_w
  double* a[NARR];
};

template <class SW>
struct KwT {
  SaT<SW> S;           // geometry, k = q[4], nu_t, U/J, the k ADI rows and rh
  double* om;
  const double* omn;
  const double* omnm1;
  double* As;
  double* Ac;
  double* Bs;
  double* ptke;
  SW* cow[9];
  SW* rhw;
  double ckin, cein;
  int ista, iend, jsta, jend, ksta, kend;  // 0-based face-loop ranges (rhs_kw_bcond.F90:40-49)
};

DESALM_DEV void kw_coef_node(double k, double w, double ren, double& as, double& ac, double& bs) {
  const double Rt = ren * k / w;
  const double Rt4 = Rt * Rt * Rt * Rt;
  as = (0.15 + Rt) / (6.0 + Rt);
  ac = ((0.27 + Rt) / (2.70 + Rt)) * 0.5555 / as;
  bs = ((1137.77 + Rt4) / (4096.00 + Rt4)) * 0.09;
}

// ptke = nu_t (2 (u_x^2 + v_y^2 + w_z^2) + (u_y + v_x)^2 + (u_z + w_x)^2 +
// (v_z + w_y)^2) on interior nodes; As, Ac, Bs on every node.
template <class SW>
__global__ void k_kw_pre(KwT<SW> K) {
  pdl_wait();
  const SaT<SW>& S = K.S;
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= S.N) return;
  double as, ac, bs;
  kw_coef_node(S.q[4][l], K.om[l], S.ren, as, ac, bs);
  K.As[l] = as; K.Ac[l] = ac; K.Bs[l] = bs;
  const int i = l % S.sj, j = (l / S.sj) % S.jm, k = l / S.sk;
  if (i < 1 || i > S.im - 2 || j < 1 || j > S.jm - 2 || k < 1 || k > S.km - 2) return;
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
  K.ptke[l] = S.nut[l] * (2.0 * (d[0][0] * d[0][0] + d[1][1] * d[1][1] + d[2][2] * d[2][2]) +
                          (d[0][1] + d[1][0]) * (d[0][1] + d[1][0]) +
                          (d[0][2] + d[2][0]) * (d[0][2] + d[2][0]) +
                          (d[1][2] + d[2][1]) * (d[1][2] + d[2][1]));
}

// Viscous fluxes of k and omega through the face l0 -> l0 + st[dir]
// (src/rhs_kw_viscous.F90:49-238): rei + nu_t / sigma at both nodes,
// sigma_k = sigma_w = 2.
template <class SW>
DESALM_DEV void kw_visc_face(const KwT<SW>& K, int dir, int l0, double rei, double out[2], double* gvt = nullptr) {
  const SaT<SW>& S = K.S;
  const int sj = S.sj, sk = S.sk;
  int l1;
  double g[2][3];
#pragma unroll
  for (int s = 0; s < 2; ++s) {
    const double* v = s == 0 ? S.q[4] : K.om;
    if (dir == 0) {
      l1 = l0 + 1;
      g[s][0] = v[l1] - v[l0];
      g[s][1] = 0.25 * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
      g[s][2] = 0.25 * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
    } else if (dir == 1) {
      l1 = l0 + sj;
      g[s][0] = 0.25 * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
      g[s][1] = v[l1] - v[l0];
      g[s][2] = 0.25 * (v[l1 + sk] - v[l1 - sk] + v[l0 + sk] - v[l0 - sk]);
    } else {
      l1 = l0 + sk;
      g[s][0] = 0.25 * (v[l1 + 1] - v[l1 - 1] + v[l0 + 1] - v[l0 - 1]);
      g[s][1] = 0.25 * (v[l1 + sj] - v[l1 - sj] + v[l0 + sj] - v[l0 - sj]);
      g[s][2] = v[l1] - v[l0];
    }
  }
  const double a1 = S.csi[0][l1] + S.csi[0][l0], a2 = S.csi[1][l1] + S.csi[1][l0], a3 = S.csi[2][l1] + S.csi[2][l0];
  const double b1 = S.eta[0][l1] + S.eta[0][l0], b2 = S.eta[1][l1] + S.eta[1][l0], b3 = S.eta[2][l1] + S.eta[2][l0];
  const double c1 = S.zet[0][l1] + S.zet[0][l0], c2 = S.zet[1][l1] + S.zet[1][l0], c3 = S.zet[2][l1] + S.zet[2][l0];
  double k1, k2, k3;
  if (dir == 0) { k1 = a1 * a1 + a2 * a2 + a3 * a3; k2 = a1 * b1 + a2 * b2 + a3 * b3; k3 = a1 * c1 + a2 * c2 + a3 * c3; }
  else if (dir == 1) { k1 = b1 * a1 + b2 * a2 + b3 * a3; k2 = b1 * b1 + b2 * b2 + b3 * b3; k3 = b1 * c1 + b2 * c2 + b3 * c3; }
  else { k1 = c1 * a1 + c2 * a2 + c3 * a3; k2 = c1 * b1 + c2 * b2 + c3 * b3; k3 = c1 * c1 + c2 * c2 + c3 * c3; }
  const double rsa = 1.0 / (S.aj[l1] + S.aj[l0]);
  const double r1 = rei + S.nut[l1] * 0.5, r0 = rei + S.nut[l0] * 0.5;  // rei + nu_t / 2
  const double vtj = 0.25 * (r1 + r0) * rsa;
  out[0] = vtj * (k1 * g[0][0] + k2 * g[0][1] + k3 * g[0][2]);
  out[1] = vtj * (k1 * g[1][0] + k2 * g[1][1] + k3 * g[1][2]);
  // the face's diffusive ADI coefficient: (1/Re + (nu_t1 + nu_t0) / 4)
  // |g_dir|^2 / (J1 + J0) with the summed metrics, which is 2 vtj times
  // the direction's own product (k1, k2 or k3)
  if (gvt) *gvt = 2.0 * vtj * (dir == 0 ? k1 : (dir == 1 ? k2 : k3));
}

// First-order flux-difference upwind fluxes of k and omega through the
// face l0 -> l0 + st (src/rhs_kw_flux.F90:20-166): the face speed is formed
// from the summed metrics and velocities over the summed Jacobians.
template <class SW>
DESALM_DEV void kw_conv_face(const KwT<SW>& K, int dir, int l0, int st, double out[2], double* ucf = nullptr) {
  const SaT<SW>& S = K.S;
  const int l1 = l0 + st;
  const double* const* mt = dir == 0 ? S.csi : (dir == 1 ? S.eta : S.zet);
  const double gcu = (mt[0][l1] + mt[0][l0]) * (S.q[1][l1] + S.q[1][l0]);
  const double gev = (mt[1][l1] + mt[1][l0]) * (S.q[2][l1] + S.q[2][l0]);
  const double gzw = (mt[2][l1] + mt[2][l0]) * (S.q[3][l1] + S.q[3][l0]);
  const double eigh = 0.5 * fabs((gcu + gev + gzw) / (S.aj[l1] + S.aj[l0]));
  const double u1 = S.uc[dir][l1], u0 = S.uc[dir][l0];
  const double* k5 = S.q[4];
  out[0] = 0.5 * (k5[l1] * u1 + k5[l0] * u0 - eigh * (k5[l1] - k5[l0]));
  out[1] = 0.5 * (K.om[l1] * u1 + K.om[l0] * u0 - eigh * (K.om[l1] - K.om[l0]));
  if (ucf) { ucf[0] = u0; ucf[1] = u1; }
}

// ADI rows of k and of omega along direction d at interior node l
// (restated from src/rhs_sa_adi_solver.F90:53-71), from the two faces the
// residual has just formed: av = |U/J| on the face + the face's diffusive
// coefficient (1/Re + (nu_t1 + nu_t0) / (2 sigma)) |g_d|^2 / (J1 + J0), with
// sigma_k = sigma_w = 2 for both scalars; their rows differ only in the
// implicit-source factor that divides them (dk for k, dw for omega).  gm, gp:
// the diffusive coefficients of the faces (l - s, l) and (l, l + s); um, up:
// their U/J pairs.
template <class SW>
DESALM_DEV void kw_adi_rows(const KwT<SW>& K, int l, int d, double gm, double gp, const double um[2],
                            const double up[2], double aj, double dtev, double fk, double fw) {
  const SaT<SW>& S = K.S;
  const double av0 = 0.5 * fabs(um[1] + um[0]) + gm;
  const double av1 = 0.5 * fabs(up[1] + up[0]) + gp;
  const double base = 0.5 * dtev * aj;
  const double cw = um[0] + av0, cp = av0 + av1, ce = up[1] - av1;
  const double dk = base / fk, dw = base / fw;
  S.co[3 * d + 0][l] = SW(-dk * cw);
  S.co[3 * d + 1][l] = SW(1.0 + dk * cp);
  S.co[3 * d + 2][l] = SW(dk * ce);
  K.cow[3 * d + 0][l] = SW(-dw * cw);
  K.cow[3 * d + 1][l] = SW(1.0 + dw * cp);
  K.cow[3 * d + 2][l] = SW(dw * ce);
}

// One fused pass over the interior of rhs_kw_prod, rhs_kw_viscous,
// rhs_kw_flux, rhs_kw_unst_visc and rhs_kw_implicit_source, giving the
// right-hand sides of k and omega already divided by dk and dw (the i sweep's
// input), and the ADI rows of both scalars, with every face flux formed once
// (a kernel of one thread per node forms each face twice, once for each of
// its nodes: 5% slower on the turbine box).  A CTA covers a tile of
// 31 x 4 x 2 nodes with 32 x 4 x 2 threads.
//   phase 1  lane L of row y, plane z forms the i face between nodes
//            i0 + L - 1 and i0 + L; the tile's j faces (5 rows of 31, both
//            planes) and k faces (3 planes of 4 x 31) are shared out over
//            all threads; each face's viscous and convective fluxes of k and
//            omega and its diffusive ADI coefficient go to shared memory
//            (component-major, so that neighbouring lanes read neighbouring
//            words);
//   phase 2  thread (L < 31, y, z) adds its node's six faces (i, j, k; plus
//            face minus minus face, viscous then convective) and finishes the
//            node.
constexpr int KWF_TX = 31, KWF_TY = 4, KWF_TZ = 2;
template <class SW>
__global__ void __launch_bounds__(256, 2) k_kw_rhs(KwT<SW> K) {
  pdl_wait();
  const SaT<SW>& S = K.S;
  __shared__ double s_fi[5][KWF_TZ][KWF_TY][32];
  __shared__ double s_fj[5][KWF_TZ][KWF_TY + 1][KWF_TX];
  __shared__ double s_fk[5][KWF_TZ + 1][KWF_TY][KWF_TX];
  const int L = threadIdx.x & 31, y = (threadIdx.x >> 5) & 3, z = threadIdx.x >> 7;
  const int i0 = blockIdx.x * KWF_TX + 1, j0 = blockIdx.y * KWF_TY + 1, k0 = blockIdx.z * KWF_TZ + 1;
  const int sj = S.sj, sk = S.sk;
  const int ni = S.im - 2, nj = S.jm - 2, nk = S.km - 2;
  const double rei = 1.0 / S.ren;
  // the face of direction dir whose lower node is l0 into component slots
  // c * cs of out (c = 0, 1: viscous k, omega; 2: diffusive coefficient;
  // 3, 4: convective k, omega)
  auto face = [&](int dir, int l0, double* out, int cs) {
    const int stp = dir == 0 ? 1 : (dir == 1 ? sj : sk);
    double fv[2], fc[2], g;
    kw_visc_face(K, dir, l0, rei, fv, &g);
    kw_conv_face(K, dir, l0, stp, fc);
    out[0] = fv[0];
    out[cs] = fv[1];
    out[2 * cs] = g;
    out[3 * cs] = fc[0];
    out[4 * cs] = fc[1];
  };
  constexpr int CI = KWF_TZ * KWF_TY * 32, CJ = KWF_TZ * (KWF_TY + 1) * KWF_TX, CK = (KWF_TZ + 1) * KWF_TY * KWF_TX;
  {
    const int i = i0 + L - 1, j = j0 + y, k = k0 + z;
    if (i <= ni && j <= nj && k <= nk) face(0, i + sj * j + sk * k, &s_fi[0][z][y][L], CI);
  }
  for (int f = threadIdx.x; f < CJ + CK; f += 256) {
    if (f < CJ) {
      const int x = f % KWF_TX, r = f / KWF_TX, yy = r % (KWF_TY + 1), zz = r / (KWF_TY + 1);
      const int i = i0 + x, j = j0 + yy - 1, k = k0 + zz;
      if (i <= ni && j <= nj && k <= nk) face(1, i + sj * j + sk * k, &s_fj[0][zz][yy][x], CJ);
    } else {
      const int g = f - CJ;
      const int x = g % KWF_TX, r = g / KWF_TX, yy = r % KWF_TY, zz = r / KWF_TY;
      const int i = i0 + x, j = j0 + yy, k = k0 + zz - 1;
      if (i <= ni && j <= nj && k <= nk) face(2, i + sj * j + sk * k, &s_fk[0][zz][yy][x], CK);
    }
  }
  __syncthreads();
  if (L >= KWF_TX) return;
  const int i = i0 + L, j = j0 + y, k = k0 + z;
  if (i > ni || j > nj || k > nk) return;
  const int l = i + sj * j + sk * k;
  const double cw2 = 0.075;
  const double kv = S.q[4][l], wv = K.om[l], aj = S.aj[l];
  // rhs_kw_prod (src/rhs_kw_prod.F90:18-31)
  const double pkw1a = K.Bs[l] * wv * kv;
  const double pk1 = (-K.ptke[l] + pkw1a) / aj;
  const double pkw2a = -K.Ac[l] * wv * K.ptke[l] / kv;
  const double pkw2b = cw2 * wv * wv;
  const double pk2 = (pkw2a + pkw2b) / aj;
  double v[2] = {0, 0}, r[2] = {0, 0};
  double gdm[3], gdp[3], ucm[3][2], ucp[3][2];
  const int st[3] = {1, sj, sk};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    // the plus face (l | l + s) and the minus face (l - s | l) of direction d
    const double* fp = d == 0 ? &s_fi[0][z][y][L + 1] : (d == 1 ? &s_fj[0][z][y + 1][L] : &s_fk[0][z + 1][y][L]);
    const double* fm = d == 0 ? &s_fi[0][z][y][L] : (d == 1 ? &s_fj[0][z][y][L] : &s_fk[0][z][y][L]);
    const int cs = d == 0 ? CI : (d == 1 ? CJ : CK);
    v[0] = v[0] + fp[0] - fm[0];
    v[1] = v[1] + fp[cs] - fm[cs];
    r[0] = r[0] + fp[3 * cs] - fm[3 * cs];
    r[1] = r[1] + fp[4 * cs] - fm[4 * cs];
    gdp[d] = fp[2 * cs];
    gdm[d] = fm[2 * cs];
    const double u0 = S.uc[d][l];
    ucm[d][0] = S.uc[d][l - st[d]];
    ucm[d][1] = u0;
    ucp[d][0] = u0;
    ucp[d][1] = S.uc[d][l + st[d]];
  }
  // rhs_kw_unst_visc (src/rhs_kw_unst_visc.F90:23-37)
  const double dtj = 2.0 * S.delti * aj;
  const double dq5dt = S.es * (3.0 * kv - 4.0 * S.qn5[l] + S.qnm1_5[l]) / dtj;
  const double dq6dt = S.es * (3.0 * wv - 4.0 * K.omn[l] + K.omnm1[l]) / dtj;
  const double r1 = r[0] + dq5dt - v[0] + pk1;
  const double r2 = r[1] + dq6dt - v[1] + pk2;
  // rhs_kw_implicit_source (src/rhs_kw_implicit_source.F90:41-53)
  const double dtev = S.dtev[l];
  const double dkv = 1.0 + K.Bs[l] * dtev * wv;
  const double dwv = 1.0 + cw2 * dtev * wv;
  S.rh[l] = SW((-dtev * aj * r1) / dkv);
  K.rhw[l] = SW((-dtev * aj * r2) / dwv);
#pragma unroll
  for (int d = 0; d < 3; ++d) kw_adi_rows(K, l, d, gdm[d], gdp[d], ucm[d], ucp[d], aj, dtev, dkv, dwv);
}

// rhs_kw_bcond's faces of one direction (src/rhs_kw_bcond.F90:51-475): side
// 0 then side 1 per thread, over the transverse ranges the reference uses
// (edges toward wall faces excluded).
template <class SW, int DIR>
__global__ void k_kw_bc(KwT<SW> K) {
  pdl_wait();
  const SaT<SW>& S = K.S;
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  int b = blockIdx.y;
  int a0, a1, b0, b1, n, st, lb;
  if (DIR == 0) { a0 = K.jsta; a1 = K.jend; b0 = K.ksta; b1 = K.kend; }
  else if (DIR == 1) { a0 = K.ista; a1 = K.iend; b0 = K.ksta; b1 = K.kend; }
  else { a0 = K.ista; a1 = K.iend; b0 = K.jsta; b1 = K.jend; }
  a += a0;
  b += b0;
  if (a > a1 || b > b1) return;
  if (DIR == 0) { n = S.im; st = 1; lb = S.sj * a + S.sk * b; }
  else if (DIR == 1) { n = S.jm; st = S.sj; lb = a + S.sk * b; }
  else { n = S.km; st = S.sk; lb = a + S.sj * b; }
  double* k5 = S.q[4];
  double* w = K.om;
  const double srenp = 60.0 / S.ren / 0.075;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int bi = 2 * DIR + side;
    const int bt = S.btype[bi];
    const int l = side == 0 ? lb : lb + (n - 1) * st;
    const int s = side == 0 ? st : -st;
    if (bt == 1) {
      const double yd = S.wd[l + s];
      w[l] = srenp / yd / yd;
      k5[l] = 0.0;
    } else if (bt == 2 || bt == 3 || bt == 5 || bt == 6) {
      double kn, wn;
      if (bt == 5) {
        const double r = S.rat[(size_t)bi * S.ratdim * S.ratdim + a + (size_t)S.ratdim * b];
        kn = (1.0 + r) * k5[l + s] - r * k5[l + 2 * s];
        wn = (1.0 + r) * w[l + s] - r * w[l + 2 * s];
      } else if (bt == 6) {
        const int lo = side == 0 ? lb + (n - 2) * st : lb + st;
        kn = k5[lo];
        wn = w[lo];
      } else {
        kn = S.sa1[bi] * k5[l + s] + S.sb1[bi] * k5[l + 2 * s];
        wn = S.sa1[bi] * w[l + s] + S.sb1[bi] * w[l + 2 * s];
      }
      k5[l] = kn > K.ckin ? kn : K.ckin;
      w[l] = wn > K.cein ? wn : K.cein;
    }
  }
}

// As, Ac, Bs and nu_t = As k / omega on every node (src/rhs_kw_bcond.F90:477-491)
template <class SW>
__global__ void k_kw_nut(KwT<SW> K) {
  pdl_wait();
  const SaT<SW>& S = K.S;
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= S.N) return;
  const double kv = S.q[4][l], wv = K.om[l];
  double as, ac, bs;
  kw_coef_node(kv, wv, S.ren, as, ac, bs);
  K.As[l] = as; K.Ac[l] = ac; K.Bs[l] = bs;
  S.nut[l] = as * kv / wv;
}

// omega on every edge where two wall faces meet, the mean of its two face
// neighbours (src/rhs_kw_bcond.F90:493-519), edges in the reference's order;
// one CTA, a barrier between edges (a corner belongs to three edges).
template <class SW>
__global__ void k_kw_edges(KwT<SW> K) {
  pdl_wait();
  const SaT<SW>& S = K.S;
  const int* bt = S.btype;
  const int im = S.im, jm = S.jm, km = S.km, sj = S.sj, sk = S.sk;
  double* w = K.om;
  // edge e: faces (f1, f2); the edge runs along axis ax; fixed coordinates
  // and the two inward steps
  const int F1[12] = {0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 3, 3};
  const int F2[12] = {2, 3, 4, 5, 2, 3, 4, 5, 4, 5, 4, 5};
  for (int e = 0; e < 12; ++e) {
    if (bt[F1[e]] == 1 && bt[F2[e]] == 1) {
      // fixed index of each face: face 2d sits at 0, face 2d+1 at m-1
      int fi = -1, fj = -1, fk = -1, s1 = 0, s2 = 0;
      auto setf = [&](int f, int& stp) {
        const int d = f / 2, hi = f % 2;
        const int ext = d == 0 ? im : (d == 1 ? jm : km);
        const int stride = d == 0 ? 1 : (d == 1 ? sj : sk);
        if (d == 0) fi = hi ? ext - 1 : 0;
        else if (d == 1) fj = hi ? ext - 1 : 0;
        else fk = hi ? ext - 1 : 0;
        stp = hi ? -stride : stride;
      };
      setf(F1[e], s1);
      setf(F2[e], s2);
      const int n = fi < 0 ? im : (fj < 0 ? jm : km);
      for (int t = threadIdx.x; t < n; t += blockDim.x) {
        const int ii = fi < 0 ? t : fi, jj = fj < 0 ? t : fj, kk = fk < 0 ? t : fk;
        const int l = ii + sj * jj + sk * kk;
        w[l] = 0.5 * (w[l + s1] + w[l + s2]);
      }
    }
    __syncthreads();
  }
}

}  // namespace desalm
