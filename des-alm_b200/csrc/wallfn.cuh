// wallfn.cuh -- K_W: the log-law wall functions of the fine level's j walls
// (wf_eta, src/wf_mpi.F90:246-413), which the reference's driver calls after
// every fine DAF step (src/mg_driver.F90:221-224).  Off unless
// desalm_case.wall_functions is set.
//
// One thread per interior (i, k) of a wall (blockIdx.z: 0 = the j = 1 wall,
// layers j = 2, 3; 1 = the j = jm wall, layers jm-1, jm-2).  A thread reads
// layer 3 and the wall's geometry and writes layer 2 only, so the nodes are
// independent.
#pragma once
#include <cfloat>
#include "common.cuh"

namespace desalm {

// u_tau of the wall law the reference solves (funcv, src/wf_mpi.F90:602-628,
// roughness ks = 0), c = Re y:
//   c u_tau^2 = u0                          when c u_tau <= 11.3,
//   u_tau (ln(c u_tau) / kappa + B) = u0    when c u_tau > 11.3,
// with funcv's zero band at the branch point (:627) taken as the root where
// u0 falls in the jump between the branches.  Solved to full precision: the
// linear branch in closed form; the log branch, convex and increasing, by
// Newton's method from the branch point (the first step lands right of the
// root, the later ones decrease monotonically onto it), at most 100 steps.
DESALM_DEV double wf_utau(double u0, double c) {
  const double kapa = 0.41, blog = 5.45, yk = 11.3;
  if (!(c > 0.0) || !(u0 > 0.0)) return 0.0;
  if (c * u0 <= yk * yk) return sqrt(u0 / c);
  const double us = yk / c;
  if (us * (log(yk) / kapa + blog) >= u0) return us;
  double ut = us;
  for (int it = 0; it < 100; ++it) {
    const double lg = log(c * ut);
    const double g = ut * (lg / kapa + blog) - u0;
    const double dg = lg / kapa + blog + 1.0 / kapa;
    const double nx = ut - g / dg;
    const bool done = fabs(nx - ut) <= 4.0 * DBL_EPSILON * nx;
    ut = nx;
    if (done) break;
  }
  return ut;
}

template <class T, class W>
__global__ void __launch_bounds__(128) k_wallfn(Lv<T, W> L, Par P, const double* x, const double* y, const double* z,
                                                const double* wd) {
  pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  if (i > L.im - 2 || k > L.km - 2) return;
  const int side = blockIdx.z;
  const int j = side == 0 ? 0 : L.jm - 1;
  const int j1 = side == 0 ? 1 : L.jm - 2;
  const int j2 = side == 0 ? 2 : L.jm - 3;
  const int sj = L.sj, sk = L.sk;
  const int l = i + sj * j + sk * k, l1 = i + sj * j1 + sk * k, l2 = i + sj * j2 + sk * k;
  const double kapa = 0.41, blog = 5.45, yplm = 11.3, qmin = 1.0E-08;
  const double ren = P.ren;
  const double u = L.q[1][l2], v = L.q[2][l2], w = L.q[3][l2];
  // u_tau from the wall-parallel speed at layer 3 (src/wf_mpi.F90:287-309)
  const double e1 = L.eta[0][l], e2 = L.eta[1][l], e3 = L.eta[2][l];
  const double vmod = sqrt(e1 * e1 + e2 * e2 + e3 * e3);
  const double qnor = (u * e1 + v * e2 + w * e3) / vmod;
  const double qsq = u * u + v * v + w * w;
  const double qpar = sqrt(dmax(qsq - qnor * qnor, 0.0));
  const double ut = wf_utau(qpar, ren * wd[l2]);
  // layer 2 (src/wf_mpi.F90:318-402)
  if (qsq > qmin) {
    const double yplus = wd[l1] * ren * ut;
    const double q2 = yplus > yplm ? (log(yplus) / kapa + blog) * ut : yplus * ut;
    int lu = l + 1, ld = l - 1;
    const double xc = 0.5 * (x[lu] - x[ld]), yc = 0.5 * (y[lu] - y[ld]), zc = 0.5 * (z[lu] - z[ld]);
    lu = l + sk; ld = l - sk;
    const double xz = 0.5 * (x[lu] - x[ld]), yz = 0.5 * (y[lu] - y[ld]), zz = 0.5 * (z[lu] - z[ld]);
    const double sg11 = sqrt(xc * xc + yc * yc + zc * zc);
    const double sg33 = sqrt(xz * xz + yz * yz + zz * zz);
    const double qc1 = (L.csi[0][l2] * u + L.csi[1][l2] * v + L.csi[2][l2] * w) * sg11;
    const double qc2 = (L.zet[0][l2] * u + L.zet[1][l2] * v + L.zet[2][l2] * w) * sg33;
    const double cgama = (xc * xz + yc * yz + zc * zz) / (sg11 * sg33);
    double fb = sqrt(qc1 * qc1 + qc2 * qc2 + 2.0 * qc1 * qc2 * cgama);
    fb = (qc1 + qc2 * cgama) / fb;
    fb = dmin(fb, 1.0);
    fb = dmax(fb, -1.0);
    const double fbeta = qc2 > 0.0 ? acos(fb) : -acos(fb);
    const double c2 = q2 * sin(fbeta) / sin(acos(cgama));
    const double c1 = q2 * cos(fbeta) - c2 * cgama;
    L.q[1][l1] = T(c1 * xc / sg11 + c2 * xz / sg33);
    L.q[2][l1] = T(c1 * yc / sg11 + c2 * yz / sg33);
    L.q[3][l1] = T(c1 * zc / sg11 + c2 * zz / sg33);
    L.q[4][l1] = T(kapa * yplus / ren);
  } else {
    L.q[1][l1] = T(0);
    L.q[2][l1] = T(0);
    L.q[3][l1] = T(0);
    L.q[4][l1] = T(0.1 / ren);
  }
}

}  // namespace desalm
