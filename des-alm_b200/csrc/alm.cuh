// alm.cuh -- actuator-line forcing (src/rhs_lines.F90:47-483) on the fine
// level, in FP64.
//
//   k_alm_forces    one CTA.  First each thread takes blade elements (turbines,
//                   blades, elements in the reference's loop order): the
//                   velocity interpolated in the element's cell, the inflow
//                   angle, the two polar lookups (tables staged in shared
//                   memory when they fit).  Then, per element: the reference
//                   keeps a lookup's previous output when the angle of attack
//                   is outside a polar's range, so a lookup that found no
//                   interval takes the value of the last element before it
//                   whose lookup did; and the lift and drag forces
//                   (forces_lines).
//   k_alm_project   one thread per kernel node of every turbine: the Gaussian
//                   projection of its turbine's element forces, scaled by 1/J,
//                   added to the force field that K_R's first pass adds to
//                   rh(2:4).  Two turbines whose kernel lists share a node add
//                   to it in either order.
#pragma once
#include "common.cuh"

namespace desalm {

constexpr int ALM_SCR = 17;  // per-element values handed from k_alm_elements to k_alm_finish

// Device copy of one context's forcing tables (flat arrays, per-turbine offsets).
struct AlmDev {
  int n_tur;
  int E;                       // all elements of all turbines
  int im, jm, km;
  double vel_scale, length_scale, vel_infty;
  const int* tur_of;           // [E] turbine of element g
  const int* ker_tur;          // [all kernel nodes] turbine of each
  int nker_all;
  int nrows;                   // polar rows in all tables
  const int* meta;             // per turbine: nblades, nelems, nangles, nker, elem0, nodeoff, jkoff, keroff
  const double* par;           // per turbine: tsr, tur_rad, hub_rad
  const double* angle;         // per turbine azimuth (updated between physical steps)
  const int* node_index;       // concatenated per turbine: [nangles * nelems][3]
  const double* node_pos;      // [nangles * nelems][27]
  const double* disk_dat;      // per turbine [jm * km][8]
  const int* polar_b;          // per turbine [jm * km]
  const int* polar_a;
  const int* ker_index;        // concatenated [nker][3]
  const double* ker_pos;       // [nker][3]
  const double* ker_dat;       // [nker][4]
  const int* polar_off;
  const double* polar_rows;
  double* scr;                 // [E][ALM_SCR]
  double* forces;              // [E][6]
};

constexpr int ALM_META = 8;
constexpr double ALM_PI = 3.141592653589793;  // src/precision.F90:43
constexpr double ALM_RHO = 1178.62;

// Polar lookup (src/rhs_lines.F90:241-281); false when no interval holds aoa.
DESALM_DEV bool alm_polar(const double* rows, double aoa, double& cl, double& cd) {
  int idx = 0, counter = 1;
  double angle1 = 1000, angle2 = 1000, cl1 = 0, cd1 = 0, cl2 = 0, cd2 = 0;
  while (angle2 != -999.0) {
    if (counter == 1) {
      angle1 = rows[3 * idx]; cl1 = rows[3 * idx + 1]; cd1 = rows[3 * idx + 2]; ++idx;
    } else {
      angle1 = angle2; cl1 = cl2; cd1 = cd2;
    }
    angle2 = rows[3 * idx]; cl2 = rows[3 * idx + 1]; cd2 = rows[3 * idx + 2]; ++idx;
    if (aoa <= angle1) {
      angle2 = -999.0;
    } else if (angle2 == -999.0) {
    } else if (aoa <= angle2 && aoa >= angle1) {
      double m = (cl2 - cl1) / (angle2 - angle1);
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

template <class T, class W>
DESALM_DEV void alm_element(const AlmDev& A, const Lv<T, W>& L, const double* rows, int g) {
  const int t = A.tur_of[g];
  const int* M = A.meta + ALM_META * t;
  const int nblades = M[0], nelems = M[1], nangles = M[2];
  const int r = g - M[4];  // element within the turbine: (blade, element)
  const int bld = r / nelems + 1, elem = r % nelems + 1;
  const double tsr = A.par[3 * t], tur_rad = A.par[3 * t + 1];
  const double omega = (A.vel_infty * tsr) / tur_rad;
  const double dth = 2.0 * ALM_PI / double(nangles);
  double angle_aux = A.angle[t] + double(bld - 1) * 2.0 * ALM_PI / double(nblades);
  if (angle_aux > 2.0 * ALM_PI) angle_aux = angle_aux - 2.0 * ALM_PI;
  int nang = int(llround(angle_aux / dth)) + 1;
  if (nang > nangles) nang -= nangles;  // the reference reads one bin past its table here
  const long e = long(nang - 1) * nelems + (elem - 1);
  const int* I = A.node_index + 3L * M[5] + 3 * e;
  const int i = I[0], j = I[1], k = I[2];
  double* S = A.scr + ALM_SCR * long(g);
  // an element whose cell's lower corner is not an interior node is skipped,
  // as the reference skips cells outside its rank (src/rhs_lines.F90:166-167)
  if (i < 2 || i > A.im - 1 || j < 2 || j > A.jm - 1 || k < 2 || k > A.km - 1) {
    S[0] = 0.0; S[3] = 0.0; S[14] = 0.0;
    return;
  }
  const double* P = A.node_pos + 27L * M[5] + 27 * e;
  const double xf = P[0], yf = P[1], zf = P[2];
  const double x000 = P[3], z000 = P[5], x100 = P[6], y100 = P[7], y110 = P[10];
  const double x001 = P[15], z001 = P[17], x101 = P[18], y101 = P[19], y111 = P[22];
  const long jk = long(j - 1) + long(A.jm) * (k - 1);
  const double* D = A.disk_dat + 8L * M[6] + 8 * jk;
  const double radius = D[0] * A.length_scale, chord = D[4], twist = D[5], inter = D[6];
  auto id = [&](int ii, int jj, int kk) { return (ii - 1) + L.sj * (jj - 1) + L.sk * (kk - 1); };
  double v[3];
#pragma unroll
  for (int m = 1; m <= 3; ++m) {  // src/rhs_lines.F90:192-214
    const T* q = L.q[m];
    const double down = 1.0 / ((x100 - x000) * (y110 - y100)) *
                        ((x100 - xf) * ((y110 - yf) * (double(q[id(i, j, k)]) + double(q[id(i, j + 1, k)]))) +
                         (xf - x000) * ((yf - y100) * (double(q[id(i + 1, j, k)]) + double(q[id(i + 1, j + 1, k)]))));
    const double up =
        1.0 / ((x101 - x001) * (y111 - y101)) *
        ((x101 - xf) * ((y111 - yf) * (double(q[id(i, j, k + 1)]) + double(q[id(i, j + 1, k + 1)]))) +
         (xf - x001) * ((yf - y101) * (double(q[id(i + 1, j, k + 1)]) + double(q[id(i + 1, j + 1, k + 1)]))));
    v[m - 1] = down + (up - down) / (z001 - z000) * (zf - z000);
  }
  const double u_x = v[0] * A.vel_scale, u_y = v[1] * A.vel_scale, u_z = v[2] * A.vel_scale;
  const double u_theta = omega * radius + u_y * sin(angle_aux) - u_z * cos(angle_aux);
  const double phi = atan2(u_x, u_theta);
  const double aoa = phi * 180.0 / ALM_PI - twist;
  double cl_b = 0, cd_b = 0, cl_a = 0, cd_a = 0;
  const int pb = A.polar_b[long(M[6]) + jk], pa = A.polar_a[long(M[6]) + jk];
  const bool fb = alm_polar(rows + 3L * A.polar_off[pb], aoa, cl_b, cd_b);
  const bool fa = alm_polar(rows + 3L * A.polar_off[pa], aoa, cl_a, cd_a);
  S[0] = fb ? 1.0 : 0.0; S[1] = cl_b; S[2] = cd_b;
  S[3] = fa ? 1.0 : 0.0; S[4] = cl_a; S[5] = cd_a;
  S[6] = cos(phi); S[7] = sqrt(u_theta * u_theta + u_x * u_x); S[8] = chord; S[9] = inter; S[10] = sin(angle_aux);
  S[11] = xf; S[12] = yf; S[13] = zf; S[14] = 1.0; S[15] = sin(phi); S[16] = cos(angle_aux);
}

// The lookups' carry-forward and the forces of element g.
DESALM_DEV void alm_finish(const AlmDev& A, int g) {
  const double* S = A.scr + ALM_SCR * long(g);
  double* F = A.forces + 6L * g;
  if (S[14] == 0.0) {  // skipped element: forces_lines keeps its zeros
    for (int c = 0; c < 6; ++c) F[c] = 0.0;
    return;
  }
  // the last element at or before g whose lookup found an interval (skipped
  // elements make no lookup); none: the values start at zero
  double cl_b = 0, cd_b = 0, cl_a = 0, cd_a = 0;
  for (int h = g; h >= 0; --h) {
    const double* T = A.scr + ALM_SCR * long(h);
    if (T[0] != 0.0) { cl_b = T[1]; cd_b = T[2]; break; }
  }
  for (int h = g; h >= 0; --h) {
    const double* T = A.scr + ALM_SCR * long(h);
    if (T[3] != 0.0) { cl_a = T[4]; cd_a = T[5]; break; }
  }
  const double cphi = S[6], urel = S[7], chord = S[8], inter = S[9], sa = S[10], sphi = S[15], ca = S[16];
  const double cl = (cl_a - cl_b) * inter + cl_b;
  const double cd = (cd_a - cd_b) * inter + cd_b;
  const double fl = 0.5 * cl * ALM_RHO * (urel * urel) * chord;
  const double fd = 0.5 * cd * ALM_RHO * (urel * urel) * chord;
  F[0] = S[11]; F[1] = S[12]; F[2] = S[13];
  F[3] = fl * cphi + fd * sphi;
  F[4] = fl * sa * sphi - fd * sa * sphi;
  F[5] = fl * ca * sphi - fd * ca * cphi;
}

constexpr int ALM_SMEM_ROWS = 2048;  // polar rows staged in shared memory (48 KB)

template <class T, class W>
__global__ void __launch_bounds__(256) k_alm_forces(AlmDev A, Lv<T, W> L) {
  pdl_wait();
  __shared__ double srows[3 * ALM_SMEM_ROWS];
  const double* rows = A.polar_rows;
  if (A.nrows <= ALM_SMEM_ROWS) {
    for (int e = threadIdx.x; e < 3 * A.nrows; e += blockDim.x) srows[e] = A.polar_rows[e];
    __syncthreads();
    rows = srows;
  }
  for (int g = threadIdx.x; g < A.E; g += blockDim.x) alm_element(A, L, rows, g);
  __syncthreads();  // every element's lookups are written before any carry-forward reads them
  for (int g = threadIdx.x; g < A.E; g += blockDim.x) alm_finish(A, g);
}

// Kernel nodes (src/rhs_lines.F90:382-448) into falm[3][N].
template <class T, class W>
__global__ void k_alm_project(AlmDev A, Lv<T, W> L, double* falm) {
  pdl_wait();
  const int kn = blockIdx.x * blockDim.x + threadIdx.x;
  if (kn >= A.nker_all) return;
  const int t = A.ker_tur[kn];
  const int* M = A.meta + ALM_META * t;
  const int* I = A.ker_index + 3 * kn;
  if (I[0] < 2 || I[0] > A.im - 1 || I[1] < 2 || I[1] > A.jm - 1 || I[2] < 2 || I[2] > A.km - 1) return;
  const double ls = A.length_scale;
  const double radius = A.ker_dat[4 * kn] * ls;
  const double dV = A.ker_dat[4 * kn + 3] * (ls * ls * ls);
  const double hub = A.par[3 * t + 2], tur = A.par[3 * t + 1];
  if (!(radius > hub)) return;
  const double xk = A.ker_pos[3 * kn], yk = A.ker_pos[3 * kn + 1], zk = A.ker_pos[3 * kn + 2];
  const double deltar = fabs(tur - hub) / double(M[1]);
  const double eps = 2.0 * pow(dV, 1.0 / 3.0);
  const double kc = 1.0 / ((eps * eps * eps) * pow(ALM_PI, 3.0 / 2.0));
  const int ne = M[0] * M[1];
  double fx = 0, fy = 0, fz = 0;
  for (int e = 0; e < ne; ++e) {
    const double* F = A.forces + 6L * (M[4] + e);
    const double dx = xk - F[0], dy = yk - F[1], dz = zk - F[2];
    const double rdis = sqrt(dx * dx + dy * dy + dz * dz) * ls;
    const double ker = kc * exp(-(rdis * rdis) / (eps * eps));
    fx = fx + ker * F[3] * deltar;
    fy = fy + ker * F[4] * deltar;
    fz = fz + ker * F[5] * deltar;
  }
  const long l = (I[0] - 1) + long(L.sj) * (I[1] - 1) + long(L.sk) * (I[2] - 1);
  const double sc = (ls / (ALM_RHO * A.vel_scale * A.vel_scale)) * (1.0 / double(L.aj[l]));
  atomicAdd(falm + l, fx * sc);
  atomicAdd(falm + L.N + l, fy * sc);
  atomicAdd(falm + 2L * L.N + l, fz * sc);
}

}  // namespace desalm
