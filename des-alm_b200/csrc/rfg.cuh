// rfg.cuh -- synthetic inflow turbulence: the random flow generator of
// Smirnov, Shi & Celik (ASME J. Fluids Eng. 123, 2001) as the reference
// drives it (rfg_init / rfg_mpi_inlet_forcing, src/rfg_inlet.F90:47-173;
// initialize_rfg / rfg_vel, src/rfg.F90:42-374), in FP64.
//
//   k_rfg_prep    once per table set (desalm_rfg_set), one thread per inflow
//                 node: the eigen-decomposition of the node's velocity
//                 correlation tensor (the reference calls LAPACK ssyev for it
//                 on every node at every step, src/rfg.F90:286-313), the
//                 scaled coordinates x / eta and the wavenumber scales
//                 upsilon / c of get_iso_velocity (src/rfg.F90:271).
//   k_rfg_inlet   once per physical step, one thread per inflow node: the sum
//                 over the spectrum's modes (src/rfg.F90:274-282), the
//                 anti-diagonalisation (src/rfg.F90:315-327) and
//                 q(2:4) = um + v on the i = 1 plane (src/rfg_inlet.F90:161).
//                 The modes are staged in shared memory a chunk at a time and
//                 read by every thread of the CTA.
//
// Inflow nodes are j = 2..jm-1, k = 2..km-1 of i = 1 (1-based), the plane of
// a block without MPI neighbours (src/rfg_inlet.F90:121-133).
#pragma once
#include "common.cuh"

namespace desalm {

constexpr int RFG_MODE = 10;     // doubles per mode: p(3), q(3), k(3), omega
constexpr int RFG_NODE = 16;     // doubles per inflow node after k_rfg_prep
constexpr int RFG_CHUNK = 128;   // modes staged per pass (10 KB of shared memory)
constexpr int RFG_THREADS = 128;

// Device copy of one context's generator tables.
struct RfgDev {
  int nm;                  // modes N
  int im, jm, km;
  const double* modes;     // [nm][RFG_MODE]
  const double* um;        // [jm * km][3] mean velocity (rfg_um)
  const double* uij;       // [jm * km][6] r11 r12 r13 r22 r23 r33 (rfg_uij)
  const double* ts;        // [jm * km] time scale tau (rfg_t_ts)
  const double* ls;        // [jm * km] length scale eta (rfg_t_ls)
  double* node;            // [jm * km][RFG_NODE]: M (9, column-major), c (3), upsilon / c (3), spare
  double* x1;              // [jm * km][3] node coordinates over eta
};

// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Jacobi 1846; the rotation angle from tan(2 phi) = 2 a_pq / (a_qq - a_pp),
// taking the smaller root t = tan(phi)), then eigenvalues in ascending order
// as LAPACK's ?syev returns them, and each eigenvector signed so that its
// component of largest magnitude (the first of equal ones) is positive.  The
// reference takes whatever signs ssyev produces; the sign fixes the
// realisation, not its statistics (the modes are symmetric in distribution).
// r = (r11, r12, r13, r22, r23, r33); V column-major (V[3 * col + row]).
DESALM_HD inline void rfg_eig3(const double* r, double* w, double* V) {
  double A[3][3] = {{r[0], r[1], r[2]}, {r[1], r[3], r[4]}, {r[2], r[4], r[5]}};
  double U[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int sweep = 0; sweep < 32; ++sweep) {
    if (A[0][1] == 0.0 && A[0][2] == 0.0 && A[1][2] == 0.0) break;
    for (int pq = 0; pq < 3; ++pq) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      const double apq = A[p][q];
      if (apq == 0.0) continue;
      const double th = (A[q][q] - A[p][p]) / (2.0 * apq);
      const double at = th < 0.0 ? -th : th;
      const double t = at < 1.0e150 ? (th >= 0.0 ? 1.0 : -1.0) / (at + sqrt(th * th + 1.0)) : 0.5 / th;
      const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      for (int i = 0; i < 3; ++i) {   // A <- A J
        const double aip = A[i][p], aiq = A[i][q];
        A[i][p] = c * aip - s * aiq;
        A[i][q] = s * aip + c * aiq;
      }
      for (int i = 0; i < 3; ++i) {   // A <- J^T A
        const double api = A[p][i], aqi = A[q][i];
        A[p][i] = c * api - s * aqi;
        A[q][i] = s * api + c * aqi;
      }
      A[p][q] = A[q][p] = 0.0;
      for (int i = 0; i < 3; ++i) {   // U <- U J
        const double uip = U[i][p], uiq = U[i][q];
        U[i][p] = c * uip - s * uiq;
        U[i][q] = s * uip + c * uiq;
      }
    }
  }
  int o[3] = {0, 1, 2};
  double d[3] = {A[0][0], A[1][1], A[2][2]};
  for (int a = 0; a < 2; ++a)        // ascending, stable
    for (int b = 0; b < 2 - a; ++b)
      if (d[o[b + 1]] < d[o[b]]) { const int tmp = o[b]; o[b] = o[b + 1]; o[b + 1] = tmp; }
  for (int col = 0; col < 3; ++col) {
    const int src = o[col];
    w[col] = d[src];
    int big = 0;
    for (int i = 1; i < 3; ++i) {
      const double ai = U[i][src] < 0.0 ? -U[i][src] : U[i][src];
      const double ab = U[big][src] < 0.0 ? -U[big][src] : U[big][src];
      if (ai > ab) big = i;
    }
    const double sg = U[big][src] < 0.0 ? -1.0 : 1.0;
    for (int i = 0; i < 3; ++i) V[3 * col + i] = sg * U[i][src];
  }
}

// Inflow node number n -> (j, k), 0-based, interior of the i = 1 plane.
DESALM_DEV void rfg_jk(int n, int jm, int& j, int& k) {
  j = 1 + n % (jm - 2);
  k = 1 + n / (jm - 2);
}

__global__ void k_rfg_prep(RfgDev R, const double* x, const double* y, const double* z, int* bad) {
  pdl_wait();
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= (R.jm - 2) * (R.km - 2)) return;
  int j, k;
  rfg_jk(n, R.jm, j, k);
  const int jk = j + R.jm * k;
  const long l = (long)R.im * jk;        // node (1, j, k)
  double w[3], M[9];
  rfg_eig3(R.uij + 6L * jk, w, M);
  const double tau = R.ts[jk], eta = R.ls[jk];
  const bool ok = w[0] > 0.0 && tau > 0.0 && eta > 0.0 && tau < INFINITY && eta < INFINITY && w[2] < INFINITY;
  if (!ok) atomicAdd(bad, 1);
  double* o = R.node + (long)RFG_NODE * jk;
  for (int t = 0; t < 9; ++t) o[t] = M[t];
  const double upsilon = eta / tau;       // src/rfg.F90:366
  for (int d = 0; d < 3; ++d) {
    const double c = sqrt(w[d]);          // src/rfg.F90:311
    o[9 + d] = c;
    o[12 + d] = upsilon / c;              // k_scale = k upsilon / c (src/rfg.F90:271)
  }
  o[15] = 0.0;
  double* xo = R.x1 + 3L * jk;            // x1 = x / eta (src/rfg.F90:365)
  xo[0] = x[l] / eta;
  xo[1] = y[l] / eta;
  xo[2] = z[l] / eta;
}

__global__ void __launch_bounds__(RFG_THREADS) k_rfg_inlet(RfgDev R, double time, double* qu, double* qv, double* qw) {
  __shared__ double sm[RFG_CHUNK * RFG_MODE];
  pdl_wait();
  const int nn = (R.jm - 2) * (R.km - 2);
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = n < nn;
  int j = 1, k = 1;
  if (live) rfg_jk(n, R.jm, j, k);
  const int jk = j + R.jm * k;
  double a0 = 0, a1 = 0, a2 = 0, x0 = 0, x1 = 0, x2 = 0, t1 = 0;
  if (live) {
    const double* o = R.node + (long)RFG_NODE * jk;
    a0 = o[12]; a1 = o[13]; a2 = o[14];
    const double* xo = R.x1 + 3L * jk;
    x0 = xo[0]; x1 = xo[1]; x2 = xo[2];
    t1 = time / R.ts[jk];                 // src/rfg.F90:364
  }
  double s0 = 0, s1 = 0, s2 = 0;
  for (int m0 = 0; m0 < R.nm; m0 += RFG_CHUNK) {
    const int cnt = min(RFG_CHUNK, R.nm - m0);
    __syncthreads();
    for (int e = threadIdx.x; e < cnt * RFG_MODE; e += blockDim.x) sm[e] = R.modes[(long)m0 * RFG_MODE + e];
    __syncthreads();
    if (live) {
      for (int m = 0; m < cnt; ++m) {
        const double* md = sm + m * RFG_MODE;
        // term1 = k_scale . x1 + omega t1 (src/rfg.F90:277-278)
        const double term = (md[6] * a0) * x0 + (md[7] * a1) * x1 + (md[8] * a2) * x2 + md[9] * t1;
        double sn, cs;
        sincos(term, &sn, &cs);
        s0 += md[0] * cs + md[3] * sn;
        s1 += md[1] * cs + md[4] * sn;
        s2 += md[2] * cs + md[5] * sn;
      }
    }
  }
  if (!live) return;
  const double cst = sqrt(2.0 / (double)R.nm);   // src/rfg.F90:281
  const double* o = R.node + (long)RFG_NODE * jk;
  const double v0 = o[9] * (cst * s0), v1 = o[10] * (cst * s1), v2 = o[11] * (cst * s2);  // c v (src/rfg.F90:324)
  const double* um = R.um + 3L * jk;
  const long l = (long)R.im * jk;
  qu[l] = um[0] + (o[0] * v0 + o[3] * v1 + o[6] * v2);   // matmul(m, v) (src/rfg.F90:325)
  qv[l] = um[1] + (o[1] * v0 + o[4] * v1 + o[7] * v2);
  qw[l] = um[2] + (o[2] * v0 + o[5] * v1 + o[8] * v2);
}

}  // namespace desalm
