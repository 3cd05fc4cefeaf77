// modal.cuh -- eigenvector matrices of the diagonalised approximate
// factorisation, rebuilt per node from the metrics instead of being stored.
//
// For a metric vector (c1, c2, c3) and sigma = sqrt(beta * alpha) the
// reference builds M (= Ma, Mb or Mc) and its analytic inverse
// (src/rhs_modal_matrices.F90:64-259).  The same closed forms are evaluated
// here, in the same operation order.
#pragma once
#include "common.cuh"

namespace desalm {

template <class T>
struct M4 {
  T a[4][4];
};

// forward matrix M of one direction (src/rhs_modal_matrices.F90:112-132)
template <class T>
DESALM_DEV void modal_fwd(T c1, T c2, T c3, T sigma, M4<T>& M) {
  const T two = T(2);
  T g = c1 * c1 + c2 * c2 + c3 * c3;
  T sg = sqrt(g);
  T dd = c2 - c3;
  T s = sqrt(two * g + dd * dd);
  M.a[0][0] = T(0); M.a[0][1] = T(0); M.a[0][2] = sigma; M.a[0][3] = sigma;
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
}

// analytic inverse (src/rhs_modal_matrices.F90:134-158)
template <class T>
DESALM_DEV void modal_inv(T c1, T c2, T c3, T sigma, M4<T>& Mi) {
  const T one = T(1), two = T(2), pt5 = T(0.5);
  T c1s = c1 * c1, c2s = c2 * c2, c3s = c3 * c3;
  T g = c1s + c2s + c3s;
  T sg = sqrt(g);
  T dd = c2 - c3;
  T s = sqrt(two * g + dd * dd);
  T dm = g + two * c2 * c3 + c1 * c1;
  T r1 = c2 + c3, r2 = c2 - c3, r3 = c2s - c3s;
  Mi.a[0][0] = T(0);
  Mi.a[0][1] = -s * (c2 + c3) / dm;
  Mi.a[0][2] = s * c1 / dm;
  Mi.a[0][3] = Mi.a[0][2];
  T ssgd = s / sg / dm;
  T sgd2 = one / sg / dm / two;
  Mi.a[1][0] = T(0);
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

// C = A * B with the k-sum in order (gfortran's matmul)
template <class T>
DESALM_DEV void mm4(const M4<T>& A, const M4<T>& B, M4<T>& C) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      T s = A.a[i][0] * B.a[0][j];
      s = s + A.a[i][1] * B.a[1][j];
      s = s + A.a[i][2] * B.a[2][j];
      s = s + A.a[i][3] * B.a[3][j];
      C.a[i][j] = s;
    }
}

template <class T, class U>
DESALM_DEV void mv4(const M4<T>& A, const U* r, U* rp) {
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    T s = A.a[i][0] * T(r[0]);
    s = s + A.a[i][1] * T(r[1]);
    s = s + A.a[i][2] * T(r[2]);
    s = s + A.a[i][3] * T(r[3]);
    rp[i] = U(s);
  }
}

// sigma and theta of a node (src/rhs_modal_matrices.F90:82-84)
template <class T>
DESALM_DEV void sigma_theta(T dtau, const Par& P, T& sigma, T& theta) {
  T alpha = T(1) + T(P.es) * T(1.5) * dtau / T(P.delti);
  sigma = sqrt(T(P.beta) * alpha);
  theta = sqrt(T(P.beta) / alpha);
}

// Ma^-1 of a node
template <class T, class W>
DESALM_DEV void mat_mai(const Lv<T, W>& L, const Par& P, int l, M4<T>& A) {
  T s, t;
  sigma_theta(L.dtau[l], P, s, t);
  modal_inv(L.csi[0][l], L.csi[1][l], L.csi[2][l], s, A);
}
// N1^-1 = Mb^-1 Ma
template <class T, class W>
DESALM_DEV void mat_n1i(const Lv<T, W>& L, const Par& P, int l, M4<T>& A) {
  T s, t;
  sigma_theta(L.dtau[l], P, s, t);
  M4<T> ma, mbi;
  modal_fwd(L.csi[0][l], L.csi[1][l], L.csi[2][l], s, ma);
  modal_inv(L.eta[0][l], L.eta[1][l], L.eta[2][l], s, mbi);
  mm4(mbi, ma, A);
}
// N2^-1 = Mc^-1 Mb
template <class T, class W>
DESALM_DEV void mat_n2i(const Lv<T, W>& L, const Par& P, int l, M4<T>& A) {
  T s, t;
  sigma_theta(L.dtau[l], P, s, t);
  M4<T> mb, mci;
  modal_fwd(L.eta[0][l], L.eta[1][l], L.eta[2][l], s, mb);
  modal_inv(L.zet[0][l], L.zet[1][l], L.zet[2][l], s, mci);
  mm4(mci, mb, A);
}
// Mc
template <class T, class W>
DESALM_DEV void mat_mc(const Lv<T, W>& L, const Par& P, int l, M4<T>& A) {
  T s, t;
  sigma_theta(L.dtau[l], P, s, t);
  modal_fwd(L.zet[0][l], L.zet[1][l], L.zet[2][l], s, A);
}

// Application of M and M^-1 to a vector in precision C, using the structure
// of the closed forms above: row 0 of M is (0, 0, sigma, sigma) and its last
// two columns are opposite; row 0 of M^-1 repeats its last entry and rows 2
// and 3 share all but the sign of their last three entries; every entry is a
// polynomial in (c1, c2, c3) times one of 1/s, 1/sqrt(g), 1/(s sqrt(g)) or
// 1/dm.  With those factors formed once, M x costs two square roots, two
// divisions and about twenty multiplies instead of the 4x4 matrix's twelve
// divisions and sixteen multiplies; the result equals mv4 of the matrix up to
// rounding.
template <class C>
DESALM_DEV void mfwd_apply(C c1, C c2, C c3, C sigma, const C x[4], C y[4]) {
  const C g = c1 * c1 + c2 * c2 + c3 * c3;
  const C rsg = C(1) / sqrt(g);
  const C dd = c2 - c3;
  const C ris = C(1) / sqrt(C(2) * g + dd * dd);
  const C risg = ris * rsg;
  const C xd = x[2] - x[3];
  const C x0s = ris * x[0], x1s = risg * x[1], xds = rsg * xd;
  y[0] = sigma * (x[2] + x[3]);
  y[1] = -(c2 + c3) * x0s + c1 * (c3 - c2) * x1s + c1 * xds;
  y[2] = c1 * x0s + (g + c2 * (c3 - c2)) * x1s + c2 * xds;
  y[3] = c1 * x0s - (g - c3 * (c3 - c2)) * x1s + c3 * xds;
}
template <class C>
DESALM_DEV void minv_apply(C c1, C c2, C c3, C sigma, const C x[4], C y[4]) {
  const C c1s = c1 * c1, c2s = c2 * c2, c3s = c3 * c3;
  const C g = c1s + c2s + c3s;
  const C rsg = C(1) / sqrt(g);
  const C dd = c2 - c3;
  const C s = sqrt(C(2) * g + dd * dd);
  const C rdm = C(1) / (g + C(2) * c2 * c3 + c1s);
  const C ssgd = s * rsg * rdm, sgd2 = C(0.5) * rsg * rdm;
  const C r1 = c2 + c3, r2 = c2 - c3, r3 = c2s - c3s;
  y[0] = s * rdm * (-(c2 + c3) * x[1] + c1 * (x[2] + x[3]));
  y[1] = ssgd * (c1 * (c3 - c2) * x[1] + (c2 * c3 + c1s + c3s) * x[2] - (c2 * c3 + c1s + c2s) * x[3]);
  const C e = sgd2 * (c1 * (C(2) * g + C(2) * c2 * c3 - c2s - c3s) * x[1] + (g * r1 + c1s * r2 + c3 * r3) * x[2] +
                      (g * r1 - c1s * r2 - c2 * r3) * x[3]);
  const C h0 = C(0.5) / sigma * x[0];
  y[2] = h0 + e;
  y[3] = h0 - e;
}

}  // namespace desalm
