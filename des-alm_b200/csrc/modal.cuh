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

// The same matrices evaluated in precision C (metrics and dtau read in the
// level's state precision and rounded to C): the line-sweep precision in
// MIXED mode, where the transforms belong to the FP32 preconditioner.
template <class C, class T, class W>
DESALM_DEV void sigma_c(const Lv<T, W>& L, const Par& P, int l, C& sigma) {
  T s, t;
  sigma_theta(L.dtau[l], P, s, t);
  sigma = C(s);
}
template <class C, class T, class W>
DESALM_DEV void mat_mai_c(const Lv<T, W>& L, const Par& P, int l, M4<C>& A) {
  C s; sigma_c(L, P, l, s);
  modal_inv(C(L.csi[0][l]), C(L.csi[1][l]), C(L.csi[2][l]), s, A);
}
template <class C, class T, class W>
DESALM_DEV void mat_n1i_c(const Lv<T, W>& L, const Par& P, int l, M4<C>& A) {
  C s; sigma_c(L, P, l, s);
  M4<C> ma, mbi;
  modal_fwd(C(L.csi[0][l]), C(L.csi[1][l]), C(L.csi[2][l]), s, ma);
  modal_inv(C(L.eta[0][l]), C(L.eta[1][l]), C(L.eta[2][l]), s, mbi);
  mm4(mbi, ma, A);
}
template <class C, class T, class W>
DESALM_DEV void mat_n2i_c(const Lv<T, W>& L, const Par& P, int l, M4<C>& A) {
  C s; sigma_c(L, P, l, s);
  M4<C> mb, mci;
  modal_fwd(C(L.eta[0][l]), C(L.eta[1][l]), C(L.eta[2][l]), s, mb);
  modal_inv(C(L.zet[0][l]), C(L.zet[1][l]), C(L.zet[2][l]), s, mci);
  mm4(mci, mb, A);
}
template <class C, class T, class W>
DESALM_DEV void mat_mc_c(const Lv<T, W>& L, const Par& P, int l, M4<C>& A) {
  C s; sigma_c(L, P, l, s);
  modal_fwd(C(L.zet[0][l]), C(L.zet[1][l]), C(L.zet[2][l]), s, A);
}

}  // namespace desalm
