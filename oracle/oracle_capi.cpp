// oracle_capi.cpp -- extern "C" entry points of the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (see oracle_core.hpp).  The entry points mirror
// include/desalm.h with the prefix desalm_oracle_; desalm_oracle_init takes
// the real type (8 = FP64 oracle, 4 = FP32 mirror of the reference's own
// arithmetic).
#include "oracle_core.hpp"
#include <malloc.h>
#include <memory>

namespace {

struct Base {
  virtual ~Base() {}
  std::string err;
  virtual int set_grid(const double*, const double*, const double*, const double*) = 0;
  virtual int set_state(const double*, const double*, const double*, const double*) = 0;
  virtual int get_state(double*, double*, double*, double*) = 0;
  virtual int get_field(int, int, double*) = 0;
  virtual int set_field(int, int, const double*) = 0;
  virtual int dims(int, int*) = 0;
  virtual int solver_daf(int, int, int) = 0;
  virtual int nlevel(int) = 0;
  virtual int prolong(int) = 0;
  virtual int residual(int, double*) = 0;
  virtual int bcond() = 0;
  virtual int des_eddy() = 0;
  virtual int kw_eddy() = 0;
  virtual int set_omega(const double*, const double*, const double*) = 0;
  virtual int get_omega(double*, double*, double*) = 0;
  virtual int kw_config(double, double) = 0;
  virtual int conservation() = 0;
  virtual int wall_functions() = 0;
  virtual int save_qold() = 0;
  virtual int begin_step() = 0;
  virtual int pseudo_iteration(desalm_step_report*) = 0;
  virtual int alm_set(const desalm_alm*) = 0;
  virtual int alm_angle(int, double) = 0;
  virtual int alm_get(int, double*) = 0;
  virtual int mg_driver(desalm_step_report*) = 0;
  virtual void phase_times(double*) = 0;
  virtual int outlet_rhs(double*) = 0;
};

template <class R>
struct Impl : Base {
  orc::Solver<R> s;
  explicit Impl(const desalm_case& c) : s(c) {}
  bool lvl_ok(int n) { return n >= 1 && n <= s.ng; }
  std::vector<R>* field(int n, int f) {
    orc::Level<R>& G = s.L[n - 1];
    if (f >= DESALM_F_Q && f < DESALM_F_Q + 5) return &G.q[f - DESALM_F_Q];
    if (f >= DESALM_F_QN && f < DESALM_F_QN + 5) return &G.qn[f - DESALM_F_QN];
    if (f >= DESALM_F_QNM1 && f < DESALM_F_QNM1 + 5) return &G.qnm1[f - DESALM_F_QNM1];
    if (f >= DESALM_F_QOLD && f < DESALM_F_QOLD + 5) return &G.qold[f - DESALM_F_QOLD];
    if (f >= DESALM_F_RH && f < DESALM_F_RH + 4) return &G.rh[f - DESALM_F_RH];
    if (f >= DESALM_F_PK && f < DESALM_F_PK + 4) return &G.pk[f - DESALM_F_PK];
    if (f >= DESALM_F_CSI && f < DESALM_F_CSI + 3) return &G.csi[f - DESALM_F_CSI];
    if (f >= DESALM_F_ETA && f < DESALM_F_ETA + 3) return &G.eta[f - DESALM_F_ETA];
    if (f >= DESALM_F_ZET && f < DESALM_F_ZET + 3) return &G.zet[f - DESALM_F_ZET];
    switch (f) {
      case DESALM_F_AJ: return &G.aj;
      case DESALM_F_NUT: return &G.nut;
      case DESALM_F_DTAU: return &G.dtau;
      case DESALM_F_DTEV: return &G.dtev;
      case DESALM_F_WD: return &G.wd;
      case DESALM_F_X: return &G.x;
      case DESALM_F_Y: return &G.y;
      case DESALM_F_Z: return &G.z;
    }
    return nullptr;
  }
  int set_grid(const double* x, const double* y, const double* z, const double* wd) override {
    s.set_grid(x, y, z, wd);
    return 0;
  }
  int set_state(const double* q, const double* qn, const double* qnm1, const double* nut) override {
    orc::Level<R>& F = s.L[0];
    for (long l = 0; l < F.N; ++l)
      for (int m = 0; m < 5; ++m) {
        F.q[m][l] = R(q[5 * l + m]);
        F.qn[m][l] = qn ? R(qn[5 * l + m]) : R(0);
        F.qnm1[m][l] = qnm1 ? R(qnm1[5 * l + m]) : R(0);
      }
    for (long l = 0; l < F.N; ++l) F.nut[l] = nut ? R(nut[l]) : R(0);
    s.have_state = true;
    return 0;
  }
  int get_state(double* q, double* qn, double* qnm1, double* nut) override {
    orc::Level<R>& F = s.L[0];
    for (long l = 0; l < F.N; ++l)
      for (int m = 0; m < 5; ++m) {
        if (q) q[5 * l + m] = double(F.q[m][l]);
        if (qn) qn[5 * l + m] = double(F.qn[m][l]);
        if (qnm1) qnm1[5 * l + m] = double(F.qnm1[m][l]);
      }
    if (nut) for (long l = 0; l < F.N; ++l) nut[l] = double(F.nut[l]);
    return 0;
  }
  int get_field(int n, int f, double* out) override {
    if (!lvl_ok(n)) return DESALM_EINVAL;
    std::vector<R>* v = field(n, f);
    if (!v) return DESALM_EINVAL;
    for (size_t l = 0; l < v->size(); ++l) out[l] = double((*v)[l]);
    return 0;
  }
  int set_field(int n, int f, const double* in) override {
    if (!lvl_ok(n)) return DESALM_EINVAL;
    std::vector<R>* v = field(n, f);
    if (!v) return DESALM_EINVAL;
    for (size_t l = 0; l < v->size(); ++l) (*v)[l] = R(in[l]);
    return 0;
  }
  // The fine level's first-pass residual, then the outlet plane's
  // (mg_brhs + nonreflect_ibc); out = rh(1:4) on the plane i = im, [4][jm*km].
  int outlet_rhs(double* out) override {
    orc::Level<R>& G = s.L[0];
    for (int m = 0; m < 4; ++m) std::fill(G.rh[m].begin(), G.rh[m].end(), R(0));
    s.residual(G, 0, true, 0);
    s.outlet_rhs(G);
    const long P = (long)G.jm * G.km;
    for (int m = 0; m < 4; ++m)
      for (int k = 1; k <= G.km; ++k)
        for (int j = 1; j <= G.jm; ++j)
          out[m * P + (j - 1) + (long)G.jm * (k - 1)] = double(G.rh[m][G.id(G.im, j, k)]);
    return 0;
  }
  int dims(int n, int* d) override {
    if (!lvl_ok(n)) return DESALM_EINVAL;
    d[0] = s.L[n - 1].im; d[1] = s.L[n - 1].jm; d[2] = s.L[n - 1].km;
    return 0;
  }
  int alm_set(const desalm_alm* a) override {
    s.alm.clear();
    s.alm_on = a && a->n_tur > 0;
    if (!s.alm_on) return 0;
    const int jm = s.L[0].jm, km = s.L[0].km;
    s.alm_vel_infty = R(a->vel_infty);
    s.alm_length_scale = R(a->length_scale);
    s.polar_off.assign(a->polar_offset, a->polar_offset + a->npolar);
    s.polar_cnt.assign(a->polar_count, a->polar_count + a->npolar);
    long nrows = 0;
    for (int p = 0; p < a->npolar; ++p) nrows = std::max<long>(nrows, a->polar_offset[p] + a->polar_count[p]);
    s.polar_rows.resize(3 * nrows);
    for (long r = 0; r < 3 * nrows; ++r) s.polar_rows[r] = R(a->polar_rows[r]);
    for (int t = 0; t < a->n_tur; ++t) {
      const desalm_alm_turbine& T = a->tur[t];
      typename orc::Solver<R>::AlmTur U;
      U.nblades = T.nblades; U.nelems = T.nelems; U.nangles = T.nangles; U.nker = T.nker;
      U.tsr = R(T.tsr); U.tur_rad = R(T.tur_rad); U.hub_rad = R(T.hub_rad); U.angle = R(T.angle);
      const long ne = long(T.nangles) * T.nelems;
      U.node_index.assign(T.node_index, T.node_index + 3 * ne);
      U.node_pos.resize(27 * ne);
      for (long e = 0; e < 27 * ne; ++e) U.node_pos[e] = R(T.node_pos[e]);
      U.disk_dat.resize(8L * jm * km);
      for (long e = 0; e < 8L * jm * km; ++e) U.disk_dat[e] = R(T.disk_dat[e]);
      U.polar_b.assign(T.polar_b, T.polar_b + long(jm) * km);
      U.polar_a.assign(T.polar_a, T.polar_a + long(jm) * km);
      U.ker_index.assign(T.ker_index, T.ker_index + 3L * T.nker);
      U.ker_pos.resize(3L * T.nker);
      U.ker_dat.resize(4L * T.nker);
      for (long e = 0; e < 3L * T.nker; ++e) U.ker_pos[e] = R(T.ker_pos[e]);
      for (long e = 0; e < 4L * T.nker; ++e) U.ker_dat[e] = R(T.ker_dat[e]);
      s.alm.push_back(std::move(U));
    }
    return 0;
  }
  int alm_angle(int t, double angle) override {
    if (t < 1 || t > (int)s.alm.size()) return DESALM_EINVAL;
    s.alm[t - 1].angle = R(angle);
    return 0;
  }
  int alm_get(int what, double* out) override {
    if (what == DESALM_ALM_FORCES) {
      for (size_t e = 0; e < s.forces_lines.size(); ++e) out[e] = double(s.forces_lines[e]);
      return 0;
    }
    if (what == DESALM_ALM_FIELD) {
      const long N = s.L[0].N;
      for (int d = 0; d < 3; ++d)
        for (long l = 0; l < N; ++l) out[d * N + l] = s.falm[d].empty() ? 0.0 : double(s.falm[d][l]);
      return 0;
    }
    return DESALM_EINVAL;
  }
  int solver_daf(int n, int recalc, int itr) override {
    if (!lvl_ok(n)) return DESALM_EINVAL;
    s.solver_daf(n - 1, recalc, itr);
    return 0;
  }
  int nlevel(int n) override {
    if (n < 2 || n > s.ng) return DESALM_EINVAL;
    s.mg_nlevel(n - 1);
    return 0;
  }
  int prolong(int n) override {
    if (n < 1 || n >= s.ng) return DESALM_EINVAL;
    s.mg_prolong(n - 1);
    return 0;
  }
  int residual(int n, double* r) override {
    if (!lvl_ok(n)) return DESALM_EINVAL;
    s.mg_residual(n - 1, r);
    return 0;
  }
  int bcond() override { s.bcond_fm(); return 0; }
  int des_eddy() override { s.des_eddy(); return 0; }
  int kw_eddy() override {
    if (s.c.turbulence != 2) return DESALM_EINVAL;
    s.kw_eddy();
    return 0;
  }
  int set_omega(const double* w, const double* wn, const double* wnm1) override {
    if (s.c.turbulence != 2 || !w) return DESALM_EINVAL;
    for (long l = 0; l < s.L[0].N; ++l) {
      s.om[l] = R(w[l]);
      s.omn[l] = wn ? R(wn[l]) : R(0);
      s.omnm1[l] = wnm1 ? R(wnm1[l]) : R(0);
    }
    return 0;
  }
  int get_omega(double* w, double* wn, double* wnm1) override {
    if (s.c.turbulence != 2) return DESALM_EINVAL;
    for (long l = 0; l < s.L[0].N; ++l) {
      if (w) w[l] = double(s.om[l]);
      if (wn) wn[l] = double(s.omn[l]);
      if (wnm1) wnm1[l] = double(s.omnm1[l]);
    }
    return 0;
  }
  int kw_config(double ckin, double cein) override {
    if (!(ckin >= 0) || !(cein > 0)) return DESALM_EINVAL;
    s.ckin = R(ckin);
    s.cein = R(cein);
    return 0;
  }
  int conservation() override { s.conservation(); return 0; }
  int wall_functions() override { s.wall_functions(); return 0; }
  int save_qold() override { s.save_qold(); return 0; }
  int begin_step() override { s.begin_step(); return 0; }
  int pseudo_iteration(desalm_step_report* rep) override {
    double res[5];
    long p0 = s.pivots;
    bool conv = s.pseudo_iteration(res);
    if (rep) {
      rep->iterations = s.itc;
      rep->converged = conv ? 1 : 0;
      for (int m = 0; m < 5; ++m) { rep->residual[m] = res[m]; rep->init_residual[m] = double(s.init_resd[m]); }
      rep->pivots = (int)(s.pivots - p0);
    }
    return 0;
  }
  int mg_driver(desalm_step_report* rep) override {
    s.begin_step();
    long p0 = s.pivots;
    double res[5] = {0, 0, 0, 0, 0};
    bool conv = false;
    for (int it = 1; it <= s.c.itmax; ++it) {
      conv = s.pseudo_iteration(res);
      if (conv) break;
    }
    if (rep) {
      rep->iterations = s.itc;
      rep->converged = conv ? 1 : 0;
      for (int m = 0; m < 5; ++m) { rep->residual[m] = res[m]; rep->init_residual[m] = double(s.init_resd[m]); }
      rep->pivots = (int)(s.pivots - p0);
    }
    return 0;
  }
  void phase_times(double* t) override { for (int i = 0; i < 8; ++i) t[i] = s.phase_s[i]; }
};

int check_case(const desalm_case* c, std::string& why) {
  if (!c) { why = "null case"; return DESALM_EINVAL; }
  if (c->ng < 1 || c->ng > 4) { why = "ng must be 1..4"; return DESALM_EINVAL; }
  if (c->im < 5 || c->jm < 5 || c->km < 5) { why = "each extent must be >= 5"; return DESALM_EINVAL; }
  if (c->turbulence < 0 || c->turbulence > 2) { why = "turbulence must be 0, 1 or 2"; return DESALM_EINVAL; }
  return 0;
}

}  // namespace

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

int desalm_oracle_init(const desalm_case* c, int real_bytes, void** out) {
  // The restatement allocates its full-size temporaries per call, as the
  // reference's routines do.  Keep freed blocks in the heap instead of
  // returning them to the system, so that the next call reuses pages that
  // are already mapped (large-grid runs otherwise spend much of their time
  // in page faults).
  mallopt(M_MMAP_MAX, 0);
  mallopt(M_TRIM_THRESHOLD, 0x7fffffff);
  std::string why;
  int rc = check_case(c, why);
  if (rc) return rc;
  try {
    Base* b = real_bytes == 4 ? (Base*)new Impl<float>(*c) : (Base*)new Impl<double>(*c);
    *out = b;
  } catch (...) {
    return DESALM_ENOMEM;
  }
  return 0;
}
void desalm_oracle_destroy(void* ctx) { delete (Base*)ctx; }
// Host threads the oracle's parallel loops use (1 in a serial build).
int desalm_oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
int desalm_oracle_level_dims(void* ctx, int n, int* d) { return ((Base*)ctx)->dims(n, d); }
int desalm_oracle_set_grid(void* ctx, const double* x, const double* y, const double* z, const double* wd) {
  return ((Base*)ctx)->set_grid(x, y, z, wd);
}
int desalm_oracle_set_state(void* ctx, const double* q, const double* qn, const double* qnm1, const double* nut) {
  return ((Base*)ctx)->set_state(q, qn, qnm1, nut);
}
int desalm_oracle_get_state(void* ctx, double* q, double* qn, double* qnm1, double* nut) {
  return ((Base*)ctx)->get_state(q, qn, qnm1, nut);
}
int desalm_oracle_get_field(void* ctx, int n, int f, double* out) { return ((Base*)ctx)->get_field(n, f, out); }
int desalm_oracle_set_field(void* ctx, int n, int f, const double* in) { return ((Base*)ctx)->set_field(n, f, in); }
int desalm_oracle_solver_daf(void* ctx, int n, int recalc, int itr) { return ((Base*)ctx)->solver_daf(n, recalc, itr); }
int desalm_oracle_mg_nlevel(void* ctx, int n) { return ((Base*)ctx)->nlevel(n); }
int desalm_oracle_mg_prolong(void* ctx, int n) { return ((Base*)ctx)->prolong(n); }
int desalm_oracle_mg_residual(void* ctx, int n, double* r) { return ((Base*)ctx)->residual(n, r); }
int desalm_oracle_bcond_fm(void* ctx) { return ((Base*)ctx)->bcond(); }
int desalm_oracle_des_eddy(void* ctx) { return ((Base*)ctx)->des_eddy(); }
int desalm_oracle_kw_eddy(void* ctx) { return ((Base*)ctx)->kw_eddy(); }
int desalm_oracle_set_omega(void* ctx, const double* w, const double* wn, const double* wnm1) {
  return ((Base*)ctx)->set_omega(w, wn, wnm1);
}
int desalm_oracle_get_omega(void* ctx, double* w, double* wn, double* wnm1) {
  return ((Base*)ctx)->get_omega(w, wn, wnm1);
}
int desalm_oracle_kw_config(void* ctx, double ckin, double cein) { return ((Base*)ctx)->kw_config(ckin, cein); }
int desalm_oracle_conservation(void* ctx) { return ((Base*)ctx)->conservation(); }
int desalm_oracle_wall_functions(void* ctx) { return ((Base*)ctx)->wall_functions(); }
int desalm_oracle_save_qold(void* ctx) { return ((Base*)ctx)->save_qold(); }
int desalm_oracle_begin_step(void* ctx) { return ((Base*)ctx)->begin_step(); }
int desalm_oracle_pseudo_iteration(void* ctx, desalm_step_report* r) { return ((Base*)ctx)->pseudo_iteration(r); }
int desalm_oracle_mg_driver(void* ctx, desalm_step_report* r) { return ((Base*)ctx)->mg_driver(r); }
void desalm_oracle_phase_times(void* ctx, double* t) { ((Base*)ctx)->phase_times(t); }
int desalm_oracle_alm_set(void* ctx, const desalm_alm* a) { return ((Base*)ctx)->alm_set(a); }
int desalm_oracle_alm_set_angle(void* ctx, int t, double angle) { return ((Base*)ctx)->alm_angle(t, angle); }
int desalm_oracle_alm_get(void* ctx, int what, double* out) { return ((Base*)ctx)->alm_get(what, out); }
int desalm_oracle_outlet_rhs(void* ctx, double* out) { return ((Base*)ctx)->outlet_rhs(out); }

// Standalone LAPACK-style tridiagonal solve (SGTSV restatement) for tests.
int desalm_oracle_gtsv(int n, int nrhs, double* dl, double* d, double* du, double* b, int ldb, long* npiv) {
  return orc::gtsv<double>(n, nrhs, dl, d, du, b, ldb, npiv);
}
// Modal matrices of one node (Ma^-1, N1^-1, N2^-1, Mc and the forward
// matrices Ma, Mb, Mc) for the analytic-inverse tests: out[7][4][4].
void desalm_oracle_modal(const double* csi, const double* eta, const double* zet, double sigma, double* out) {
  orc::M4<double> ma, mai, mb, mbi, mc, mci;
  orc::modal_pair(csi[0], csi[1], csi[2], sigma, ma, mai);
  orc::modal_pair(eta[0], eta[1], eta[2], sigma, mb, mbi);
  orc::modal_pair(zet[0], zet[1], zet[2], sigma, mc, mci);
  orc::M4<double> n1i = orc::mm4(mbi, ma), n2i = orc::mm4(mci, mb);
  const orc::M4<double>* all[7] = {&mai, &n1i, &n2i, &mc, &ma, &mb, &mci};
  for (int t = 0; t < 7; ++t)
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) out[t * 16 + i * 4 + j] = all[t]->a[i][j];
}

}  // extern "C"
