"""Python binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's CPU-baseline leg.  The product never loads it.

OracleSolver exposes the same methods as desalm.solver.Solver so a test can
drive both through identical call sequences.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from desalm.abi import Alm, Case, StepReport, level_dims, make_alm

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        L.desalm_oracle_init.argtypes = [C.POINTER(Case), ip, C.POINTER(vp)]
        L.desalm_oracle_destroy.argtypes = [vp]
        L.desalm_oracle_destroy.restype = None
        for name, args in [
            ("level_dims", [vp, ip, C.POINTER(C.c_int)]),
            ("set_grid", [vp, dp, dp, dp, dp]),
            ("set_state", [vp, dp, dp, dp, dp]),
            ("get_state", [vp, dp, dp, dp, dp]),
            ("get_field", [vp, ip, ip, dp]),
            ("set_field", [vp, ip, ip, dp]),
            ("solver_daf", [vp, ip, ip, ip]),
            ("mg_nlevel", [vp, ip]),
            ("mg_prolong", [vp, ip]),
            ("mg_residual", [vp, ip, dp]),
            ("bcond_fm", [vp]),
            ("des_eddy", [vp]),
            ("conservation", [vp]),
            ("wall_functions", [vp]),
            ("save_qold", [vp]),
            ("begin_step", [vp]),
            ("pseudo_iteration", [vp, C.POINTER(StepReport)]),
            ("mg_driver", [vp, C.POINTER(StepReport)]),
            ("alm_set", [vp, C.POINTER(Alm)]),
            ("alm_set_angle", [vp, ip, C.c_double]),
            ("alm_get", [vp, ip, dp]),
            ("outlet_rhs", [vp, dp]),
            ("kw_eddy", [vp]),
            ("set_omega", [vp, dp, dp, dp]),
            ("get_omega", [vp, dp, dp, dp]),
            ("kw_config", [vp, C.c_double, C.c_double]),
        ]:
            f = getattr(L, "desalm_oracle_" + name)
            f.argtypes = args
            f.restype = C.c_int
        L.desalm_oracle_phase_times.argtypes = [vp, dp]
        L.desalm_oracle_phase_times.restype = None
        L.desalm_oracle_gtsv.argtypes = [ip, ip, dp, dp, dp, dp, ip, C.POINTER(C.c_long)]
        L.desalm_oracle_gtsv.restype = C.c_int
        L.desalm_oracle_modal.argtypes = [dp, dp, dp, C.c_double, dp]
        L.desalm_oracle_modal.restype = None
        L.desalm_oracle_threads.argtypes = []
        L.desalm_oracle_threads.restype = C.c_int
        _LIB = L
    return _LIB


def threads():
    """Host threads the oracle's parallel loops use."""
    return int(lib().desalm_oracle_threads())


def _p(a):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class OracleError(RuntimeError):
    pass


class OracleSolver:
    """The CPU restatement; real_bytes = 8 (FP64 oracle) or 4 (FP32 mirror)."""

    def __init__(self, case, real_bytes=8):
        self.case = case.copy()
        self.L = lib()
        self.ctx = C.c_void_p()
        rc = self.L.desalm_oracle_init(C.byref(self.case), real_bytes, C.byref(self.ctx))
        if rc:
            raise OracleError("desalm_oracle_init failed: %d" % rc)

    def __del__(self):
        if getattr(self, "ctx", None) and self.ctx.value:
            self.L.desalm_oracle_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def _ck(self, rc, what):
        if rc:
            raise OracleError("%s failed: %d" % (what, rc))

    def dims(self, n):
        return level_dims(self.case, n)

    def set_grid(self, x, y, z, wd=None):
        x, y, z, wd = map(_f64, (x, y, z, wd))
        self._ck(self.L.desalm_oracle_set_grid(self.ctx, _p(x), _p(y), _p(z), _p(wd)), "set_grid")

    def set_state(self, q, qn=None, qnm1=None, nut=None):
        q, qn, qnm1, nut = map(_f64, (q, qn, qnm1, nut))
        self._ck(self.L.desalm_oracle_set_state(self.ctx, _p(q), _p(qn), _p(qnm1), _p(nut)), "set_state")

    def get_state(self):
        N = self.case.im * self.case.jm * self.case.km
        q, qn, qnm1, nut = (np.zeros(5 * N), np.zeros(5 * N), np.zeros(5 * N), np.zeros(N))
        self._ck(self.L.desalm_oracle_get_state(self.ctx, _p(q), _p(qn), _p(qnm1), _p(nut)), "get_state")
        return dict(q=q, qn=qn, qnm1=qnm1, nut=nut)

    def get_field(self, n, f):
        im, jm, km = self.dims(n)
        out = np.zeros(im * jm * km)
        self._ck(self.L.desalm_oracle_get_field(self.ctx, n, f, _p(out)), "get_field")
        return out

    def set_field(self, n, f, v):
        v = _f64(v)
        self._ck(self.L.desalm_oracle_set_field(self.ctx, n, f, _p(v)), "set_field")

    def solver_daf(self, n, recalc, itr):
        self._ck(self.L.desalm_oracle_solver_daf(self.ctx, n, recalc, itr), "solver_daf")

    def mg_nlevel(self, n):
        self._ck(self.L.desalm_oracle_mg_nlevel(self.ctx, n), "mg_nlevel")

    def mg_prolong(self, n):
        self._ck(self.L.desalm_oracle_mg_prolong(self.ctx, n), "mg_prolong")

    def mg_residual(self, n):
        r = np.zeros(5)
        self._ck(self.L.desalm_oracle_mg_residual(self.ctx, n, _p(r)), "mg_residual")
        return r

    def bcond_fm(self):
        self._ck(self.L.desalm_oracle_bcond_fm(self.ctx), "bcond_fm")

    def des_eddy(self):
        self._ck(self.L.desalm_oracle_des_eddy(self.ctx), "des_eddy")

    def conservation(self):
        self._ck(self.L.desalm_oracle_conservation(self.ctx), "conservation")

    def kw_eddy(self):
        self._ck(self.L.desalm_oracle_kw_eddy(self.ctx), "kw_eddy")

    def set_omega(self, w, wn=None, wnm1=None):
        w, wn, wnm1 = map(_f64, (w, wn, wnm1))
        self._ck(self.L.desalm_oracle_set_omega(self.ctx, _p(w), _p(wn), _p(wnm1)), "set_omega")

    def get_omega(self):
        N = self.case.im * self.case.jm * self.case.km
        w, wn, wnm1 = np.zeros(N), np.zeros(N), np.zeros(N)
        self._ck(self.L.desalm_oracle_get_omega(self.ctx, _p(w), _p(wn), _p(wnm1)), "get_omega")
        return dict(omega=w, omega_n=wn, omega_nm1=wnm1)

    def kw_config(self, ckin, cein):
        self._ck(self.L.desalm_oracle_kw_config(self.ctx, float(ckin), float(cein)), "kw_config")

    def wall_functions(self):
        self._ck(self.L.desalm_oracle_wall_functions(self.ctx), "wall_functions")

    def save_qold(self):
        self._ck(self.L.desalm_oracle_save_qold(self.ctx), "save_qold")

    def begin_step(self):
        self._ck(self.L.desalm_oracle_begin_step(self.ctx), "begin_step")

    def pseudo_iteration(self):
        rep = StepReport()
        self._ck(self.L.desalm_oracle_pseudo_iteration(self.ctx, C.byref(rep)), "pseudo_iteration")
        return rep.as_dict()

    def mg_driver(self):
        rep = StepReport()
        self._ck(self.L.desalm_oracle_mg_driver(self.ctx, C.byref(rep)), "mg_driver")
        return rep.as_dict()

    def alm_set(self, spec):
        if spec is None:
            self._ck(self.L.desalm_oracle_alm_set(self.ctx, None), "alm_set")
            self._alm_n = 0
            return
        a, keep = make_alm(spec)
        self._ck(self.L.desalm_oracle_alm_set(self.ctx, C.byref(a)), "alm_set")
        self._alm_n = sum(T["nblades"] * T["nelems"] for T in spec["turbines"])

    def alm_set_angle(self, n_t, angle):
        self._ck(self.L.desalm_oracle_alm_set_angle(self.ctx, int(n_t), float(angle)), "alm_set_angle")

    def alm_get(self, what):
        N = self.case.im * self.case.jm * self.case.km
        out = np.zeros(6 * self._alm_n if what == 0 else 3 * N)
        self._ck(self.L.desalm_oracle_alm_get(self.ctx, int(what), _p(out)), "alm_get")
        return out.reshape(-1, 6) if what == 0 else out.reshape(3, N)

    def outlet_rhs(self):
        """The fine level's residual with the characteristics outlet's on the
        plane i = im: rh(1:4) there as a (4, km, jm) array."""
        c = self.case
        out = np.zeros(4 * c.jm * c.km)
        self._ck(self.L.desalm_oracle_outlet_rhs(self.ctx, _p(out)), "outlet_rhs")
        return out.reshape(4, c.km, c.jm)

    def phase_times(self):
        t = np.zeros(8)
        self.L.desalm_oracle_phase_times(self.ctx, _p(t))
        return dict(residual=t[0], daf_solve=t[1], bcond=t[2], transfers=t[3], sa=t[4], norm=t[5])


def gtsv(dl, d, du, b):
    """SGTSV restatement on copies; b is (n,) or (nrhs, n). Returns (x, info, pivots)."""
    dl, d, du = (np.array(a, dtype=np.float64) for a in (dl, d, du))
    b = np.array(b, dtype=np.float64)
    n = d.shape[0]
    nrhs = 1 if b.ndim == 1 else b.shape[0]
    bb = np.ascontiguousarray(b.reshape(nrhs, n))
    piv = C.c_long(0)
    info = lib().desalm_oracle_gtsv(n, nrhs, _p(dl), _p(d), _p(du), _p(bb), n, C.byref(piv))
    return bb.reshape(b.shape), info, piv.value


def modal(csi, eta, zet, sigma):
    """(Mai, N1i, N2i, Mc, Ma, Mb, Mci) of one node as 4x4 arrays."""
    out = np.zeros(7 * 16)
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (csi, eta, zet)]
    lib().desalm_oracle_modal(_p(a[0]), _p(a[1]), _p(a[2]), float(sigma), _p(out))
    return out.reshape(7, 4, 4)
