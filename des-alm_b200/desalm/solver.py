"""ctypes binding of libdesalm.so (the CUDA implementation of include/desalm.h).

Solver mirrors the reference's subroutine chain (solver_daf, mg_nlevel,
mg_prolong, mg_residual, bcond_fm, des_eddy, conservation, mg_driver) one
method per C entry point.  There is no CPU fallback: constructing a Solver
fails loudly when the library or a CUDA device is missing.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from .abi import Alm, Case, LpReport, Rfg, StepReport, level_dims, make_alm

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# DESALM_LIBRARY selects another build of the same library (tuning variants)
LIB_PATH = os.environ.get("DESALM_LIBRARY") or os.path.join(PKG_ROOT, "libdesalm.so")
_LIB = None


class DesalmError(RuntimeError):
    pass


def build(force=False):
    """Compile libdesalm.so for sm_100a in place (make -C csrc)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(PKG_ROOT, "csrc")], check=True)
    return LIB_PATH


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise DesalmError("libdesalm.so is not built (run make -C des-alm_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        fp = C.POINTER(C.c_float)
        L.desalm_init.argtypes = [C.POINTER(Case), C.POINTER(vp)]
        L.desalm_init.restype = C.c_int
        L.desalm_destroy.argtypes = [vp]
        L.desalm_destroy.restype = None
        L.desalm_last_error.argtypes = [vp]
        L.desalm_last_error.restype = C.c_char_p
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
            ("kw_eddy", [vp]),
            ("set_state_f32", [vp, fp, fp, fp, fp]),
            ("get_state_f32", [vp, fp, fp, fp, fp]),
            ("set_grid_f32", [vp, fp, fp, fp, fp]),
            ("set_omega", [vp, dp, dp, dp]),
            ("get_omega", [vp, dp, dp, dp]),
            ("kw_config", [vp, C.c_double, C.c_double]),
            ("conservation", [vp]),
            ("wall_functions", [vp]),
            ("save_qold", [vp]),
            ("begin_step", [vp]),
            ("pseudo_iteration", [vp, C.POINTER(StepReport)]),
            ("mg_driver", [vp, C.POINTER(StepReport)]),
            ("sync", [vp]),
            ("profile", [vp, ip]),
            ("kernel_stats", [vp, dp, C.POINTER(C.c_long), dp, C.POINTER(C.c_long)]),
        ]:
            f = getattr(L, "desalm_" + name)
            f.argtypes = args
            f.restype = C.c_int
        fp = C.POINTER(C.c_float)
        for name, args in [
            ("lp_config", [vp, ip, ip, C.c_float, C.c_float]),
            ("lp_report_get", [vp, C.POINTER(LpReport)]),
            ("lp_blend", [vp, C.c_float]),
            ("lp_fields", [vp, ip]),
            ("lp_get_params", [vp, fp]),
            ("lp_set_params", [vp, fp]),
            ("lp_eval", [vp, fp, fp, fp, dp, fp]),
            ("lp_get_buffer", [vp, ip, fp]),
        ]:
            f = getattr(L, "desalm_" + name)
            f.argtypes = args
            f.restype = C.c_int
        cp = C.c_char_p
        for name, args in [
            ("grid_read", [cp, ip, ip, ip, ip, dp, dp, dp, dp]),
            ("grid_write", [cp, ip, ip, ip, ip, dp, dp, dp, dp]),
            ("solu_read", [cp, ip, ip, ip, ip, dp, dp, dp]),
            ("solu_write", [cp, ip, ip, ip, ip, dp, dp, dp]),
            ("filestat_read", [cp, dp, C.POINTER(C.c_int), dp, ip]),
            ("filestat_write", [cp, C.c_double, ip, dp, ip]),
            ("checkpoint_read", [vp, cp]),
            ("checkpoint_write", [vp, cp]),
            ("lp_checkpoint_read", [vp, cp]),
            ("lp_checkpoint_write", [vp, cp]),
            ("alm_set", [vp, C.POINTER(Alm)]),
            ("watchdog_selftest", [vp, C.c_double]),
            ("alm_set_angle", [vp, ip, C.c_double]),
            ("alm_get", [vp, ip, dp]),
            ("rfg_set", [vp, C.POINTER(Rfg)]),
            ("rfg_inlet", [vp, C.c_double]),
            ("rfg_modes", [ip, C.c_longlong, dp, dp, dp, dp]),
        ]:
            f = getattr(L, "desalm_" + name)
            f.argtypes = args
            f.restype = C.c_int
        L.desalm_io_error.argtypes = []
        L.desalm_io_error.restype = C.c_char_p
        L.desalm_stream.argtypes = [vp]
        L.desalm_stream.restype = C.c_void_p
        L.desalm_kernel_class_count.argtypes = []
        L.desalm_kernel_class_count.restype = C.c_int
        L.desalm_sweep_widths.argtypes = [vp, C.POINTER(C.c_int)]
        L.desalm_sweep_widths.restype = C.c_int
        L.desalm_turb_sweep_widths.argtypes = [vp, C.POINTER(C.c_int)]
        L.desalm_turb_sweep_widths.restype = C.c_int
        L.desalm_set_sweep_widths.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.desalm_set_sweep_widths.restype = C.c_int
        L.desalm_mg_driver_batch.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(StepReport)]
        L.desalm_mg_driver_batch.restype = C.c_int
        _LIB = L
    return _LIB


# kernel classes reported by desalm_kernel_stats (order of the C enum)
KERNEL_CLASSES = ["dtau", "resid", "sweep_i", "sweep_j", "sweep_k", "recalc", "bcond", "pfix",
                  "nlevel", "prolong", "rsmooth", "norm", "sa_rhs", "sa_sweep", "sa_bc",
                  "xform_i", "xform_j", "xform_k", "sa_aux", "learn", "alm", "outlet", "wallfn", "misc"]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _f32p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------- file formats
def _io(rc, what):
    if rc:
        raise DesalmError("%s failed (%d): %s" % (what, rc, lib().desalm_io_error().decode()))


def _b(path):
    return os.fsencode(path)


def grid_read(path, im, jm, km, turbulence):
    """The reference's grid file -> dict(x, y, z, wd) of (im*jm*km,) doubles."""
    N = im * jm * km
    x, y, z, wd = (np.zeros(N) for _ in range(4))
    _io(lib().desalm_grid_read(_b(path), im, jm, km, int(turbulence), _p(x), _p(y), _p(z), _p(wd)), "grid_read")
    return dict(x=x, y=y, z=z, wd=wd if turbulence else None)


def grid_write(path, im, jm, km, turbulence, x, y, z, wd=None):
    x, y, z, wd = map(_f64, (x, y, z, wd))
    _io(lib().desalm_grid_write(_b(path), im, jm, km, int(turbulence), _p(x), _p(y), _p(z), _p(wd)), "grid_write")


def solu_read(path, im, jm, km, turbulence):
    """The reference's restart file -> dict(q, qn, nut) in the ABI layouts."""
    N = im * jm * km
    q, qn, nut = np.zeros(5 * N), np.zeros(5 * N), np.zeros(N)
    _io(lib().desalm_solu_read(_b(path), im, jm, km, int(turbulence), _p(q), _p(qn), _p(nut)), "solu_read")
    return dict(q=q, qn=qn, nut=nut)


def solu_write(path, im, jm, km, turbulence, q, qn, nut=None):
    q, qn, nut = map(_f64, (q, qn, nut))
    _io(lib().desalm_solu_write(_b(path), im, jm, km, int(turbulence), _p(q), _p(qn), _p(nut)), "solu_write")


def filestat_read(path, n_tur):
    t, n = C.c_double(0.0), C.c_int(0)
    ang = np.zeros(max(1, n_tur))
    _io(lib().desalm_filestat_read(_b(path), C.byref(t), C.byref(n), _p(ang), n_tur), "filestat_read")
    return t.value, n.value, ang[:n_tur]


def filestat_write(path, time, ntime, angles=()):
    a = _f64(np.asarray(angles, dtype=np.float64).reshape(-1))
    _io(lib().desalm_filestat_write(_b(path), float(time), int(ntime), _p(a) if a.size else None, a.size),
        "filestat_write")


def rfg_modes(nmodes, seed):
    """desalm_rfg_modes (host only): the generator's mode tables p, q, k
    (nmodes, 3) and omega (nmodes,) for a seed."""
    p, q, k = (np.zeros(3 * nmodes) for _ in range(3))
    w = np.zeros(nmodes)
    rc = lib().desalm_rfg_modes(int(nmodes), int(seed), _p(p), _p(q), _p(k), _p(w))
    if rc:
        raise DesalmError("rfg_modes failed (%d)" % rc)
    return dict(p=p.reshape(nmodes, 3), q=q.reshape(nmodes, 3), k=k.reshape(nmodes, 3), omega=w)


def mg_driver_batch(solvers):
    """One physical step of each independent block (desalm_mg_driver_batch):
    the graph-path steps run concurrently.  Returns the step reports."""
    L = lib()
    n = len(solvers)
    ctxs = (C.c_void_p * n)(*[s.ctx for s in solvers])
    reps = (StepReport * n)()
    rc = L.desalm_mg_driver_batch(ctxs, n, reps)
    if rc:
        why = "; ".join(L.desalm_last_error(s.ctx).decode() for s in solvers if L.desalm_last_error(s.ctx))
        raise DesalmError("mg_driver_batch failed (%d): %s" % (rc, why))
    return [r.as_dict() for r in reps]


class OvList:
    """A point list of a rank's share of a sharded overset exchange
    (desalm_ov_list_*): host cells with trilinear weights (gather) or donee
    nodes (scatter) on the given Solvers, values moved through device
    buffers (integer addresses, e.g. torch's data_ptr())."""

    def __init__(self, solvers, pts, coef=None):
        self.L = lib()
        L = self.L
        L.desalm_ov_list_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_int),
                                            C.POINTER(C.c_double), C.POINTER(C.c_void_p)]
        L.desalm_ov_list_create.restype = C.c_int
        L.desalm_ov_list_destroy.argtypes = [C.c_void_p]
        L.desalm_ov_list_destroy.restype = None
        L.desalm_ov_list_last_error.argtypes = [C.c_void_p]
        L.desalm_ov_list_last_error.restype = C.c_char_p
        L.desalm_ov_list_fields.argtypes = [C.c_void_p, C.c_int]
        L.desalm_ov_list_fields.restype = C.c_int
        L.desalm_ov_list_gather.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.desalm_ov_list_gather.restype = C.c_int
        L.desalm_ov_list_scatter.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.desalm_ov_list_scatter.restype = C.c_int
        self.solvers = list(solvers)
        self._pts = np.ascontiguousarray(np.asarray(pts, np.int32).reshape(-1, 4))
        self.n = len(self._pts)
        self._coef = None if coef is None else np.ascontiguousarray(np.asarray(coef, np.float64).reshape(-1, 3))
        arr = (C.c_void_p * len(self.solvers))(*[s.ctx.value for s in self.solvers])
        self.h = C.c_void_p()
        pc = self._coef.ctypes.data_as(C.POINTER(C.c_double)) if self._coef is not None else None
        rc = L.desalm_ov_list_create(arr, len(self.solvers), self.n, self._pts.ctypes.data_as(C.POINTER(C.c_int)), pc,
                                     C.byref(self.h))
        if rc:
            raise DesalmError("desalm_ov_list_create failed (%d)" % rc)

    def _ck(self, rc, what):
        if rc < 0:
            raise DesalmError("%s failed (%d): %s" % (what, rc, self.L.desalm_ov_list_last_error(self.h).decode()))
        return rc

    def fields(self, what):
        return self._ck(self.L.desalm_ov_list_fields(self.h, int(what)), "ov_list_fields")

    def gather(self, what, out_ptr):
        self._ck(self.L.desalm_ov_list_gather(self.h, int(what), C.c_void_p(int(out_ptr))), "ov_list_gather")

    def scatter(self, what, in_ptr):
        self._ck(self.L.desalm_ov_list_scatter(self.h, int(what), C.c_void_p(int(in_ptr))), "ov_list_scatter")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.desalm_ov_list_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        self.close()


class Overset:
    """Overset blocks (desalm_overset_*): Solvers on one GPU coupled by a
    donor map (see cases.overset_pair)."""

    def __init__(self, solvers, ov):
        from .abi import make_overset_map
        self.L = lib()
        self.solvers = list(solvers)
        L = self.L
        L.desalm_overset_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]
        L.desalm_overset_create.restype = C.c_int
        L.desalm_overset_destroy.argtypes = [C.c_void_p]
        L.desalm_overset_destroy.restype = None
        L.desalm_overset_last_error.argtypes = [C.c_void_p]
        L.desalm_overset_last_error.restype = C.c_char_p
        L.desalm_overset_exchange.argtypes = [C.c_void_p, C.c_int]
        L.desalm_overset_exchange.restype = C.c_int
        L.desalm_overset_mg_driver.argtypes = [C.c_void_p, C.POINTER(StepReport)]
        L.desalm_overset_mg_driver.restype = C.c_int
        arr = (C.c_void_p * len(self.solvers))(*[s.ctx.value for s in self.solvers])
        m, self._keep = make_overset_map(ov)
        self.ov = C.c_void_p()
        rc = L.desalm_overset_create(arr, len(self.solvers), C.cast(C.pointer(m), C.c_void_p), C.byref(self.ov))
        if rc:
            raise DesalmError("desalm_overset_create failed (%d)" % rc)

    def _ck(self, rc, what):
        if rc:
            raise DesalmError("%s failed (%d): %s" % (what, rc, self.L.desalm_overset_last_error(self.ov).decode()))

    def exchange(self, what):
        self._ck(self.L.desalm_overset_exchange(self.ov, int(what)), "overset_exchange")

    def mg_driver(self):
        reps = (StepReport * len(self.solvers))()
        self._ck(self.L.desalm_overset_mg_driver(self.ov, reps), "overset_mg_driver")
        return [r.as_dict() for r in reps]

    def close(self):
        if getattr(self, "ov", None) is not None and self.ov.value:
            self.L.desalm_overset_destroy(self.ov)
            self.ov = C.c_void_p()

    def __del__(self):
        self.close()


class Solver:
    """One device context (one block, one GPU) of the pseudo-time iteration."""

    def __init__(self, case):
        self.case = case.copy()
        self.L = lib()
        self.ctx = C.c_void_p()
        rc = self.L.desalm_init(C.byref(self.case), C.byref(self.ctx))
        if rc:
            msg = self.L.desalm_last_error(self.ctx).decode() if self.ctx.value else ""
            if self.ctx.value:
                self.L.desalm_destroy(self.ctx)
                self.ctx = C.c_void_p()
            raise DesalmError("desalm_init failed (%d): %s" % (rc, msg))

    def close(self):
        if getattr(self, "ctx", None) is not None and self.ctx.value:
            self.L.desalm_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        self.close()

    def _ck(self, rc, what):
        if rc:
            raise DesalmError("%s failed (%d): %s" % (what, rc, self.L.desalm_last_error(self.ctx).decode()))

    def dims(self, n):
        return level_dims(self.case, n)

    def set_grid(self, x, y, z, wd=None):
        x, y, z, wd = map(_f64, (x, y, z, wd))
        self._ck(self.L.desalm_set_grid(self.ctx, _p(x), _p(y), _p(z), _p(wd)), "set_grid")

    def set_state(self, q, qn=None, qnm1=None, nut=None):
        q, qn, qnm1, nut = map(_f64, (q, qn, qnm1, nut))
        self._ck(self.L.desalm_set_state(self.ctx, _p(q), _p(qn), _p(qnm1), _p(nut)), "set_state")

    def get_state(self):
        N = self.case.im * self.case.jm * self.case.km
        q, qn, qnm1, nut = (np.zeros(5 * N), np.zeros(5 * N), np.zeros(5 * N), np.zeros(N))
        self._ck(self.L.desalm_get_state(self.ctx, _p(q), _p(qn), _p(qnm1), _p(nut)), "get_state")
        return dict(q=q, qn=qn, qnm1=qnm1, nut=nut)

    def set_state_f32(self, q, qn=None, qnm1=None, nut=None):
        q, qn, qnm1, nut = map(_f32, (q, qn, qnm1, nut))
        self._ck(self.L.desalm_set_state_f32(self.ctx, _f32p(q), _f32p(qn), _f32p(qnm1), _f32p(nut)), "set_state_f32")

    def get_state_f32(self):
        N = self.case.im * self.case.jm * self.case.km
        q, qn, qnm1, nut = (np.zeros(5 * N, np.float32), np.zeros(5 * N, np.float32), np.zeros(5 * N, np.float32),
                            np.zeros(N, np.float32))
        self._ck(self.L.desalm_get_state_f32(self.ctx, _f32p(q), _f32p(qn), _f32p(qnm1), _f32p(nut)), "get_state_f32")
        return dict(q=q, qn=qn, qnm1=qnm1, nut=nut)

    def set_grid_f32(self, x, y, z, wd=None):
        x, y, z, wd = map(_f32, (x, y, z, wd))
        self._ck(self.L.desalm_set_grid_f32(self.ctx, _f32p(x), _f32p(y), _f32p(z), _f32p(wd)), "set_grid_f32")

    def get_field(self, n, f):
        im, jm, km = self.dims(n)
        out = np.zeros(im * jm * km)
        self._ck(self.L.desalm_get_field(self.ctx, n, f, _p(out)), "get_field")
        return out

    def set_field(self, n, f, v):
        v = _f64(v)
        self._ck(self.L.desalm_set_field(self.ctx, n, f, _p(v)), "set_field")

    def solver_daf(self, n, recalc, itr):
        self._ck(self.L.desalm_solver_daf(self.ctx, n, recalc, itr), "solver_daf")

    def mg_nlevel(self, n):
        self._ck(self.L.desalm_mg_nlevel(self.ctx, n), "mg_nlevel")

    def mg_prolong(self, n):
        self._ck(self.L.desalm_mg_prolong(self.ctx, n), "mg_prolong")

    def mg_residual(self, n):
        r = np.zeros(5)
        self._ck(self.L.desalm_mg_residual(self.ctx, n, _p(r)), "mg_residual")
        return r

    def bcond_fm(self):
        self._ck(self.L.desalm_bcond_fm(self.ctx), "bcond_fm")

    def des_eddy(self):
        self._ck(self.L.desalm_des_eddy(self.ctx), "des_eddy")

    def kw_eddy(self):
        self._ck(self.L.desalm_kw_eddy(self.ctx), "kw_eddy")

    def set_omega(self, w, wn=None, wnm1=None):
        w, wn, wnm1 = map(_f64, (w, wn, wnm1))
        self._ck(self.L.desalm_set_omega(self.ctx, _p(w), _p(wn), _p(wnm1)), "set_omega")

    def get_omega(self):
        N = self.case.im * self.case.jm * self.case.km
        w, wn, wnm1 = np.zeros(N), np.zeros(N), np.zeros(N)
        self._ck(self.L.desalm_get_omega(self.ctx, _p(w), _p(wn), _p(wnm1)), "get_omega")
        return dict(omega=w, omega_n=wn, omega_nm1=wnm1)

    def kw_config(self, ckin, cein):
        self._ck(self.L.desalm_kw_config(self.ctx, float(ckin), float(cein)), "kw_config")

    def conservation(self):
        self._ck(self.L.desalm_conservation(self.ctx), "conservation")

    def kernel_tiles(self):
        """CTA tiles of the residual kernels, [level][kernel][axis] (kernel 0
        K_R, 1 the recalculated residual, 2 the turbulence residual)."""
        out = (C.c_int * 36)()
        self._ck(self.L.desalm_kernel_tiles(self.ctx, out), "kernel_tiles")
        return np.array(list(out)).reshape(4, 3, 3)

    def sweep_widths(self):
        """Kernel of the DAF sweeps, [level][direction]: 1 lines in lanes,
        16/8/4 slab lines per CTA (0: not tuned, lines in lanes)."""
        out = (C.c_int * 12)()
        self._ck(self.L.desalm_sweep_widths(self.ctx, out), "sweep_widths")
        return np.array(list(out)).reshape(4, 3)

    def turb_sweep_widths(self):
        """Kernel of the turbulence sweeps per direction: 1 lines in lanes,
        32/16/8 slab lines per CTA (0: not tuned, lines in lanes)."""
        out = (C.c_int * 3)()
        self._ck(self.L.desalm_turb_sweep_widths(self.ctx, out), "turb_sweep_widths")
        return np.array(list(out))

    def set_sweep_widths(self, nl=None, turb=None):
        """Sets the sweep kernels (nl: [4][3] or 12 values; turb: 3 values)."""
        a = None if nl is None else (C.c_int * 12)(*[int(v) for v in np.asarray(nl).reshape(-1)])
        b = None if turb is None else (C.c_int * 3)(*[int(v) for v in np.asarray(turb).reshape(-1)])
        self._ck(self.L.desalm_set_sweep_widths(self.ctx, a, b), "set_sweep_widths")

    def wall_functions(self):
        self._ck(self.L.desalm_wall_functions(self.ctx), "wall_functions")

    def save_qold(self):
        self._ck(self.L.desalm_save_qold(self.ctx), "save_qold")

    def begin_step(self):
        self._ck(self.L.desalm_begin_step(self.ctx), "begin_step")

    def pseudo_iteration(self):
        rep = StepReport()
        self._ck(self.L.desalm_pseudo_iteration(self.ctx, C.byref(rep)), "pseudo_iteration")
        return rep.as_dict()

    def mg_driver(self):
        rep = StepReport()
        self._ck(self.L.desalm_mg_driver(self.ctx, C.byref(rep)), "mg_driver")
        return rep.as_dict()

    def sync(self):
        self._ck(self.L.desalm_sync(self.ctx), "sync")

    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        return self.L.desalm_stream(self.ctx)

    def profile(self, enable=True):
        self._ck(self.L.desalm_profile(self.ctx, 1 if enable else 0), "profile")

    def kernel_stats(self):
        """{class: {level: (ms, launches, nodes)}} since the last profile() call,
        and the total number of kernel launches."""
        n = self.L.desalm_kernel_class_count() * 4
        ms = np.zeros(n)
        la = (C.c_long * n)()
        nodes = np.zeros(n)
        tot = C.c_long(0)
        self._ck(self.L.desalm_kernel_stats(self.ctx, _p(ms), la, _p(nodes), C.byref(tot)), "kernel_stats")
        out = {}
        for c, name in enumerate(KERNEL_CLASSES):
            for lvl in range(4):
                t = c * 4 + lvl
                if la[t]:
                    out.setdefault(name, {})[lvl + 1] = (float(ms[t]), int(la[t]), float(nodes[t]))
        return out, int(tot.value)

    def watchdog_selftest(self, seconds):
        """The status of desalm_watchdog_selftest (DESALM_ETIMEOUT when the
        device's bounded wait gave up as it must)."""
        return int(self.L.desalm_watchdog_selftest(self.ctx, float(seconds)))

    def last_error(self):
        return self.L.desalm_last_error(self.ctx).decode()

    # ------------------------------------------------ actuator-line forcing
    def alm_set(self, spec):
        """Turn the actuator-line forcing on (spec: see cases.alm_rotor) or off (None)."""
        if spec is None:
            self._ck(self.L.desalm_alm_set(self.ctx, None), "alm_set")
            self._alm_n = 0
            return
        a, keep = make_alm(spec)
        self._ck(self.L.desalm_alm_set(self.ctx, C.byref(a)), "alm_set")
        self._alm_n = sum(T["nblades"] * T["nelems"] for T in spec["turbines"])

    def alm_set_angle(self, n_t, angle):
        self._ck(self.L.desalm_alm_set_angle(self.ctx, int(n_t), float(angle)), "alm_set_angle")

    def alm_get(self, what):
        N = self.case.im * self.case.jm * self.case.km
        out = np.zeros(6 * self._alm_n if what == 0 else 3 * N)
        self._ck(self.L.desalm_alm_get(self.ctx, int(what), _p(out)), "alm_get")
        return out.reshape(-1, 6) if what == 0 else out.reshape(3, N)

    def rfg_set(self, spec):
        """Turn the synthetic inflow turbulence on (spec: dict with p, q, k
        of shape (N, 3), omega (N,), um (km, jm, 3), uij (km, jm, 6), t_ts and
        t_ls (km, jm); see cases.rfg_inflow) or off (None)."""
        if spec is None:
            self._ck(self.L.desalm_rfg_set(self.ctx, None), "rfg_set")
            return
        keep = {n: _f64(np.asarray(spec[n], dtype=np.float64).reshape(-1))
                for n in ("p", "q", "k", "omega", "um", "uij", "t_ts", "t_ls")}
        r = Rfg(len(keep["omega"]), *(_p(keep[n]) for n in ("p", "q", "k", "omega", "um", "uij", "t_ts", "t_ls")))
        self._ck(self.L.desalm_rfg_set(self.ctx, C.byref(r)), "rfg_set")

    def rfg_inlet(self, time):
        self._ck(self.L.desalm_rfg_inlet(self.ctx, float(time)), "rfg_inlet")

    # ------------------------------------------------ checkpoint / restart
    def checkpoint_write(self, path):
        self._ck(self.L.desalm_checkpoint_write(self.ctx, _b(path)), "checkpoint_write")

    def checkpoint_read(self, path):
        self._ck(self.L.desalm_checkpoint_read(self.ctx, _b(path)), "checkpoint_read")

    def lp_checkpoint_write(self, path):
        self._ck(self.L.desalm_lp_checkpoint_write(self.ctx, _b(path)), "lp_checkpoint_write")

    def lp_checkpoint_read(self, path):
        self._ck(self.L.desalm_lp_checkpoint_read(self.ctx, _b(path)), "lp_checkpoint_read")

    # ------------------------------------------------ learned initial guess
    def lp_config(self, train_steps=-1, warm=-1, lr=-1.0, ymax=-1.0):
        self._ck(self.L.desalm_lp_config(self.ctx, int(train_steps), int(warm), float(lr), float(ymax)), "lp_config")

    def lp_blend(self, alpha=-1.0):
        """alpha < 0: automatic blend of each field's correction; else fixed."""
        self._ck(self.L.desalm_lp_blend(self.ctx, float(alpha)), "lp_blend")

    def lp_fields(self, mask=0x1f):
        """Bit f of mask: field f (p, u, v, w, nu_tilde) takes the correction."""
        self._ck(self.L.desalm_lp_fields(self.ctx, int(mask)), "lp_fields")

    def lp_report(self):
        r = LpReport()
        self._ck(self.L.desalm_lp_report_get(self.ctx, C.byref(r)), "lp_report_get")
        return r.as_dict()

    def lp_params(self):
        theta = np.zeros(self.lp_report()["nparam"], dtype=np.float32)
        self._ck(self.L.desalm_lp_get_params(self.ctx, _f32p(theta)), "lp_get_params")
        return theta

    def lp_set_params(self, theta):
        theta = _f32(theta)
        if theta.size != self.lp_report()["nparam"]:
            raise ValueError("expected %d parameters" % self.lp_report()["nparam"])
        self._ck(self.L.desalm_lp_set_params(self.ctx, _f32p(theta)), "lp_set_params")

    def lp_eval(self, x, t=None):
        """Forward pass on features x [16, N]; with a target t [5, N] also the
        loss and the parameter gradient.  Returns (y [5, N], loss, grad)."""
        N = self.case.im * self.case.jm * self.case.km
        x = _f32(x).reshape(16, N)
        t = None if t is None else _f32(t).reshape(5, N)
        y = np.zeros((5, N), dtype=np.float32)
        loss = C.c_double(0.0)
        grad = None if t is None else np.zeros(self.lp_report()["nparam"], dtype=np.float32)
        self._ck(self.L.desalm_lp_eval(self.ctx, _f32p(x), _f32p(t), _f32p(y), C.byref(loss), _f32p(grad)), "lp_eval")
        return y, (loss.value if t is not None else None), grad

    def lp_buffer(self, which):
        N = self.case.im * self.case.jm * self.case.km
        size = {0: 16 * N, 1: 5 * N, 2: 5 * N, 3: 16, 4: 5}[which]
        out = np.zeros(size, dtype=np.float32)
        self._ck(self.L.desalm_lp_get_buffer(self.ctx, which, _f32p(out)), "lp_get_buffer")
        return out if which >= 3 else out.reshape(-1, N)
