"""ctypes mirror of include/desalm.h (structs, constants, field ids).

The C ABI is the product boundary; this module only describes it for Python
callers (tests, bench, examples).  Field layouts follow the reference's
Fortran arrays: q(1:5, i, j, k) with the component fastest, then i, j, k.
"""
import ctypes as C

DESALM_OK = 0
DESALM_EINVAL = -1
DESALM_ENOMEM = -2
DESALM_ECUDA = -3
DESALM_ENONFINITE = -4
DESALM_ESINGULAR = -5
DESALM_ETIMEOUT = -6
DESALM_ENOTREADY = -7
DESALM_EIO = -8

FP64 = 0
MIXED = 1
PRED_QN = 0
PRED_LINEAR = 1
PRED_LEARNED = 2

LP_FEATURES, LP_TARGET, LP_OUTPUT, LP_SCALES, LP_ALPHA = 0, 1, 2, 3, 4

BC_INTERFACE, BC_WALL, BC_SYMMETRY, BC_FREESTREAM, BC_INFLOW, BC_OUTLET, BC_PERIODIC = 0, 1, 2, 3, 4, 5, 6

F_Q, F_QN, F_QNM1, F_QOLD, F_RH, F_PK = 0, 8, 16, 24, 32, 40
F_CSI, F_ETA, F_ZET, F_AJ, F_NUT, F_DTAU, F_DTEV, F_WD = 48, 52, 56, 60, 61, 62, 63, 64
F_X, F_Y, F_Z = 65, 66, 67


class Case(C.Structure):
    _fields_ = [
        ("im", C.c_int), ("jm", C.c_int), ("km", C.c_int),
        ("ng", C.c_int),
        ("icrs", C.c_int), ("jcrs", C.c_int), ("kcrs", C.c_int),
        ("iter", C.c_int * 4),
        ("itmax", C.c_int),
        ("it_min", C.c_int),
        ("er_min", C.c_double), ("eo_min", C.c_double),
        ("delti", C.c_double),
        ("ren", C.c_double), ("beta", C.c_double),
        ("cfl1", C.c_double), ("vnn1", C.c_double),
        ("cfl2", C.c_double), ("vnn2", C.c_double),
        ("itk", C.c_int),
        ("ep", (C.c_double * 3) * 2),
        ("pdiss_coef", C.c_double),
        ("btype", C.c_int * 6), ("bdir", C.c_int * 6),
        ("ifix", C.c_int), ("jfix", C.c_int), ("kfix", C.c_int),
        ("turbulence", C.c_int),
        ("unsteady", C.c_int),
        ("conservation", C.c_int),
        ("precision_mode", C.c_int),
        ("predictor", C.c_int),
        ("use_graph", C.c_int),
        ("wall_functions", C.c_int),
        ("reserved", C.c_int * 5),
    ]

    def copy(self):
        c = Case()
        C.pointer(c)[0] = self
        return c

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if name == "ep":
                v = [[v[a][b] for b in range(3)] for a in range(2)]
            elif hasattr(v, "__len__"):
                v = list(v)
            d[name] = v
        return d


class StepReport(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("converged", C.c_int),
        ("residual", C.c_double * 5),
        ("init_residual", C.c_double * 5),
        ("pivots", C.c_int),
        ("pivot_lines", C.c_int),
        ("reserved", C.c_int * 6),
    ]

    def as_dict(self):
        return {"iterations": self.iterations, "converged": bool(self.converged),
                "residual": list(self.residual), "init_residual": list(self.init_residual),
                "pivots": self.pivots, "pivot_lines": self.pivot_lines}


class LpReport(C.Structure):
    _fields_ = [
        ("nparam", C.c_long),
        ("samples", C.c_long),
        ("train_steps", C.c_long),
        ("predictions", C.c_long),
        ("fallbacks", C.c_long),
        ("first_loss", C.c_double),
        ("last_loss", C.c_double),
        ("heldout_ratio", C.c_double),
        ("alpha", C.c_double * 5),
    ]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["alpha"] = list(self.alpha)
        return d


class AlmTurbine(C.Structure):
    _fields_ = [
        ("nblades", C.c_int), ("nelems", C.c_int), ("nangles", C.c_int),
        ("tsr", C.c_double), ("tur_rad", C.c_double), ("hub_rad", C.c_double), ("angle", C.c_double),
        ("node_index", C.POINTER(C.c_int)), ("node_pos", C.POINTER(C.c_double)),
        ("disk_dat", C.POINTER(C.c_double)), ("polar_b", C.POINTER(C.c_int)), ("polar_a", C.POINTER(C.c_int)),
        ("nker", C.c_int), ("ker_index", C.POINTER(C.c_int)), ("ker_pos", C.POINTER(C.c_double)),
        ("ker_dat", C.POINTER(C.c_double)),
    ]


class Alm(C.Structure):
    _fields_ = [
        ("n_tur", C.c_int), ("tur", C.POINTER(AlmTurbine)),
        ("vel_infty", C.c_double), ("length_scale", C.c_double),
        ("npolar", C.c_int), ("polar_offset", C.POINTER(C.c_int)), ("polar_count", C.POINTER(C.c_int)),
        ("polar_rows", C.POINTER(C.c_double)),
    ]


ALM_FORCES, ALM_FIELD = 0, 1


class Rfg(C.Structure):
    """desalm_rfg: the random flow generator's tables (synthetic inflow)."""
    _fields_ = [
        ("nmodes", C.c_int),
        ("p", C.POINTER(C.c_double)), ("q", C.POINTER(C.c_double)), ("k", C.POINTER(C.c_double)),
        ("omega", C.POINTER(C.c_double)),
        ("um", C.POINTER(C.c_double)), ("uij", C.POINTER(C.c_double)),
        ("t_ts", C.POINTER(C.c_double)), ("t_ls", C.POINTER(C.c_double)),
    ]


def make_alm(spec):
    """A desalm_alm structure from a dict (see cases.alm_rotor); returns the
    structure and the arrays it points into, which must outlive the call."""
    import numpy as np
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(np.asarray(a, dtype=dt).reshape(-1))
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_int if dt == np.int32 else C.c_double))

    tur = (AlmTurbine * len(spec["turbines"]))()
    for t, T in enumerate(spec["turbines"]):
        u = tur[t]
        u.nblades, u.nelems, u.nangles = T["nblades"], T["nelems"], T["nangles"]
        u.tsr, u.tur_rad, u.hub_rad, u.angle = T["tsr"], T["tur_rad"], T["hub_rad"], T["angle"]
        u.node_index = arr(T["node_index"], np.int32)
        u.node_pos = arr(T["node_pos"], np.float64)
        u.disk_dat = arr(T["disk_dat"], np.float64)
        u.polar_b = arr(T["polar_b"], np.int32)
        u.polar_a = arr(T["polar_a"], np.int32)
        u.nker = len(T["ker_index"])
        u.ker_index = arr(T["ker_index"], np.int32)
        u.ker_pos = arr(T["ker_pos"], np.float64)
        u.ker_dat = arr(T["ker_dat"], np.float64)
    keep.append(tur)
    polars = spec["polars"]
    counts = [len(p) for p in polars]
    offs = list(np.cumsum([0] + counts[:-1]))
    a = Alm()
    a.n_tur = len(spec["turbines"])
    a.tur = C.cast(tur, C.POINTER(AlmTurbine))
    a.vel_infty, a.length_scale = spec["vel_infty"], spec["length_scale"]
    a.npolar = len(polars)
    a.polar_offset = arr(offs, np.int32)
    a.polar_count = arr(counts, np.int32)
    a.polar_rows = arr(np.concatenate([np.asarray(p, np.float64).reshape(-1) for p in polars]), np.float64)
    return a, keep


def level_dims(case, n):
    """Extents of level n (1-based): src/init.F90:257-263."""
    im, jm, km = case.im, case.jm, case.km
    for _ in range(1, n):
        im = (im + case.icrs) // (2 ** case.icrs)
        jm = (jm + case.jcrs) // (2 ** case.jcrs)
        km = (km + case.kcrs) // (2 ** case.kcrs)
    return im, jm, km


class OversetMap(C.Structure):
    _fields_ = [
        ("n", C.c_int),
        ("donee", C.POINTER(C.c_int)),
        ("host", C.POINTER(C.c_int)),
        ("coef", C.POINTER(C.c_double)),
    ]


def make_overset_map(ov):
    """desalm_overset_map of the dict cases.overset_pair returns; the arrays
    stay referenced by the returned keep list."""
    import numpy as _np
    d = _np.ascontiguousarray(ov["donee"], _np.int32)
    h = _np.ascontiguousarray(ov["host"], _np.int32)
    c = _np.ascontiguousarray(ov["coef"], _np.float64)
    m = OversetMap()
    m.n = int(ov["n"])
    m.donee = d.ctypes.data_as(C.POINTER(C.c_int))
    m.host = h.ctypes.data_as(C.POINTER(C.c_int))
    m.coef = c.ctypes.data_as(C.POINTER(C.c_double))
    return m, [d, h, c]
