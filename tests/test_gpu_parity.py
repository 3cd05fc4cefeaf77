"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

FP64 path: relative L2 <= 1e-12 per field for one application of each
entry point on identical inputs, and <= 1e-10 after several whole
pseudo-iterations.  The GPU evaluates the reference's expressions with
round-off-level differences only: two-ended line eliminations (each half in
SGTSV's no-interchange order), reciprocals of J, of the BDF2 and alpha
denominators and of the eliminated diagonals, structured modal transforms,
fused multiply-adds and a different order of the norm's partial sums.
MIXED path (FP64 state and residual, FP32 line-sweep work, modal transforms
and SA ADI): stated tolerances below.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _solver():
    from desalm.solver import Solver
    return Solver


def make_pair(case, grid, state, oracle_mod, real_bytes=8):
    Solver = _solver()
    g = Solver(case)
    o = oracle_mod.OracleSolver(case, real_bytes)
    for s in (g, o):
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return g, o


def perturbed_state(case, seed, nut_scale=0.0):
    """A random state with O(1) velocity and pressure and O(1e-2) history."""
    rng = np.random.default_rng(seed)
    N = case.im * case.jm * case.km
    q = rng.normal(0.0, 1.0, size=(N, 5)) * np.array([0.3, 1.0, 0.5, 0.5, 0.0])
    qn = q + rng.normal(0.0, 1e-2, size=(N, 5))
    qnm1 = qn + rng.normal(0.0, 1e-2, size=(N, 5))
    nut = nut_scale * rng.uniform(0.0, 1.0, size=N) / case.ren
    return dict(q=q.reshape(-1), qn=qn.reshape(-1), qnm1=qnm1.reshape(-1), nut=nut)


def check_fields(g, o, n, fields, tol, what=""):
    for f in fields:
        a, b = g.get_field(n, f), o.get_field(n, f)
        err = rel_l2(a, b)
        assert err <= tol, "%s level %d field %d: rel L2 %.3e > %.1e" % (what, n, f, err, tol)


Q4 = [abi.F_Q + m for m in range(4)]


@pytest.mark.parametrize("shape", [(17, 17, 17), (25, 17, 21)])
def test_metrics_all_levels(shape, oracle_mod):
    case, grid, state = _reshape_cavity(shape, seed=3)
    g, o = make_pair(case, grid, state, oracle_mod)
    for n in range(1, case.ng + 1):
        check_fields(g, o, n, [abi.F_CSI + d for d in range(3)] + [abi.F_ETA + d for d in range(3)] +
                     [abi.F_ZET + d for d in range(3)] + [abi.F_AJ], TOL64, "metrics")


def _reshape_cavity(shape, seed=0):
    """Cavity-type case on a perturbed box of the given (odd) shape."""
    im, jm, km = shape
    rng = np.random.default_rng(seed)
    case, _, _ = cases.cavity(n=17, seed=seed)
    case.im, case.jm, case.km = im, jm, km
    xs, ys, zs = (np.linspace(0, 1, n) for n in (im, jm, km))
    X = np.broadcast_to(xs[None, None, :], (km, jm, im)).copy()
    Y = np.broadcast_to(ys[None, :, None], (km, jm, im)).copy()
    Z = np.broadcast_to(zs[:, None, None], (km, jm, im)).copy()
    bump = np.sin(np.pi * X) * np.sin(np.pi * Y) * np.sin(np.pi * Z)
    for A in (X, Y, Z):
        A += 0.02 / 16 * bump * np.sin(2 * np.pi * (X + 2 * Y) + rng.uniform(0, 6))
    grid = dict(x=X.reshape(-1), y=Y.reshape(-1), z=Z.reshape(-1), wd=None)
    state = perturbed_state(case, seed)
    return case, grid, state


@pytest.mark.parametrize("shape", [(17, 17, 17), (25, 17, 21)])
@pytest.mark.parametrize("recalc", [0, 1])
def test_solver_daf_fine(shape, recalc, oracle_mod):
    case, grid, state = _reshape_cavity(shape, seed=5)
    state = perturbed_state(case, 7, nut_scale=5.0)
    g, o = make_pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.solver_daf(1, recalc, 1)
    check_fields(g, o, 1, [abi.F_Q + m for m in range(4)] + [abi.F_DTAU], TOL64, "solver_daf fine q")
    if recalc:
        check_fields(g, o, 1, [abi.F_RH + m for m in range(4)], TOL64, "solver_daf fine rh")


@pytest.mark.parametrize("itr", [1, 2])
def test_solver_daf_coarse(itr, oracle_mod):
    case, grid, state = _reshape_cavity((25, 17, 21), seed=11)
    g, o = make_pair(case, grid, state, oracle_mod)
    rng = np.random.default_rng(12)
    N2 = int(np.prod(abi.level_dims(case, 2)))
    fields = {}
    for m in range(4):
        fields[abi.F_Q + m] = rng.normal(0, 0.5, N2)
        fields[abi.F_QN + m] = fields[abi.F_Q + m] + rng.normal(0, 1e-2, N2)
        fields[abi.F_QNM1 + m] = fields[abi.F_QN + m] + rng.normal(0, 1e-2, N2)
        fields[abi.F_PK + m] = rng.normal(0, 1e-2, N2)
    fields[abi.F_NUT] = rng.uniform(0, 3e-3, N2)
    im, jm, km = abi.level_dims(case, 2)
    bnd = np.zeros((km, jm, im), bool)
    bnd[0], bnd[-1], bnd[:, 0], bnd[:, -1], bnd[:, :, 0], bnd[:, :, -1] = (True,) * 6
    for m in range(4):
        fields[abi.F_PK + m][bnd.reshape(-1)] = 0.0
    for s in (g, o):
        for f, v in fields.items():
            s.set_field(2, f, v)
        s.solver_daf(2, 1, itr)
    check_fields(g, o, 2, Q4 + [abi.F_PK + m for m in range(4)] + [abi.F_RH + m for m in range(4)], TOL64,
                 "solver_daf coarse")


def test_nlevel_and_prolong(oracle_mod):
    case, grid, state = _reshape_cavity((25, 17, 21), seed=21)
    g, o = make_pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.solver_daf(1, 1, 1)          # produces the fine rh used by the restriction
        s.mg_nlevel(2)
    check_fields(g, o, 2, Q4 + [abi.F_PK + m for m in range(4)] + [abi.F_QOLD + m for m in range(4)] +
                 [abi.F_NUT], TOL64, "mg_nlevel")
    rng = np.random.default_rng(22)
    N2 = int(np.prod(abi.level_dims(case, 2)))
    dq = [rng.normal(0, 1e-2, N2) for _ in range(4)]
    for s in (g, o):
        for m in range(4):
            s.set_field(2, abi.F_Q + m, s.get_field(2, abi.F_QOLD + m) + dq[m])
        s.mg_prolong(1)
    check_fields(g, o, 1, Q4, TOL64, "mg_prolong")


def test_bcond_fm(oracle_mod):
    case, grid, state = _reshape_cavity((17, 17, 17), seed=31)
    case.btype[0] = abi.BC_SYMMETRY
    case.btype[2] = abi.BC_FREESTREAM
    case.btype[4] = abi.BC_PERIODIC
    case.btype[5] = abi.BC_PERIODIC
    case.ifix, case.jfix, case.kfix = 5, 6, 7
    g, o = make_pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.bcond_fm()
    check_fields(g, o, 1, Q4, TOL64, "bcond_fm")


@pytest.mark.parametrize("crs", [(1, 1, 1), (0, 1, 1)])
def test_pseudo_iterations_cavity(crs, oracle_mod):
    case, grid, state = cases.cavity(n=17, seed=41)
    case.icrs, case.jcrs, case.kcrs = crs
    g, o = make_pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(6):
        rg = g.pseudo_iteration()
        ro = o.pseudo_iteration()
        check_fields(g, o, 1, Q4, 1e-10, "pseudo-iteration %d" % it)
        assert np.allclose(rg["residual"][:4], ro["residual"][:4], rtol=0, atol=1e-9)
        assert rg["iterations"] == ro["iterations"]


def test_mixed_precision_step(oracle_mod):
    """MIXED: FP32 line-sweep work and modal transforms (FP64 state and
    residual on every level) against the FP64 oracle.  Stated tolerance:
    relative L2 of q after 4 pseudo-iterations <= 2e-5."""
    case, grid, state = cases.cavity(n=17, seed=51)
    case.precision_mode = abi.MIXED
    g, o = make_pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(4):
        g.pseudo_iteration()
        o.pseudo_iteration()
    for m in range(4):
        err = rel_l2(g.get_field(1, abi.F_Q + m), o.get_field(1, abi.F_Q + m))
        assert err <= 2e-5, (m, err)


def _small_channel(seed=61):
    case, grid, state = cases.channel(im=17, jm=17, km=17, seed=seed)
    return case, grid, state


def test_des_eddy(oracle_mod):
    case, grid, state = _small_channel()
    case.itk = 2
    g, o = make_pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.des_eddy()
    check_fields(g, o, 1, [abi.F_Q + 4, abi.F_NUT], TOL64, "des_eddy")


def test_conservation(oracle_mod):
    case, grid, state = _reshape_cavity((17, 17, 17), seed=71)
    case.btype[0] = abi.BC_INFLOW
    case.btype[1] = abi.BC_FREESTREAM
    rng = np.random.default_rng(72)
    q = state["q"].reshape(-1, 5)
    q[:, 1] = 1.0 + 0.05 * rng.normal(size=q.shape[0])
    state["q"] = q.reshape(-1)
    g, o = make_pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.conservation()
    check_fields(g, o, 1, Q4, TOL64, "conservation")


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_pseudo_iterations_channel_sa(precision, oracle_mod):
    case, grid, state = _small_channel(seed=81)
    case.precision_mode = precision
    g, o = make_pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    tol = 1e-10 if precision == abi.FP64 else 5e-5
    for it in range(4):
        g.pseudo_iteration()
        o.pseudo_iteration()
    check_fields(g, o, 1, Q4 + [abi.F_Q + 4, abi.F_NUT], tol, "SA pseudo-iterations")


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
@pytest.mark.parametrize("which", ["cavity", "channel"])
def test_long_lines_narrow_slabs(which, precision, oracle_mod):
    """257-node i lines do not fit 16 lines per CTA in shared memory: the DAF
    sweeps fall back to 4 (FP64) or 8 (MIXED) lines per CTA, rsmooth to 8 and
    the SA sweeps to 8 (FP64) or 16 (MIXED).  Two pseudo-iterations against
    the oracle at the tolerances of the other pseudo-iteration tests."""
    if which == "cavity":
        case, grid, state = _reshape_cavity((257, 17, 17), seed=95)
    else:
        case, grid, state = cases.channel(im=257, jm=17, km=17, seed=96)
    case.precision_mode = precision
    g, o = make_pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(2):
        g.pseudo_iteration()
        o.pseudo_iteration()
    tol = 1e-10 if precision == abi.FP64 else (2e-5 if which == "cavity" else 5e-5)
    fields = Q4 + ([abi.F_Q + 4, abi.F_NUT] if which == "channel" else [])
    check_fields(g, o, 1, fields, tol, "long lines %s" % which)


@pytest.mark.parametrize("which", ["cavity", "channel"])
def test_graph_step_matches_eager(which, oracle_mod):
    """use_graph = 1 replays the pseudo-time loop as one CUDA graph with a
    device-side while node; it must reproduce the eager driver exactly."""
    from desalm.solver import Solver
    if which == "cavity":
        case, grid, state = cases.cavity(n=17, seed=91, itmax=9)
    else:
        case, grid, state = _small_channel(seed=92)
        case.itmax = 7
    case.it_min = 3
    case.er_min = -0.5       # converges inside the cap on some steps
    out = []
    for graph in (0, 1):
        c = case.copy()
        c.use_graph = graph
        s = Solver(c)
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        reps = [s.mg_driver() for _ in range(3)]
        out.append((reps, s.get_state()))
    (r0, s0), (r1, s1) = out
    for a, b in zip(r0, r1):
        assert a["iterations"] == b["iterations"] and a["converged"] == b["converged"]
        assert np.allclose(a["residual"][:4], b["residual"][:4], rtol=0, atol=1e-12)
    assert np.array_equal(s0["q"], s1["q"])
