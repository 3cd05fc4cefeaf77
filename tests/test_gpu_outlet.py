"""The characteristics outlet (btype 5) on the GPU against the oracle, through
the C ABI, on the open-box wake case (uniform inflow at i = 1, outlet at
i = im, stretched and perturbed grid).

FP64 path: relative L2 <= 1e-12 per field for one fine DAF step (every node,
the outlet plane included) and <= 1e-10 after whole pseudo-iterations, as
for the interior.  The outlet's residual is formed with the stored 1/J and
one reciprocal of the characteristic scale where the reference divides, and
the outlet row of the csi line is eliminated in the two-ended order: both
differ from the oracle by rounding only.  MIXED path: the tolerances of the
other MIXED pseudo-iteration tests (5e-5 with the SA model).
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu

Q4 = [abi.F_Q + m for m in range(4)]


def _pair(case, grid, state, oracle_mod):
    from desalm.solver import Solver
    g = Solver(case)
    o = oracle_mod.OracleSolver(case)
    for s in (g, o):
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return g, o


def _with_history(state, seed):
    """q^n and q^{n-1} a little off q, so that the BDF2 terms do not vanish."""
    rng = np.random.default_rng(seed)
    st = dict(state)
    q = state["q"].reshape(-1, 5)
    qn = q.copy()
    qn[:, :4] += rng.normal(0.0, 1e-3, size=(q.shape[0], 4))
    qnm1 = qn.copy()
    qnm1[:, :4] += rng.normal(0.0, 1e-3, size=(q.shape[0], 4))
    st["qn"], st["qnm1"] = qn.reshape(-1), qnm1.reshape(-1)
    return st


def _check(g, o, fields, tol, what):
    for f in fields:
        e = rel_l2(g.get_field(1, f), o.get_field(1, f))
        assert e <= tol, "%s field %d: %.3e" % (what, f, e)


@pytest.mark.parametrize("turbulence", [0, 1])
@pytest.mark.parametrize("recalc", [0, 1])
def test_outlet_daf_step(turbulence, recalc, oracle_mod):
    case, grid, state = cases.wake(im=25, jm=17, km=21, turbulence=turbulence, seed=3)
    state = _with_history(state, 4)
    g, o = _pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.solver_daf(1, recalc, 1)
    _check(g, o, Q4 + [abi.F_DTAU], 1e-12, "solver_daf")
    a = g.get_field(1, abi.F_Q + 1).reshape(21, 17, 25)
    b = o.get_field(1, abi.F_Q + 1).reshape(21, 17, 25)
    q0 = state["q"].reshape(21, 17, 25, 5)[..., 1]
    assert np.abs(b[1:-1, 1:-1, -1] - q0[1:-1, 1:-1, -1]).max() > 1e-6   # the plane moved
    assert rel_l2(a[:, :, -1], b[:, :, -1]) <= 1e-12
    if recalc:
        _check(g, o, [abi.F_RH + m for m in range(4)], 1e-12, "recalc rh")


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
@pytest.mark.parametrize("turbulence", [0, 1])
def test_outlet_pseudo_iterations(precision, turbulence, oracle_mod):
    case, grid, state = cases.wake(im=33, jm=17, km=17, turbulence=turbulence, seed=5)
    case.precision_mode = precision
    g, o = _pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(4):
        rg = g.pseudo_iteration()
        ro = o.pseudo_iteration()
        if precision == abi.FP64:
            assert np.allclose(rg["residual"][:4], ro["residual"][:4], rtol=0, atol=1e-9)
    tol = 1e-10 if precision == abi.FP64 else 5e-5
    fields = Q4 + ([abi.F_Q + 4, abi.F_NUT] if turbulence else [])
    _check(g, o, fields, tol, "pseudo-iterations")


def test_outlet_side_faces_btype5_sa(oracle_mod):
    """btype 5 on the j faces as well: bcond_fm leaves them, rhs_sa_bcond
    extrapolates nu_tilde with the grid ratio, and their semi-explicit rows
    are off."""
    case, grid, state = cases.wake(im=25, jm=17, km=17, turbulence=1, side=abi.BC_OUTLET, seed=7)
    g, o = _pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(3):
        g.pseudo_iteration()
        o.pseudo_iteration()
    _check(g, o, Q4 + [abi.F_Q + 4, abi.F_NUT], 1e-10, "btype-5 sides")


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_outlet_long_lines(precision, oracle_mod):
    """257-node i lines: the i sweep's narrow slabs with the outlet row."""
    case, grid, state = cases.wake(im=257, jm=17, km=17, turbulence=1, seed=9)
    case.precision_mode = precision
    g, o = _pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(2):
        g.pseudo_iteration()
        o.pseudo_iteration()
    _check(g, o, Q4 + [abi.F_Q + 4], 1e-10 if precision == abi.FP64 else 5e-5, "long lines")


def test_outlet_graph_step_matches_eager():
    from desalm.solver import Solver
    case, grid, state = cases.wake(im=33, jm=17, km=17, turbulence=1, seed=11, itmax=6)
    case.it_min = 2
    out = []
    for graph in (0, 1):
        c = case.copy()
        c.use_graph = graph
        s = Solver(c)
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        reps = [s.mg_driver() for _ in range(2)]
        out.append((reps, s.get_state()))
    (r0, s0), (r1, s1) = out
    for a, b in zip(r0, r1):
        assert a["iterations"] == b["iterations"]
    assert np.array_equal(s0["q"], s1["q"])
    assert np.array_equal(s0["nut"], s1["nut"])


def test_outlet_with_actuator_lines(oracle_mod):
    """The forcing (run beside the SA sub-iterations) and the outlet kernel
    (run beside the residual) share the second stream and its events: with
    both on, the steps match the oracle and the captured step matches the
    eager one bit for bit.  Re 13,773: at Re 1000 this synthetic rotor's
    force scale ls / (rho V^2) is about 850 and the flow blows up, in the
    oracle too."""
    from desalm.solver import Solver
    im, jm, km = 33, 25, 25
    case, grid, state = cases.wake(im=im, jm=jm, km=km, turbulence=1, seed=13, itmax=4, re=13773.0)
    xs = grid["x"].reshape(km, jm, im)[0, 0, :]
    ys = grid["y"].reshape(km, jm, im)[0, :, 0]
    zs = grid["z"].reshape(km, jm, im)[:, 0, 0]
    tur, polars = cases.alm_rotor(xs, ys, zs, (xs[im // 3], 1.0, 1.0), 0.5, seed=5)
    spec = dict(turbines=[tur], polars=polars, vel_infty=0.1, length_scale=1.0)
    g, o = _pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.alm_set(spec)
        s.begin_step()
    for _ in range(3):
        g.pseudo_iteration()
        o.pseudo_iteration()
    _check(g, o, Q4 + [abi.F_Q + 4, abi.F_NUT], 1e-10, "outlet + forcing")
    out = []
    for graph in (0, 1):
        c = case.copy()
        c.use_graph = graph
        S = Solver(c)
        S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        S.alm_set(spec)
        S.mg_driver()
        out.append(S.get_state())
    assert np.array_equal(out[0]["q"], out[1]["q"])
    assert np.array_equal(out[0]["nut"], out[1]["nut"])
