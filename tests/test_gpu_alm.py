"""Actuator-line forcing (rhs_lines) on the GPU against the oracle's
restatement, through the C ABI, on the SA channel with synthetic rotors.

FP64 path: relative L2 <= 1e-12 per field for one fine DAF step and for the
element forces and the projected force field; <= 1e-10 over whole
pseudo-iterations.  The GPU differs from the oracle by rounding only (libm
against CUDA's sin, cos, atan2, exp and pow, and the order in which two
turbines' projections add up on a node).  The polars include one so narrow
that many elements find no interval: the reference then keeps the previous
element's values, and both sides must carry them forward alike.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _pair(case, grid, state, spec, oracle_mod):
    from desalm.solver import Solver
    g = Solver(case)
    o = oracle_mod.OracleSolver(case)
    for s in (g, o):
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        if spec is not None:
            s.alm_set(spec)
    return g, o


def _perturb(state, seed):
    """The channel's start plus O(1e-2) noise, so that the interpolated
    velocities differ between cells."""
    rng = np.random.default_rng(seed)
    st = dict(state)
    q = state["q"].reshape(-1, 5).copy()
    q[:, 1:4] += rng.normal(0.0, 1e-2, size=(q.shape[0], 3))
    st["q"] = q.reshape(-1)
    return st


def _check_fields(g, o, fields, tol, what):
    for f in fields:
        a, b = g.get_field(1, f), o.get_field(1, f)
        assert rel_l2(a, b) <= tol, "%s field %d: %.3e" % (what, f, rel_l2(a, b))


def test_alm_daf_step_matches_oracle(oracle_mod):
    case, grid, state, spec = cases.channel_alm(n_tur=2)
    state = _perturb(state, 1)
    g, o = _pair(case, grid, state, spec, oracle_mod)
    for s in (g, o):
        s.begin_step()
        s.solver_daf(1, 0, 1)
    fg, fo = g.alm_get(abi.ALM_FORCES), o.alm_get(abi.ALM_FORCES)
    assert np.abs(fo[:, 3:]).max() > 0
    assert rel_l2(fg, fo) <= 1e-12
    Fg, Fo = g.alm_get(abi.ALM_FIELD), o.alm_get(abi.ALM_FIELD)
    assert np.count_nonzero(Fo[0]) > 100
    assert rel_l2(Fg, Fo) <= 1e-12
    _check_fields(g, o, [abi.F_Q + m for m in range(4)], 1e-12, "solver_daf")


def test_alm_recalculated_residual_has_no_forcing(oracle_mod):
    """The recalculated residual (src/solver_daf.F90:432-463) does not call
    rhs_lines."""
    case, grid, state, spec = cases.channel_alm(n_tur=1)
    state = _perturb(state, 2)
    g, o = _pair(case, grid, state, spec, oracle_mod)
    for s in (g, o):
        s.begin_step()
        s.solver_daf(1, 1, 1)
    _check_fields(g, o, [abi.F_RH + m for m in range(4)], 1e-12, "recalc rh")
    _check_fields(g, o, [abi.F_Q + m for m in range(4)], 1e-12, "solver_daf")


def test_alm_pseudo_iterations_with_angle_updates(oracle_mod):
    case, grid, state, spec = cases.channel_alm(n_tur=2, itmax=3)
    case.use_graph = 0
    state = _perturb(state, 3)
    g, o = _pair(case, grid, state, spec, oracle_mod)
    for step in range(2):
        for s in (g, o):
            for t in (1, 2):
                s.alm_set_angle(t, 0.3 + 0.7 * step + 1.1 * t)
            s.begin_step()
            for _ in range(2):
                s.pseudo_iteration()
    _check_fields(g, o, [abi.F_Q + m for m in range(5)], 1e-10, "pseudo-iterations")


def test_alm_graph_step_equals_eager_and_off_equals_none(oracle_mod):
    """The captured physical step includes the forcing (the graph is built
    again when the forcing changes), and turning the forcing off gives the
    run without it, bit for bit."""
    from desalm.solver import Solver
    case, grid, state, spec = cases.channel_alm(n_tur=1, itmax=4)
    state = _perturb(state, 4)

    def run(graph, setup):
        c = case.copy()
        c.use_graph = graph
        S = Solver(c)
        S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        setup(S)
        S.mg_driver()
        return S.get_state()

    def on_after_first(S):
        S.mg_driver()          # a graph without the forcing exists now
        S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        S.alm_set(spec)

    a = run(1, on_after_first)
    b = run(0, lambda S: S.alm_set(spec))
    for k in ("q", "qn", "nut"):
        assert np.array_equal(a[k], b[k]), k
    c = run(1, lambda S: (S.alm_set(spec), S.alm_set(None)))
    d = run(1, lambda S: None)
    for k in ("q", "qn", "nut"):
        assert np.array_equal(c[k], d[k]), k
    assert not np.array_equal(a["q"], d["q"])
