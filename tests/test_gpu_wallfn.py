"""Wall functions (wf_eta, src/wf_mpi.F90:246-413) on the GPU against the
oracle, through the C ABI, on the SA channel with a coarse wall spacing
(first cell 0.08 of the half height: layer 2 at y+ ~ 50, in the log law).

FP64: relative L2 <= 1e-12 per field for one call of desalm_wall_functions
(both sides solve the same wall law to full precision; they differ in the
rounding of CUDA's log, acos, sin and cos against libm's), <= 1e-10 over
pseudo-iterations with wall_functions = 1.  MIXED: 5e-5, as for the other SA
pseudo-iteration tests.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu

Q5 = [abi.F_Q + m for m in range(5)]


def _pair(case, grid, state, oracle_mod):
    from desalm.solver import Solver
    g = Solver(case)
    o = oracle_mod.OracleSolver(case)
    for s in (g, o):
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return g, o


def _case(seed, **kw):
    case, grid, state = cases.channel(im=33, jm=17, km=17, wall_first=0.08, seed=seed, **kw)
    rng = np.random.default_rng(seed + 100)
    q = state["q"].reshape(-1, 5)
    q[:, 1:4] += rng.normal(0.0, 0.05, size=(q.shape[0], 3))
    state["q"] = q.reshape(-1)
    return case, grid, state


def test_wall_functions_call(oracle_mod):
    case, grid, state = _case(1)
    g, o = _pair(case, grid, state, oracle_mod)
    for s in (g, o):
        s.wall_functions()
    for f in Q5:
        e = rel_l2(g.get_field(1, f), o.get_field(1, f))
        assert e <= 1e-12, (f, e)
    a = g.get_field(1, abi.F_Q + 1).reshape(17, 17, 33)
    b = state["q"].reshape(17, 17, 33, 5)[..., 1]
    assert np.abs(a[1:-1, 1, 1:-1] - b[1:-1, 1, 1:-1]).max() > 1e-3   # layer 2 was set


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_pseudo_iterations_with_wall_functions(precision, oracle_mod):
    case, grid, state = _case(2)
    case.wall_functions = 1
    case.precision_mode = precision
    g, o = _pair(case, grid, state, oracle_mod)
    g.begin_step()
    o.begin_step()
    for it in range(3):
        g.pseudo_iteration()
        o.pseudo_iteration()
    tol = 1e-10 if precision == abi.FP64 else 5e-5
    for f in Q5 + [abi.F_NUT]:
        e = rel_l2(g.get_field(1, f), o.get_field(1, f))
        assert e <= tol, (f, e)


def test_wall_functions_graph_matches_eager():
    from desalm.solver import Solver
    case, grid, state = _case(3, itmax=5)
    case.wall_functions = 1
    case.it_min = 2
    out = []
    for graph in (0, 1):
        c = case.copy()
        c.use_graph = graph
        s = Solver(c)
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        s.mg_driver()
        out.append(s.get_state())
    assert np.array_equal(out[0]["q"], out[1]["q"])
    assert np.array_equal(out[0]["nut"], out[1]["nut"])


def test_wall_functions_need_the_wall_distance():
    from desalm.solver import Solver, DesalmError
    case, grid, state = _case(4)
    case.wall_functions = 1
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"])          # no wall distance
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    with pytest.raises(DesalmError, match="wall distance"):
        S.mg_driver()
    with pytest.raises(DesalmError, match="wall distance"):
        S.wall_functions()
