"""Failure detection, with the failure made on the host (no GPU fault, trap
or hang): corrupted input, a singular grid, and the device watchdog forced
to give up.  Every case must end in an error status from the C ABI, after
which the context still works.
"""
import ctypes as C
import time

import numpy as np
import pytest

from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _solver(case, grid, state):
    from desalm.solver import Solver
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return S


def _status(S, what, *args):
    f = getattr(S.L, "desalm_" + what)
    rep = abi.StepReport()
    return int(f(S.ctx, C.byref(rep), *args))


@pytest.mark.parametrize("graph", [0, 1])
def test_nan_in_the_state_is_reported(graph):
    case, grid, state = cases.cavity(n=17, seed=3, itmax=10)
    case.use_graph = graph
    q = state["q"].copy()
    q[5 * (8 + 17 * 8 + 289 * 8) + 2] = np.nan  # v at the interior node (9, 9, 9)
    S = _solver(case, grid, dict(state, q=q))
    assert _status(S, "mg_driver") == abi.DESALM_ENONFINITE
    assert "non-finite" in S.last_error()
    # the context stays usable: a clean state steps normally afterwards
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    S.mg_driver()
    assert np.isfinite(S.get_state()["q"]).all()


def test_singular_grid_is_reported():
    """Two grid planes collapsed onto a third: the central difference
    x(i+1) - x(i-1) vanishes at i = 10, the Jacobian there is infinite, and
    the non-finite residual (or a zero pivot) is reported as a status."""
    case, grid, state = cases.cavity(n=17, seed=4, itmax=5)
    n = case.im
    x = grid["x"].reshape(n, n, n).copy()
    x[:, :, 9] = x[:, :, 8]                    # i = 10 and 11 onto i = 9
    x[:, :, 10] = x[:, :, 8]
    S = _solver(case, dict(grid, x=x.reshape(-1)), state)
    rc = _status(S, "mg_driver")
    assert rc in (abi.DESALM_ENONFINITE, abi.DESALM_ESINGULAR), rc


def test_watchdog_gives_up_and_reports():
    case, grid, state = cases.cavity(n=17, seed=5, itmax=3)
    S = _solver(case, grid, state)
    t0 = time.perf_counter()
    assert S.watchdog_selftest(0.05) == abi.DESALM_ETIMEOUT
    assert time.perf_counter() - t0 < 5.0
    assert "gave up" in S.last_error()
    S.mg_driver()                              # the context still works
    assert np.isfinite(S.get_state()["q"]).all()
