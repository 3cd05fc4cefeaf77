"""Synthetic inflow turbulence (desalm_rfg_set / desalm_rfg_inlet) on the GPU
against the oracle (oracle/rfg_oracle.py), through the C ABI, on the open-box
wake case.

The inflow plane's velocities agree with the oracle to a relative L2 of
1e-12: both sum the same modes in the same order, and differ by the rounding
of sin/cos and of the wavenumber scale (the GPU multiplies k by the node's
stored upsilon / c where the reference divides k upsilon by c).  Every other
entry of the state is untouched, bit for bit.  A physical step then holds the
forced plane (inflow face, btype 4) under the q^n guess and under linear
extrapolation, which forces the plane again after the guess.
"""
import numpy as np
import pytest

import rfg_oracle
from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _spec(case, kind, nmodes, seed):
    spec = cases.rfg_inflow(case, u=1.0, intensity=0.05, length_scale=0.3, nmodes=nmodes, seed=seed)
    if kind == "aniso":
        rng = np.random.default_rng(seed)
        km, jm = case.km, case.jm
        uij = np.zeros((km, jm, 6))
        for k in range(km):
            for j in range(jm):
                Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
                lam = np.array([1.0, 2.2, 3.7]) * 0.05 ** 2 * rng.uniform(0.8, 1.2)
                R = Q @ np.diag(lam) @ Q.T
                uij[k, j] = (R[0, 0], R[0, 1], R[0, 2], R[1, 1], R[1, 2], R[2, 2])
        spec["uij"] = uij
        spec["t_ts"] = rng.uniform(0.1, 0.5, size=(km, jm))
        spec["t_ls"] = rng.uniform(0.1, 0.4, size=(km, jm))
        spec["um"][..., 1] = rng.uniform(-0.1, 0.1, size=(km, jm))
    return spec


def _solver(case, grid, state, spec):
    from desalm.solver import Solver
    g = Solver(case)
    g.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    g.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    g.rfg_set(spec)
    return g


def _q(a, case):
    return np.asarray(a).reshape(case.km, case.jm, case.im, 5)


@pytest.mark.parametrize("kind", ["isotropic", "aniso"])
def test_rfg_inlet_matches_oracle(kind):
    case, grid, state = cases.wake(im=17, jm=21, km=19, turbulence=0, ng=2, seed=2)
    spec = _spec(case, kind, 300, 7)   # 300 modes: two full shared-memory chunks and a ragged one
    g = _solver(case, grid, state, spec)
    dims = (case.im, case.jm, case.km)
    q0 = _q(state["q"], case)
    for t in (0.0, 0.37, 12.5):
        g.rfg_inlet(t)
        st = g.get_state()
        qg = _q(st["q"], case)
        qo = rfg_oracle.inlet_forcing(q0.copy(), grid, dims, t, spec)
        plane = (slice(1, -1), slice(1, -1), 0, slice(1, 4))
        e = rel_l2(qg[plane] - spec["um"][1:-1, 1:-1], qo[plane] - spec["um"][1:-1, 1:-1])
        assert e <= 1e-12, "t = %g: fluctuation relative L2 %.3e" % (t, e)
        rest = np.ones(qg.shape, bool)
        rest[plane] = False
        assert np.array_equal(qg[rest], q0[rest])
        assert np.array_equal(st["qn"], state["qn"]) and np.array_equal(st["qnm1"], state["qnm1"])
    g.close()


@pytest.mark.parametrize("predictor", [abi.PRED_QN, abi.PRED_LINEAR])
def test_physical_step_holds_the_forced_plane(predictor):
    case, grid, state = cases.wake(im=17, jm=21, km=19, turbulence=0, ng=2, seed=3, itmax=3)
    case.predictor = predictor
    spec = _spec(case, "aniso", 200, 9)
    g = _solver(case, grid, state, spec)
    plane = (slice(1, -1), slice(1, -1), 0, slice(1, 4))
    t = 0.05
    g.rfg_inlet(t)
    forced = _q(g.get_state()["q"], case)[plane].copy()
    qo = rfg_oracle.inlet_forcing(_q(state["q"], case).copy(), grid, (case.im, case.jm, case.km), t, spec)
    assert rel_l2(forced - spec["um"][1:-1, 1:-1], qo[plane] - spec["um"][1:-1, 1:-1]) <= 1e-12
    g.mg_driver()
    st = g.get_state()
    assert np.array_equal(_q(st["q"], case)[plane], forced)
    assert np.array_equal(_q(st["qn"], case)[plane], forced)   # q shifted into q^n after the forcing
    assert np.all(np.isfinite(st["q"]))
    g.close()


def test_rfg_rejects_bad_tables_and_stale_grids():
    from desalm.solver import DesalmError, Solver
    case, grid, state = cases.wake(im=17, jm=21, km=19, turbulence=0, ng=2, seed=4)
    spec = _spec(case, "isotropic", 16, 1)
    g = Solver(case)
    with pytest.raises(DesalmError) as e:
        g.rfg_set(spec)                       # before the grid: the nodes' coordinates are unknown
    assert "grid" in str(e.value)
    g.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    g.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    spec["uij"][5, 7] = (1e-4, 2e-4, 0.0, 1e-4, 0.0, 1e-4)   # eigenvalues -1e-4, 1e-4, 3e-4
    with pytest.raises(DesalmError) as e:
        g.rfg_set(spec)
    assert "positive definite" in str(e.value)
    with pytest.raises(DesalmError) as e:
        g.rfg_inlet(0.0)                      # the failed set left the generator off
    assert "no generator tables" in str(e.value)
    spec["uij"][5, 7] = spec["uij"][5, 8]
    g.rfg_set(spec)
    g.rfg_inlet(0.0)
    g.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))   # a new grid: the node tables are stale
    with pytest.raises(DesalmError) as e:
        g.rfg_inlet(0.0)
    assert "no generator tables" in str(e.value)
    g.close()
