"""Overset blocks on the GPU (desalm_overset_*) against the oracle's
restatement (oracle/overset_oracle.py): the donor exchange of the momentum and
turbulence fields, and a coupled physical step of two blocks in lockstep
(mg_bintp_mom after each fine DAF step, mg_bintp_tur after each fine SA
update; the convergence norm over both blocks).  FP64: relative L2 <= 1e-12
for one exchange and <= 1e-10 after the coupled pseudo-iterations; MIXED:
<= 5e-5."""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _build(oracle_mod, precision=abi.FP64, itmax=3):
    from desalm.solver import Overset, Solver
    blocks, ov = cases.overset_pair(turbulence=1, itmax=itmax)
    gs, os_ = [], []
    for case, grid, state in blocks:
        case.precision_mode = precision
        case.er_min = -100.0
        case.eo_min = -100.0
        g = Solver(case)
        o = oracle_mod.OracleSolver(case)
        for s in (g, o):
            s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
            s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        gs.append(g)
        os_.append(o)
    return gs, os_, Overset(gs, ov), ov


def test_exchange_matches_oracle(oracle_mod):
    import overset_oracle as oo
    gs, os_, X, ov = _build(oracle_mod)
    X.exchange(0)
    X.exchange(1)
    oo.exchange(os_, ov, [0, 1, 2, 3])
    oo.exchange(os_, ov, [4])
    for g, o in zip(gs, os_):
        for m in range(5):
            assert rel_l2(g.get_field(1, abi.F_Q + m), o.get_field(1, abi.F_Q + m)) <= 1e-12
    X.close()


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_coupled_step_matches_oracle(precision, oracle_mod):
    import overset_oracle as oo
    gs, os_, X, ov = _build(oracle_mod, precision)
    rg = X.mg_driver()
    ro = oo.mg_driver(os_, ov)
    assert rg[0]["iterations"] == ro["iterations"] == 3
    tol = 1e-10 if precision == abi.FP64 else 5e-5
    for g, o in zip(gs, os_):
        for f in [abi.F_Q + m for m in range(5)] + [abi.F_NUT]:
            e = rel_l2(g.get_field(1, f), o.get_field(1, f))
            assert e <= tol, (f, e)
    if precision == abi.FP64:
        assert np.allclose(rg[0]["residual"][:4], ro["residual"][:4], rtol=0, atol=1e-9)
    X.close()


def test_coupled_kw_step_matches_oracle(oracle_mod):
    """Two k-omega blocks: the turbulence exchange carries k and omega
    (mg_bintp_tur's fields), FP64, three coupled pseudo-iterations."""
    import overset_oracle as oo
    from desalm.solver import Overset, Solver
    blocks, ov = cases.overset_pair(turbulence=1, itmax=3)
    gs, os_ = [], []
    for case, grid, state in blocks:
        case, grid, state, om = cases.with_kw(case, grid, state)
        case.er_min = -100.0
        case.eo_min = -100.0
        g = Solver(case)
        o = oracle_mod.OracleSolver(case)
        for s in (g, o):
            s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
            s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
            s.set_omega(om["omega"], om["omega_n"], om["omega_nm1"])
        gs.append(g)
        os_.append(o)
    X = Overset(gs, ov)
    rg = X.mg_driver()
    ro = oo.mg_driver(os_, ov)
    assert rg[0]["iterations"] == ro["iterations"] == 3
    for g, o in zip(gs, os_):
        for f in [abi.F_Q + m for m in range(5)] + [abi.F_NUT]:
            e = rel_l2(g.get_field(1, f), o.get_field(1, f))
            assert e <= 1e-10, (f, e)
        e = rel_l2(g.get_omega()["omega"], o.get_omega()["omega"])
        assert e <= 1e-10, e
    X.close()
