"""The warp-shuffle cyclic reduction (k_psweep) that solves the DAF line
systems of at most 32 rows (the coarse levels, and every level of a small
grid): chosen by that rule, never by timing, reported as width 2.  It
eliminates in another order than the Thomas kernels, so it is checked
against the FP64 oracle (whose SGTSV is the reference's solver) and against
the lines-in-lanes Thomas kernel to rounding; systems that need SGTSV's
interchanges take its pivoting elimination inside the warp, with the
oracle's interchange count."""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu

Q4 = [abi.F_Q + m for m in range(4)]


def _pair(oracle_mod, precision, widths=None, case_fn=None):
    from desalm.solver import Solver
    c, g, st = case_fn() if case_fn else cases.wake(im=41, jm=17, km=17, turbulence=1, seed=31, itmax=4)
    c.precision_mode = precision
    gpu = Solver(c)
    o = oracle_mod.OracleSolver(c)
    for s in (gpu, o):
        s.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
        s.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
    if widths is not None:
        gpu.set_sweep_widths(widths)
    return c, gpu, o


def test_short_lines_take_the_cyclic_reduction():
    from desalm.solver import Solver
    c, g, st = cases.wake(im=41, jm=17, km=17, turbulence=1, seed=31, itmax=4)
    S = Solver(c)
    S.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
    w = S.sweep_widths()
    # fine i lines: 39 interior rows + the outlet row; everything else <= 32
    assert w[0, 0] in (1, 4, 8, 16)
    assert (w[0, 1:] == 2).all() and (w[1:c.ng] == 2).all()
    S.close()


@pytest.mark.parametrize("precision,tol", [(abi.FP64, 1e-10), (abi.MIXED, 5e-5)])
def test_cyclic_reduction_matches_oracle(precision, tol, oracle_mod):
    c, gpu, o = _pair(oracle_mod, precision)
    for s in (gpu, o):
        s.begin_step()
    for _ in range(3):
        rg, ro = gpu.pseudo_iteration(), o.pseudo_iteration()
        assert rg["pivots"] == 0 and ro["pivots"] == 0
    errs = [rel_l2(gpu.get_field(1, f), o.get_field(1, f)) for f in Q4 + [abi.F_Q + 4]]
    assert max(errs) <= tol, errs
    gpu.close()


def test_cyclic_reduction_agrees_with_thomas(oracle_mod):
    """Forcing the Thomas kernel (width 1) on every level changes the FP64
    fields only by rounding."""
    from desalm.solver import Solver
    out = []
    for forced in (False, True):
        c, g, st = cases.wake(im=41, jm=17, km=17, turbulence=1, seed=32, itmax=4)
        S = Solver(c)
        S.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
        S.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
        if forced:
            w = np.zeros((4, 3), np.int32)
            w[:c.ng] = 1
            S.set_sweep_widths(w)
        S.begin_step()
        for _ in range(2):
            S.pseudo_iteration()
        out.append(S.get_state()["q"])
        S.close()
    a, b = out
    assert not np.array_equal(a, b)          # another elimination order
    assert rel_l2(a, b) <= 1e-13


def test_cyclic_reduction_pivoting_lines(oracle_mod):
    """The cavity whose characteristic rows lose column dominance
    (tests/test_gpu_pivot.py): every line has 15 rows, so the systems that
    need interchanges are solved by the warp's pivoting fallback; the
    interchanges counted equal the oracle's."""
    def cav():
        c, g, st = cases.cavity(n=17, seed=3)
        for d in range(3):
            c.ep[0][d] = 0.2
        c.cfl1 = 3.0
        c.delti = 1.0
        c.unsteady = 0
        return c, g, st
    c, gpu, o = _pair(oracle_mod, abi.FP64, case_fn=cav)
    assert (gpu.sweep_widths()[:c.ng] == 2).all()
    for s in (gpu, o):
        s.begin_step()
    pg = po = pl = 0
    for _ in range(2):
        rg, ro = gpu.pseudo_iteration(), o.pseudo_iteration()
        pg += rg["pivots"]
        po += ro["pivots"]
        pl += rg["pivot_lines"]
    assert po > 100 and pg == po and pl > 0, (pg, po, pl)
    errs = [rel_l2(gpu.get_field(1, f), o.get_field(1, f)) for f in Q4]
    assert max(errs) <= 1e-10, errs
    gpu.close()
