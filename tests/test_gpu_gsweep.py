"""The two kernels of the line sweeps: the lines-in-lanes kernel (k_gsweep,
k_sa_gsweep: a warp solves 32 lines, the eliminated rows kept in a global
scratch) and the shared-memory slab kernel (k_sweep4, k_sa_sweep4) do the same
operations in the same order, so a physical step must give the same bits
whichever is chosen, for the DAF sweeps of every level and the turbulence
sweeps (SA and k-omega), with the characteristics outlet row, in FP64 and
MIXED mode, and on line systems that need SGTSV's pivoting."""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _make(which):
    if which == "wake_sa":
        return cases.wake(im=41, jm=17, km=17, turbulence=1, seed=21, itmax=4) + (None,)
    if which == "channel_kw":
        c, g, s = cases.channel(im=33, jm=33, km=17, seed=22)
        return cases.with_kw(c, g, s)
    if which == "pivot_cavity":
        c, g, s = cases.cavity(n=17, seed=3)
        for d in range(3):
            c.ep[0][d] = 0.2
        c.cfl1 = 3.0
        c.delti = 1.0
        c.unsteady = 0
        return c, g, s, None
    raise ValueError(which)


def _solver(which, precision, nl, turb):
    from desalm.solver import Solver
    c, g, st, om = _make(which)
    c.precision_mode = precision
    c.use_graph = 0
    S = Solver(c)
    S.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
    S.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
    if om is not None:
        S.set_omega(om["omega"], om["omega_n"], om["omega_nm1"])
    w = np.zeros((4, 3), np.int32)
    w[:c.ng] = nl
    S.set_sweep_widths(w, [turb] * 3)
    return S, c


@pytest.mark.parametrize("which", ["wake_sa", "channel_kw", "pivot_cavity"])
@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_lanes_and_slab_give_the_same_bits(which, precision):
    lanes, c = _solver(which, precision, 1, 1)
    slab, _ = _solver(which, precision, 4, 8)
    assert (lanes.sweep_widths()[:c.ng] == 1).all() and (lanes.turb_sweep_widths() == 1).all()
    assert (slab.sweep_widths()[:c.ng] == 4).all() and (slab.turb_sweep_widths() == 8).all()
    for s in (lanes, slab):
        s.begin_step()
    piv = [0, 0]
    plines = [0, 0]
    for _ in range(3):
        for t, s in enumerate((lanes, slab)):
            r = s.pseudo_iteration()
            piv[t] += r["pivots"]
            plines[t] += r["pivot_lines"]
    a, b = lanes.get_state(), slab.get_state()
    for k in ("q", "nut"):
        assert np.array_equal(a[k], b[k]), (k, rel_l2(a[k], b[k]))
    if c.turbulence == 2:
        assert np.array_equal(lanes.get_omega()["omega"], slab.get_omega()["omega"])
    assert piv[0] == piv[1] and plines[0] == plines[1], (piv, plines)
    if which == "pivot_cavity":
        assert piv[0] > 0 and plines[0] > 0
    lanes.close()
    slab.close()


def test_graph_step_with_lanes_equals_eager():
    """The captured physical step with the lines-in-lanes kernels equals the
    eager one bit for bit."""
    from desalm.solver import Solver
    out = []
    for graph in (0, 1):
        c, g, st = cases.wake(im=41, jm=17, km=17, turbulence=1, seed=23, itmax=5)
        c.use_graph = graph
        S = Solver(c)
        S.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
        S.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
        S.set_sweep_widths(np.array([[1, 1, 1]] * c.ng + [[0, 0, 0]] * (4 - c.ng)), [1, 1, 1])
        r = S.mg_driver()
        out.append((r["iterations"], S.get_state()["q"]))
        S.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])


def test_set_sweep_widths_checks_its_arguments():
    from desalm.solver import Solver, DesalmError
    c, g, st = cases.cavity(n=17, seed=3)
    S = Solver(c)
    S.set_grid(g["x"], g["y"], g["z"])
    before = (S.sweep_widths().copy(), S.turb_sweep_widths().copy())
    bad = np.zeros((4, 3), np.int32)
    bad[0, 0] = 5                       # not a width
    with pytest.raises(DesalmError):
        S.set_sweep_widths(bad)
    bad = np.zeros((4, 3), np.int32)
    bad[c.ng, 0] = 1                    # a level the case does not have
    with pytest.raises(DesalmError):
        S.set_sweep_widths(bad)
    with pytest.raises(DesalmError):
        S.set_sweep_widths(None, [1, 2, 1])
    assert np.array_equal(S.sweep_widths(), before[0])
    assert np.array_equal(S.turb_sweep_widths(), before[1])
    S.close()
