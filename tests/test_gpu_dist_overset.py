"""The sharded overset path on the GPU with one rank (desalm.overset_dist with
GpuExchange over desalm_ov_list): the device lists gather the donor values
into a packed buffer and write the received ones, and the lockstep driver
over the blocks' fine-grained entry points steps like the library's own
multi-block driver (desalm_overset_mg_driver) and like the oracle's.  The
cross-rank transfers and the partition are covered with gloo ranks on the CPU
(tests/test_dist_overset.py)."""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _solvers(specs, precision=abi.FP64):
    from desalm.solver import Solver
    out = []
    for case, grid, state in specs:
        case.precision_mode = precision
        s = Solver(case)
        s.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        s.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        out.append(s)
    return out


def _specs(nblocks=3, itmax=3):
    specs, ov = cases.overset_chain(nblocks, seed=7, turbulence=1, itmax=itmax)
    for c, _, _ in specs:
        c.er_min = -100.0
        c.eo_min = -100.0
    return specs, ov


def test_list_exchange_equals_library_exchange():
    """One exchange through the packed device lists writes the same bits as
    desalm_overset_exchange."""
    from desalm.overset_dist import GpuExchange, Partition
    from desalm.solver import Overset
    specs, ov = _specs()
    a = _solvers(specs)
    b = _solvers(specs)
    part = Partition(ov, [0] * len(specs), 0, 1)
    ex = GpuExchange(part, a)
    X = Overset(b, ov)
    for what in (0, 1):
        ex(what)
        X.exchange(what)
    for sa, sb in zip(a, b):
        for m in range(5):
            assert np.array_equal(sa.get_field(1, abi.F_Q + m), sb.get_field(1, abi.F_Q + m)), m
    ex.close()
    X.close()


def test_sharded_driver_one_rank_matches_library_and_oracle(oracle_mod):
    import overset_oracle as oo
    from desalm.overset_dist import GpuExchange, Partition, mg_driver
    from desalm.solver import Overset
    specs, ov = _specs()
    nb = len(specs)
    a = _solvers(specs)
    part = Partition(ov, [0] * nb, 0, 1)
    ex = GpuExchange(part, a)
    c0 = specs[0][0]
    rep = mg_driver(a, part, ex, None, nb, (c0.im - 2) * (c0.jm - 2) * (c0.km - 2))
    b = _solvers(specs)
    X = Overset(b, ov)
    rb = X.mg_driver()
    os_ = []
    for case, grid, state in specs:
        o = oracle_mod.OracleSolver(case)
        o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        os_.append(o)
    ro = oo.mg_driver(os_, ov)
    assert rep["iterations"] == rb[0]["iterations"] == ro["iterations"] == 3
    assert np.allclose(rep["residual"], rb[0]["residual"], rtol=0, atol=1e-12)
    for sa, sb, so in zip(a, b, os_):
        for f in [abi.F_Q + m for m in range(5)] + [abi.F_NUT]:
            assert rel_l2(sa.get_field(1, f), sb.get_field(1, f)) <= 1e-12, f
            assert rel_l2(sa.get_field(1, f), so.get_field(1, f)) <= 1e-10, f
    ex.close()
    X.close()


def test_list_arguments_are_checked():
    from desalm.solver import DesalmError, OvList
    specs, ov = _specs(2)
    a = _solvers(specs)
    c = specs[0][0]
    with pytest.raises(DesalmError):
        OvList(a, [[2, 1, 1, 1]], [[0.5, 0.5, 0.5]])           # no such block
    with pytest.raises(DesalmError):
        OvList(a, [[0, c.im, 1, 1]], [[0.5, 0.5, 0.5]])        # host cell past the block's last cell
    with pytest.raises(DesalmError):
        OvList(a, [[0, 1, c.jm + 1, 1]], None)                 # donee outside the block
    g = OvList(a, [[0, 1, 1, 1]], [[0.0, 0.0, 0.0]])
    assert g.fields(0) == 4 and g.fields(1) == 1
    with pytest.raises(DesalmError):
        g.scatter(0, 0)                                         # a gather list cannot scatter
    g.close()
