"""The k-omega model (turbulence = 2) on the GPU through the C ABI, against
the oracle's restatement (parity unpinned: the reference builds none of it).
- one desalm_kw_eddy call, FP64: k, omega and nu_t at relative L2 <= 1e-12,
  on a channel with walls and on an open wake box (inflow, characteristics
  outlet, symmetry and periodic faces), and on a box walled on every face
  (the wall-edge averages);
- three pseudo-iterations with the model: <= 1e-10 in FP64, <= 5e-5 in MIXED
  (FP32 ADI rows and line solves) for q, omega and nu_t;
- the graph-replayed physical step equals the eager one bit for bit.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _case(which):
    if which == "channel":
        case, grid, state = cases.channel(im=33, jm=33, km=17, seed=11)
    elif which == "wake":
        case, grid, state = cases.wake(im=41, jm=17, km=17, seed=12)
    else:
        case, grid, state = cases.cavity(n=17, seed=13)
        x, y, z = grid["x"], grid["y"], grid["z"]
        grid["wd"] = np.minimum.reduce([x, 1 - x, y, 1 - y, z, 1 - z]) + 1e-3
    return cases.with_kw(case, grid, state)


def _pair(which, precision, oracle_mod, graph=0):
    from desalm.solver import Solver
    c, g, st, om = _case(which)
    c.precision_mode = precision
    c.use_graph = graph
    gpu = Solver(c)
    o = oracle_mod.OracleSolver(c)
    for s in (gpu, o):
        s.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
        s.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
        s.set_omega(om["omega"], om["omega_n"], om["omega_nm1"])
    return c, gpu, o


def _errs(gpu, o):
    return {"k": rel_l2(gpu.get_field(1, abi.F_Q + 4), o.get_field(1, abi.F_Q + 4)),
            "omega": rel_l2(gpu.get_omega()["omega"], o.get_omega()["omega"]),
            "nu_t": rel_l2(gpu.get_field(1, abi.F_NUT), o.get_field(1, abi.F_NUT))}


@pytest.mark.parametrize("which", ["channel", "wake", "walls"])
def test_kw_eddy_call(which, oracle_mod):
    c, gpu, o = _pair(which, abi.FP64, oracle_mod)
    for s in (gpu, o):
        s.kw_eddy()
    e = _errs(gpu, o)
    assert max(e.values()) <= 1e-12, e
    gpu.close()


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
@pytest.mark.parametrize("which", ["channel", "wake"])
def test_kw_pseudo_iterations(which, precision, oracle_mod):
    c, gpu, o = _pair(which, precision, oracle_mod)
    gpu.begin_step()
    o.begin_step()
    for _ in range(3):
        gpu.pseudo_iteration()
        o.pseudo_iteration()
    tol = 1e-10 if precision == abi.FP64 else 5e-5
    e = _errs(gpu, o)
    for m in range(4):
        e["q%d" % m] = rel_l2(gpu.get_field(1, abi.F_Q + m), o.get_field(1, abi.F_Q + m))
    assert max(e.values()) <= tol, e
    gpu.close()


def test_kw_graph_matches_eager(oracle_mod):
    from desalm.solver import Solver
    c, g, st, om = _case("wake")
    c.predictor = abi.PRED_LINEAR
    c.itmax = 6
    c.it_min = 2
    c.er_min = -0.5
    out = []
    for graph in (0, 1):
        cc = c.copy()
        cc.use_graph = graph
        s = Solver(cc)
        s.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
        s.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
        s.set_omega(om["omega"], om["omega_n"], om["omega_nm1"])
        reps = [s.mg_driver() for _ in range(3)]
        out.append((reps, s.get_state(), s.get_omega()))
        s.close()
    (r0, s0, w0), (r1, s1, w1) = out
    assert [a["iterations"] for a in r0] == [b["iterations"] for b in r1]
    assert np.array_equal(s0["q"], s1["q"])
    assert np.array_equal(w0["omega"], w1["omega"])
