"""The FP32 entry points (desalm_set_state_f32, desalm_get_state_f32,
desalm_set_grid_f32) take the reference's real(rdf) = FP32 arrays
(src/precision.F90:11) without a double copy on the caller's side: the
values arrive widened exactly, leave rounded to nearest, and a physical step
begun from them equals the step begun from the same values passed as
doubles, bit for bit."""
import numpy as np
import pytest

from desalm import cases

pytestmark = pytest.mark.gpu


def test_f32_state_and_grid_round_trip():
    from desalm.solver import Solver
    case, grid, state = cases.channel(im=33, jm=25, km=17, seed=4)
    case.use_graph = 0
    f = {k: (None if v is None else np.asarray(v, np.float32)) for k, v in state.items()}
    g32 = {k: (None if v is None else np.asarray(v, np.float32)) for k, v in grid.items()}
    a, b = Solver(case), Solver(case)
    a.set_grid_f32(g32["x"], g32["y"], g32["z"], g32["wd"])
    a.set_state_f32(f["q"], f["qn"], f["qnm1"], f["nut"])
    b.set_grid(*(g32[k].astype(np.float64) for k in ("x", "y", "z", "wd")))
    b.set_state(*(f[k].astype(np.float64) for k in ("q", "qn", "qnm1", "nut")))
    sa = a.get_state()
    for k in ("q", "qn", "qnm1", "nut"):
        assert np.array_equal(sa[k], f[k].astype(np.float64)), k
    ra, rb = a.mg_driver(), b.mg_driver()
    assert ra["iterations"] == rb["iterations"]
    sa, sb = a.get_state(), b.get_state()
    assert np.array_equal(sa["q"], sb["q"])
    s32 = a.get_state_f32()
    for k in ("q", "qn", "qnm1", "nut"):
        assert s32[k].dtype == np.float32
        assert np.array_equal(s32[k], sa[k].astype(np.float32)), k
    a.close()
    b.close()
