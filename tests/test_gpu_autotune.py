"""The autotuner: desalm_set_grid times the DAF sweeps of every level and
direction with the lines-in-lanes kernel and at 16, 8 and 4 slab lines per
CTA, the turbulence sweeps likewise, and the residual kernels (first pass,
recalculation, turbulence residual) at eight CTA tiles of 128 threads (the
first pass and recalculation also as the face-shared kernel, tile 31 x 4 x 2),
and keeps the fastest of each.  Widths and tiles may change the time only, so a
tuned context must step exactly like one on the shared-memory rule and the
default kernels and tile (DESALM_AUTOTUNE=0), and the timing runs must leave the state
alone."""
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


@pytest.mark.parametrize("precision", [abi.FP64, abi.MIXED])
def test_tuned_widths_change_nothing_but_time(precision, monkeypatch):
    case, grid, state = cases.wake(im=65, jm=33, km=33, turbulence=1, seed=4, itmax=5)
    case.precision_mode = precision
    case.use_graph = 1
    tuned = _solver(case, grid, state)
    monkeypatch.setenv("DESALM_AUTOTUNE", "0")
    rule = _solver(case, grid, state)
    monkeypatch.delenv("DESALM_AUTOTUNE")
    w = tuned.sweep_widths()
    assert set(np.unique(w[:case.ng])) <= {1, 2, 4, 8, 16} and not w[case.ng:].any()
    assert set(tuned.turb_sweep_widths()) <= {1, 8, 16, 32}
    assert not rule.turb_sweep_widths().any()
    assert not rule.sweep_widths().any()
    tiles = tuned.kernel_tiles()
    shapes = {(32, 4, 1), (32, 2, 2), (32, 1, 4), (64, 2, 1), (64, 1, 2), (128, 1, 1), (16, 8, 1), (16, 4, 2)}
    for n in range(case.ng):
        for w in range(3 if n == 0 else 2):
            # 31 x 4 x 2 is the face-shared K_R kernel (first pass and recalculation)
            assert tuple(tiles[n, w]) in (shapes | {(31, 4, 2)} if w < 2 else shapes)
    assert all(tuple(t) == (32, 4, 1) for t in rule.kernel_tiles()[:case.ng, :2].reshape(-1, 3))
    # the timing runs at set_grid touched no state
    assert np.array_equal(tuned.get_state()["q"], rule.get_state()["q"])
    for _ in range(2):
        ra, rb = tuned.mg_driver(), rule.mg_driver()
        assert ra["iterations"] == rb["iterations"]
    for k in ("q", "nut"):
        assert np.array_equal(tuned.get_state()[k], rule.get_state()[k]), k
    # setting the grid again re-tunes and drops the captured step
    tuned.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    rule.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    tuned.mg_driver()
    rule.mg_driver()
    assert np.array_equal(tuned.get_state()["q"], rule.get_state()["q"])
