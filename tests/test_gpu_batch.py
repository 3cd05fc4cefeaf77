"""desalm_mg_driver_batch: independent blocks of uneven sizes stepped together
(their captured steps in flight at once) must each equal the block stepped
alone with desalm_mg_driver, bit for bit, reports included; contexts off the
graph path (eager, or the learned guess) step in turn inside the batch with
the same result."""
import numpy as np
import pytest

from desalm import abi, cases

pytestmark = pytest.mark.gpu

SHAPES = [(17, 17, 17, 1, 1), (25, 17, 21, 0, 1), (33, 17, 17, 1, 0), (21, 21, 17, 1, 1)]


def _block(shape, seed):
    im, jm, km, turb, graph = shape
    case, grid, state = cases.wake(im=im, jm=jm, km=km, turbulence=turb, seed=seed, itmax=6)
    case.it_min = 2
    case.use_graph = graph
    case.precision_mode = abi.MIXED if seed % 2 else abi.FP64
    case.predictor = abi.PRED_LINEAR
    return case, grid, state


def _solver(case, grid, state):
    from desalm.solver import Solver
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return S


def test_batch_equals_blocks_alone():
    from desalm.solver import mg_driver_batch
    blocks = [_block(s, b) for b, s in enumerate(SHAPES)]
    alone = [_solver(*b) for b in blocks]
    batch = [_solver(*b) for b in blocks]
    for step in range(3):
        ra = [S.mg_driver() for S in alone]
        rb = mg_driver_batch(batch)
        for a, b in zip(ra, rb):
            assert a["iterations"] == b["iterations"] and a["converged"] == b["converged"]
            assert np.array_equal(a["residual"], b["residual"])
    for a, b in zip(alone, batch):
        sa, sb = a.get_state(), b.get_state()
        for k in ("q", "qn", "nut"):
            assert np.array_equal(sa[k], sb[k]), k


def test_batch_with_a_learned_block():
    from desalm.solver import mg_driver_batch
    blocks = [_block(SHAPES[0], 0), _block(SHAPES[2], 1)]
    blocks[1][0].predictor = abi.PRED_LEARNED
    alone = [_solver(*b) for b in blocks]
    batch = [_solver(*b) for b in blocks]
    for S in alone + batch:
        if S.case.predictor == abi.PRED_LEARNED:
            S.lp_config(train_steps=2, warm=1)
    for step in range(3):
        for S in alone:
            S.mg_driver()
        mg_driver_batch(batch)
    for a, b in zip(alone, batch):
        assert np.array_equal(a.get_state()["q"], b.get_state()["q"])
