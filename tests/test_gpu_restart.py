"""Checkpoint and restart of a context's device state in the reference's
restart-file layout, and of the learned guess's training state.

- After desalm_checkpoint_read the state equals the FP32 rounding of the
  state written (the reference's files are FP32), and q^{n-1} is zero as after
  the reference's restart.
- One more physical step from the restarted context matches the step from the
  original context to 1e-6 of the largest velocity, in every field: both start
  the step with the same history (the shift refills q^{n-1} from q^n) up to
  that FP32 rounding (6e-8 of the O(1) velocities).  A field's own norm is not
  the scale: the pressure is a near-constant 1e-3 whose variations are what
  the step moves.
- The learned guess's parameters and Adam moments come back bit for bit.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

pytestmark = pytest.mark.gpu


def _solver(case, grid, state):
    from desalm.solver import Solver
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return S


def _f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def test_checkpoint_restart_sa_channel(tmp_path):
    case, grid, state = cases.channel(im=17, jm=17, km=17, itmax=20)
    case.precision_mode = abi.MIXED
    A = _solver(case, grid, state)
    for _ in range(2):
        A.mg_driver()
    p = tmp_path / "solu.000"
    A.checkpoint_write(p)
    before = A.get_state()
    B = _solver(case, grid, state)
    B.checkpoint_read(p)
    got = B.get_state()
    for k in ("q", "qn", "nut"):
        assert np.array_equal(got[k], _f32(before[k])), k
    assert not got["qnm1"].any()
    A.mg_driver()
    B.mg_driver()
    a, b = A.get_state()["q"].reshape(-1, 5), B.get_state()["q"].reshape(-1, 5)
    scale = np.abs(a[:, 1:4]).max()
    for m in range(5):
        assert np.abs(b[:, m] - a[:, m]).max() <= 1e-6 * scale, m


def test_learned_guess_checkpoint(tmp_path):
    case, grid, state = cases.cavity(n=17, seed=2, itmax=8)
    case.predictor = abi.PRED_LEARNED
    A = _solver(case, grid, state)
    A.lp_config(train_steps=3, warm=1)
    for _ in range(3):
        A.mg_driver()
    p = tmp_path / "lp.ckpt"
    A.lp_checkpoint_write(p)
    B = _solver(case, grid, state)
    B.lp_checkpoint_read(p)
    assert np.array_equal(B.lp_params(), A.lp_params())
    assert B.lp_report()["samples"] == A.lp_report()["samples"]
    # the restored moments continue Adam where it stopped: one evaluation of
    # the same features gives the same output and gradient
    N = case.im * case.jm * case.km
    rng = np.random.default_rng(0)
    x = np.zeros((16, N), np.float32)
    x[:15] = rng.normal(size=(15, N))
    t = rng.normal(size=(5, N)).astype(np.float32)
    ya, la, ga = A.lp_eval(x, t)
    yb, lb, gb = B.lp_eval(x, t)
    assert np.array_equal(ya, yb)
    assert abs(la - lb) <= 1e-12 * la  # the loss sums blocks in any order
    assert rel_l2(gb, ga) <= 1e-6
