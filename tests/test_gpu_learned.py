"""The learned initial guess (predictor DESALM_PRED_LEARNED) on the GPU
against the numpy restatement in oracle/lp_oracle.py, through the C ABI.

Tolerances:
- network output, loss and whole parameter gradient against the oracle
  rounded to BF16 at the same points: relative L2 <= 2e-3 (the tensor cores
  sum in FP32 in another order; a sum that lands on the other side of a BF16
  rounding boundary moves one activation by one BF16 ulp); each layer's share
  of the gradient: <= 1e-2, since those flips compound through the backward
  chain and the first layer's gradient sums, with cancellation, over few
  nodes on the small grid (measured on a B200: output 2.4e-4, first layer
  3.7e-3 at 17^3 and 7.7e-4 at 41^3, the same at every stencil offset; the
  other layers <= 4e-4);
- against the all-FP64 oracle: relative L2 <= 3e-2 (BF16 quantisation);
- scales and targets: relative 1e-6 (FP64 RMS sums in another order may move
  a scale by one FP32 ulp); features given the GPU's scales: bit-identical;
- zero network, or a network whose output is not finite: bit-identical to the
  linear extrapolation.
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases

import lp_oracle as lp

pytestmark = pytest.mark.gpu


def _solver(case, grid, state):
    from desalm.solver import Solver
    S = Solver(case)
    S.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    S.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    return S


def _cavity(n, predictor, itmax=12):
    case, grid, state = cases.cavity(n=n, seed=5, itmax=itmax)
    case.predictor = predictor
    return case, grid, state


def _soa(a):
    """AoS q(5, i, j, k) -> [5, N]."""
    return np.asarray(a).reshape(-1, 5).T.copy()


@pytest.mark.parametrize("n", [17, 41])
def test_network_forward_and_gradient_match_oracle(n):
    """17^3: one partial tile; 41^3: 539 tiles, more than the grid, so the
    convolution's tile loop strides and the last tile is partial."""
    case, grid, state = _cavity(n, abi.PRED_LEARNED)
    S = _solver(case, grid, state)
    dims = (case.im, case.jm, case.km)
    N = case.im * case.jm * case.km
    rng = np.random.default_rng(n)
    theta = lp.init_params(seed=n, last_scale=1.0)
    theta[lp.nparam() - 5:] = rng.normal(0.0, 0.1, 5)        # output biases
    S.lp_set_params(theta)
    x = np.zeros((16, N), np.float32)
    x[:15] = rng.normal(size=(15, N))
    t = rng.normal(size=(5, N)).astype(np.float32)
    y, loss, grad = S.lp_eval(x, t)
    y_q, _ = lp.forward(theta, x, dims, quantize=True)
    loss_q, grad_q = lp.loss_grad(theta, x, t, dims, quantize=True)
    assert rel_l2(y, y_q) <= 2e-3
    assert abs(loss - loss_q) <= 2e-3 * loss_q
    assert rel_l2(grad, grad_q) <= 2e-3
    # per layer too: each layer's share of the gradient is checked separately
    off = 0
    for ci, co in lp.LAYERS:
        nl = co * ci * 27 + co
        assert rel_l2(grad[off:off + nl], grad_q[off:off + nl]) <= 1e-2, (ci, co)
        off += nl
    y_e, _ = lp.forward(theta, x, dims, quantize=False)
    assert rel_l2(y, y_e) <= 3e-2
    _, grad_e = lp.loss_grad(theta, x, t, dims, quantize=False)
    assert rel_l2(grad, grad_e) <= 3e-2
    # the parameters are untouched by an evaluation
    assert np.array_equal(S.lp_params(), theta)


def _run(predictor, steps, setup=None, n=17):
    case, grid, state = _cavity(n, predictor)
    S = _solver(case, grid, state)
    if setup:
        setup(S)
    reps = [S.mg_driver() for _ in range(steps)]
    return S, S.get_state(), reps


def test_zero_network_is_linear_extrapolation_bitwise():
    def setup(S):
        S.lp_set_params(np.zeros(lp.nparam(), np.float32))
        S.lp_config(train_steps=2, warm=0, lr=0.0)
    S, st, reps = _run(abi.PRED_LEARNED, 4, setup)
    _, st_lin, reps_lin = _run(abi.PRED_LINEAR, 4)
    for k in ("q", "qn", "qnm1", "nut"):
        assert np.array_equal(st[k], st_lin[k]), k
    assert [r["iterations"] for r in reps] == [r["iterations"] for r in reps_lin]
    assert S.lp_report()["alpha"] == [0.0] * 5
    r = S.lp_report()
    # step 1 cannot train (q^{n-2} unknown); steps 2..4 train on one sample each
    assert r["samples"] == 3 and r["train_steps"] == 6 and r["predictions"] == 4
    assert np.array_equal(S.lp_params(), np.zeros(lp.nparam(), np.float32))


def test_masked_fields_keep_the_linear_guess():
    """desalm_lp_fields: a field whose bit is clear takes no correction; with
    every bit clear a trained network gives the linear run bit for bit, and
    with only p's bit set u, v, w follow the linear guess at each step's
    start."""
    def none(S):
        S.lp_config(train_steps=2, warm=0)
        S.lp_fields(0)
    S, st, reps = _run(abi.PRED_LEARNED, 4, none)
    _, st_lin, reps_lin = _run(abi.PRED_LINEAR, 4)
    for k in ("q", "qn", "qnm1", "nut"):
        assert np.array_equal(st[k], st_lin[k]), k
    assert S.lp_report()["alpha"] == [0.0] * 5
    assert S.lp_report()["train_steps"] > 0
    with pytest.raises(Exception):
        S.lp_fields(32)

    def p_only(S):
        S.lp_config(train_steps=2, warm=0)
        S.lp_fields(1)
    S, _, _ = _run(abi.PRED_LEARNED, 3, p_only)
    assert S.lp_report()["alpha"][1:] == [0.0] * 4


def test_learned_runs_repeat_bit_for_bit():
    """The learned guess's sums (scales, loss, held-out dots) add their
    per-CTA partials in a fixed order, so two identical runs agree bit for
    bit: parameters, report and state."""
    def setup(S):
        S.lp_config(train_steps=3, warm=1)
    A, sa, ra = _run(abi.PRED_LEARNED, 4, setup)
    B, sb, rb = _run(abi.PRED_LEARNED, 4, setup)
    assert np.array_equal(A.lp_params(), B.lp_params())
    assert A.lp_report() == B.lp_report()
    for k in ("q", "qn", "qnm1", "nut"):
        assert np.array_equal(sa[k], sb[k]), k
    assert [r["iterations"] for r in ra] == [r["iterations"] for r in rb]


def test_non_finite_network_output_falls_back_to_linear():
    def setup(S):
        th = np.zeros(lp.nparam(), np.float32)
        th[lp.nparam() - 5:] = np.nan                        # every output NaN
        S.lp_set_params(th)
        S.lp_config(train_steps=1, warm=0, lr=0.0)
    S, st, _ = _run(abi.PRED_LEARNED, 3, setup)
    _, st_lin, _ = _run(abi.PRED_LINEAR, 3)
    for k in ("q", "qn", "qnm1"):
        assert np.array_equal(st[k], st_lin[k]), k
    assert np.isnan(S.lp_buffer(abi.LP_OUTPUT)).all()


def test_features_targets_and_guess_match_oracle():
    case, grid, state = _cavity(17, abi.PRED_LEARNED)
    S = _solver(case, grid, state)
    S.lp_config(train_steps=3, warm=1, lr=1e-3)
    hist = [_soa(state["qnm1"]), _soa(state["qn"]), _soa(state["q"])]   # oldest first
    checked = 0
    for step in range(5):
        before = S.get_state()
        q, qn, qnm1 = _soa(before["q"]), _soa(before["qn"]), _soa(before["qnm1"])
        S.begin_step()
        r = S.lp_report()
        if step >= 1:
            # this step's sample: scales of (q^n, q^{n-1}, q^{n-2}) as they
            # were before the shift, target from the converged q
            rs_learn, _ = lp.scales(qn, qnm1, hist[-4])
            t = S.lp_buffer(abi.LP_TARGET)
            want = lp.target(q, qn, qnm1, rs_learn)
            assert np.allclose(t, want, rtol=1e-6, atol=1e-6 * max(1e-30, np.abs(want).max()))
        if r["predictions"] > 0 and step >= 1:
            # the guess: scales and features of (q, q^n, q^{n-1}) after the shift
            rs, s5 = lp.scales(q, qn, qnm1)
            got_rs = S.lp_buffer(abi.LP_SCALES)
            assert np.array_equal(got_rs > 0, rs > 0)
            assert np.allclose(got_rs, rs, rtol=1e-6, atol=0)
            x = S.lp_buffer(abi.LP_FEATURES)
            assert np.array_equal(x, lp.features(q, qn, qnm1, got_rs))
            y = S.lp_buffer(abi.LP_OUTPUT)
            alpha = S.lp_buffer(abi.LP_ALPHA)
            assert ((alpha >= 0) & (alpha <= 1)).all()
            s5_gpu = np.array([np.float32(1.0) / got_rs[3 * f + 1] if got_rs[3 * f + 1] > 0 else 0.0
                               for f in range(5)], np.float32)
            assert np.allclose(s5_gpu, s5, rtol=1e-6, atol=0)
            g = _soa(S.get_state()["q"])
            assert np.allclose(g, lp.guess(q, qn, y, s5, alpha=alpha), rtol=0, atol=1e-6 * max(1.0, np.abs(g).max()))
            checked += 1
        S.pseudo_iteration()
        hist.append(_soa(S.get_state()["q"]))
    assert S.lp_report()["samples"] == 4 and checked == 4


def test_blown_up_learned_step_restarts_from_linear_guess():
    """A network whose output is huge but finite (no output limit): the step
    begun from its guess ends with a non-finite norm, desalm_mg_driver starts
    it again from the linear extrapolation, and the run then matches the
    linear run bit for bit; the next guesses wait for warm more samples."""
    def setup(S):
        th = np.zeros(lp.nparam(), np.float32)
        th[lp.nparam() - 5:] = 1e30
        S.lp_set_params(th)
        S.lp_config(train_steps=1, warm=2, lr=0.0, ymax=3e38)
        S.lp_blend(1.0)                                      # no held-out damping
        S.lp_fields(0x1f)                                    # every field corrected
    S, st, reps = _run(abi.PRED_LEARNED, 4, setup)
    _, st_lin, reps_lin = _run(abi.PRED_LINEAR, 4)
    r = S.lp_report()
    # steps 1-2: too few samples; step 3: guess, blow-up, restart; step 4: held
    assert r["predictions"] == 1 and r["fallbacks"] == 1, r
    for k in ("q", "qn", "qnm1", "nut"):
        assert np.array_equal(st[k], st_lin[k]), k
    assert [x["iterations"] for x in reps] == [x["iterations"] for x in reps_lin]


def test_training_lowers_the_loss_on_a_sample():
    """Two physical steps: the second trains 40 Adam steps on its one sample;
    the loss of the last step is below that of the first."""
    def setup(S):
        S.lp_config(train_steps=40, warm=100, lr=1e-3)
    S, st, _ = _run(abi.PRED_LEARNED, 2, setup)
    r = S.lp_report()
    assert r["samples"] == 1 and r["train_steps"] == 40 and r["predictions"] == 0
    assert np.isfinite(r["first_loss"]) and np.isfinite(r["last_loss"])
    assert r["last_loss"] < r["first_loss"], r


def test_heldout_blend_matches_oracle():
    """With no training steps and no guesses, the output buffer after a
    sample is the held-out pass of the current network on it: the blend and
    the held-out error ratio follow from it and the target."""
    def setup(S):
        S.lp_set_params(lp.init_params(seed=11, last_scale=1.0))
        S.lp_config(train_steps=0, warm=100)
        S.lp_fields(0x1f)                                    # the oracle blends every field
    S, _, _ = _run(abi.PRED_LEARNED, 3, setup)
    y = S.lp_buffer(abi.LP_OUTPUT)
    t = S.lp_buffer(abi.LP_TARGET)
    want = lp.blend(y, t)
    got = S.lp_buffer(abi.LP_ALPHA)
    assert np.allclose(got, want, rtol=1e-5, atol=1e-7)
    r = S.lp_report()
    a = want.astype(np.float64)
    yc = np.clip(y, -8.0, 8.0).astype(np.float64)
    num = sum(np.sum((t[f] - a[f] * yc[f]) ** 2) for f in range(5))
    den = sum(np.sum(t[f].astype(np.float64) ** 2) for f in range(5))
    assert abs(r["heldout_ratio"] - num / den) <= 1e-5 * max(1.0, num / den)
    assert r["heldout_ratio"] <= 1.0 + 1e-9
