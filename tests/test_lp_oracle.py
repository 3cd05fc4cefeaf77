"""Self-checks of the numpy restatement of the learned initial guess
(oracle/lp_oracle.py), on the CPU.

There is no reference output for the network (the reference starts each
physical step from q^n), so the oracle is pinned by identities instead: the
data and weight gradients are the adjoints of the convolution, the loss
gradient matches central finite differences, BF16 rounding is nearest-even,
and Adam's first step has its closed form.
"""
import numpy as np

import lp_oracle as lp

DIMS = (5, 4, 3)  # im, jm, km
N = DIMS[0] * DIMS[1] * DIMS[2]


def test_bf16_rounding_is_nearest_even():
    one = np.float32(1.0)
    ulp = np.float32(2.0 ** -7)          # BF16 spacing at 1
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, 1.0 + 2.0 ** -8 + 2.0 ** -20, -2.5, 0.0],
                    dtype=np.float32)
    want = np.array([1.0, 1.0, 1.0 + 2 * ulp, 1.0 + ulp, -2.5, 0.0], dtype=np.float32)
    assert np.array_equal(lp.bf16(vals), want)
    assert np.isnan(lp.bf16(np.array([np.nan], np.float32)))[0]
    assert lp.bf16(np.array([one], np.float32))[0] == one


def test_parameter_count():
    assert lp.nparam() == 72677
    th = lp.init_params(1)
    assert th.size == lp.nparam()
    assert np.array_equal(lp.flatten(lp.unflatten(th)), th)


def test_convolution_adjoints():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(7, N))
    W = rng.normal(size=(6, 7, 27))
    dy = rng.normal(size=(6, N))
    y = lp.conv(x, W, None, DIMS)
    lhs = np.sum(y * dy)
    assert np.isclose(lhs, np.sum(x * lp.conv_dgrad(dy, W, DIMS)), rtol=1e-12)
    assert np.isclose(lhs, np.sum(W * lp.conv_wgrad(x, dy, DIMS)), rtol=1e-12)


def test_convolution_zero_padding_by_loops():
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, N))
    W = rng.normal(size=(3, 2, 27))
    b = rng.normal(size=3)
    y = lp.conv(x, W, b, DIMS)
    im, jm, km = DIMS
    X = x.reshape(2, km, jm, im)
    for (i, j, k) in [(0, 0, 0), (4, 3, 2), (2, 1, 1), (0, 3, 1)]:
        s = b.copy()
        for o in range(27):
            di, dj, dk = o % 3 - 1, (o // 3) % 3 - 1, o // 9 - 1
            ii, jj, kk = i + di, j + dj, k + dk
            if 0 <= ii < im and 0 <= jj < jm and 0 <= kk < km:
                s += W[:, :, o] @ X[:, kk, jj, ii]
        assert np.allclose(y[:, i + im * (j + jm * k)], s, rtol=1e-12, atol=1e-12)


def test_loss_gradient_matches_finite_differences():
    rng = np.random.default_rng(2)
    theta = lp.init_params(3, last_scale=1.0).astype(np.float64)
    theta += rng.normal(0.0, 0.01, theta.size)          # non-zero biases too
    x = rng.normal(size=(16, N))
    t = rng.normal(size=(5, N))
    loss, g = lp.loss_grad(theta, x, t, DIMS, quantize=False)
    idx = np.concatenate([rng.choice(theta.size, 40, replace=False),
                          [0, theta.size - 1, lp.nparam() - 5]])  # includes output biases
    h = 1e-6
    for e in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[e] += h
        tm[e] -= h
        fd = (lp.loss_grad(tp, x, t, DIMS, quantize=False)[0] - lp.loss_grad(tm, x, t, DIMS, quantize=False)[0]) / (2 * h)
        assert abs(fd - g[e]) <= 1e-6 * max(1.0, abs(g[e])) + 1e-9, (e, fd, g[e])


def test_quantized_close_to_exact():
    rng = np.random.default_rng(4)
    theta = lp.init_params(5, last_scale=1.0)
    x = rng.normal(size=(16, N)).astype(np.float32)
    t = rng.normal(size=(5, N)).astype(np.float32)
    y_q, _ = lp.forward(theta, x, DIMS, quantize=True)
    y_e, _ = lp.forward(theta, x, DIMS, quantize=False)
    assert np.linalg.norm(y_q - y_e) / np.linalg.norm(y_e) < 2e-2
    l_q, g_q = lp.loss_grad(theta, x, t, DIMS, quantize=True)
    l_e, g_e = lp.loss_grad(theta, x, t, DIMS, quantize=False)
    assert abs(l_q - l_e) / l_e < 1e-2
    assert np.linalg.norm(g_q - g_e) / np.linalg.norm(g_e) < 3e-2


def test_adam_first_step_closed_form():
    theta = np.array([1.0, -2.0, 0.5])
    g = np.array([0.3, -4.0, 0.0])
    th, m, v = lp.adam(theta, g, np.zeros(3), np.zeros(3), 1, lr=0.01)
    # first step: m_hat = g, v_hat = g^2 -> theta - lr g / (|g| + eps)
    assert np.allclose(th, theta - 0.01 * g / (np.abs(g) + 1e-8))


def test_features_target_guess_identities():
    rng = np.random.default_rng(6)
    qnm2 = rng.normal(size=(5, N))
    qnm1 = qnm2 + 0.01 * rng.normal(size=(5, N))
    qn = qnm1 + 0.01 * rng.normal(size=(5, N))
    q = 2 * qn - qnm1 + 1e-4 * rng.normal(size=(5, N))
    rs, s5 = lp.scales(qn, qnm1, qnm2)
    x = lp.features(qn, qnm1, qnm2, rs)
    assert x.shape == (16, N) and not x[15].any()
    # every scaled channel has RMS ~1 (up to BF16 rounding)
    rms = np.sqrt(np.mean(x[:15].astype(np.float64) ** 2, axis=1))
    assert np.allclose(rms, 1.0, atol=1e-2)
    t = lp.target(q, qn, qnm1, rs)
    # the guess with the exact target as output reproduces q to FP32 rounding
    assert np.allclose(lp.guess(qn, qnm1, t, s5, ymax=1e30), q, rtol=0, atol=1e-9)
    # a non-finite output keeps the linear extrapolation
    y = t.copy()
    y[:, 3] = np.nan
    gq = lp.guess(qn, qnm1, y, s5)
    assert np.array_equal(gq[:, 3], 2.0 * qn[:, 3] - qnm1[:, 3])
    # the output is limited to [-ymax, ymax] scale units
    y = np.full_like(t, 100.0)
    assert np.allclose(lp.guess(qn, qnm1, y, s5, ymax=8.0) - (2.0 * qn - qnm1), 8.0 * s5[:, None].astype(np.float64))


def test_still_channels_have_zero_scale():
    rng = np.random.default_rng(7)
    qn = rng.normal(size=(5, N))
    qn[4] = 0.0                                   # a zero field
    qnm1 = qn.copy()
    qnm1[1] += 1e-3 * rng.normal(size=N)          # only u moves between n-1 and n
    qnm2 = qnm1 + 1e-15 * qn                      # below 1e-12 of the field: still
    rs, s5 = lp.scales(qn, qnm1, qnm2)
    assert rs[3 * 4] == 0 and rs[15] == 0
    for f in range(5):
        assert (s5[f] > 0) == (f == 1) and (rs[3 * f + 1] > 0) == (f == 1)
        assert rs[3 * f + 2] == 0
    t = lp.target(qn + 1e-3, qn, qnm1, rs)
    assert not t[[0, 2, 3, 4]].any() and t[1].any()


def test_blend_least_squares_factor():
    rng = np.random.default_rng(8)
    t = rng.normal(size=(5, N)).astype(np.float32)
    y = np.stack([2 * t[0], -t[1], np.zeros(N), 0.5 * t[3], t[4]]).astype(np.float32)
    y[4, 0] = np.nan
    a = lp.blend(y, t, ymax=1e30)
    assert np.allclose(a[[0, 1, 2, 3]], [0.5, 0.0, 0.0, 1.0], atol=1e-6)
    assert 0.0 < a[4] <= 1.0
    # the blended correction never does worse than none on the sample it was fitted to
    for f in range(5):
        yc = np.where(np.isfinite(y[f]), y[f], 0.0).astype(np.float64)
        assert np.sum((t[f] - a[f] * yc) ** 2) <= np.sum(t[f].astype(np.float64) ** 2) + 1e-9
