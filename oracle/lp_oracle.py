"""numpy restatement of the learned initial guess (predictor DESALM_PRED_LEARNED).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA
kernels in des-alm_b200/csrc/learn.cuh.  The product never loads it.

The reference has no learned guess: its mg_driver starts every physical step
from q^n (src/mg_driver.F90:48-51), and the linear extrapolation and this
network are extensions on top of that step.  Parity is therefore against this
restatement of the published mathematics the kernels implement (a 3x3x3
convolution with zero padding, ReLU, the mean squared error and its gradient
by back-propagation, Adam after Kingma and Ba, 2015), self-checked by finite
differences in tests/test_lp_oracle.py.  Parity unpinned: there is no
reference output to pin it to.

With quantize=True the functions round to BF16 (round to nearest even) at the
same points as the CUDA path: the features, the weights, the activations of
the hidden layers, the output error and the hidden-layer gradients; all sums
are taken in FP64, so the CUDA path (FP32 sums in another order) differs by
rounding only.  With quantize=False everything is FP64.
"""
import numpy as np

# (cin, cout) of the four layers; 15 input channels = q^n, q^n - q^{n-1},
# q^{n-1} - q^{n-2} of (p, u, v, w, nu_tilde)
LAYERS = [(15, 32), (32, 32), (32, 32), (32, 5)]


def nparam():
    return sum(co * ci * 27 + co for ci, co in LAYERS)


def bf16(a):
    """Round float32 values to BF16 (nearest, ties to even); returns float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32)
    nan = np.isnan(a)
    if nan.any():
        out = out.copy()
        out[nan] = np.nan
    return out


def unflatten(theta):
    """Flat vector -> [(W[cout][cin][27], b[cout])] per layer."""
    theta = np.asarray(theta)
    out, off = [], 0
    for ci, co in LAYERS:
        W = theta[off:off + co * ci * 27].reshape(co, ci, 27)
        off += co * ci * 27
        b = theta[off:off + co]
        off += co
        out.append((W, b))
    return out


def flatten(layers):
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers])


def init_params(seed=0, last_scale=0.1):
    """He-normal weights, zero biases (the CUDA path draws its own with another generator)."""
    rng = np.random.default_rng(seed)
    layers = []
    for l, (ci, co) in enumerate(LAYERS):
        sd = np.sqrt(2.0 / (27.0 * ci)) * (last_scale if l == len(LAYERS) - 1 else 1.0)
        layers.append((rng.normal(0.0, sd, (co, ci, 27)).astype(np.float32), np.zeros(co, np.float32)))
    return flatten(layers)


def _offsets():
    # o = (dk+1)*9 + (dj+1)*3 + (di+1)
    return [(o % 3 - 1, (o // 3) % 3 - 1, o // 9 - 1) for o in range(27)]


def _shift(x, dims, di, dj, dk):
    """x[c][l] -> x[c][l + off] with zeros outside the grid; x is [c, km, jm, im]."""
    im, jm, km = dims
    out = np.zeros_like(x)
    si = slice(max(0, -di), im - max(0, di))
    sj = slice(max(0, -dj), jm - max(0, dj))
    sk = slice(max(0, -dk), km - max(0, dk))
    ti = slice(max(0, di), im - max(0, -di))
    tj = slice(max(0, dj), jm - max(0, -dj))
    tk = slice(max(0, dk), km - max(0, -dk))
    out[:, sk, sj, si] = x[:, tk, tj, ti]
    return out


def conv(x, W, b, dims):
    """y[co][l] = b[co] + sum_{ci,o} W[co][ci][o] x[ci][l + off(o)], FP64 sums."""
    im, jm, km = dims
    xs = np.asarray(x, dtype=np.float64).reshape(-1, km, jm, im)
    y = np.zeros((W.shape[0], km, jm, im))
    for o, (di, dj, dk) in enumerate(_offsets()):
        y += np.tensordot(np.asarray(W[:, :, o], np.float64), _shift(xs, dims, di, dj, dk), axes=(1, 0))
    if b is not None:
        y += np.asarray(b, np.float64)[:, None, None, None]
    return y.reshape(W.shape[0], -1)


def conv_dgrad(dy, W, dims):
    """dx[ci][m] = sum_{co,o} W[co][ci][o] dy[co][m - off(o)] (zero outside the grid)."""
    im, jm, km = dims
    ds = np.asarray(dy, dtype=np.float64).reshape(-1, km, jm, im)
    dx = np.zeros((W.shape[1], km, jm, im))
    for o, (di, dj, dk) in enumerate(_offsets()):
        dx += np.tensordot(np.asarray(W[:, :, o], np.float64).T, _shift(ds, dims, -di, -dj, -dk), axes=(1, 0))
    return dx.reshape(W.shape[1], -1)


def conv_wgrad(x, dy, dims):
    """dW[co][ci][o] = sum_l x[ci][l + off(o)] dy[co][l]."""
    im, jm, km = dims
    xs = np.asarray(x, dtype=np.float64).reshape(-1, km, jm, im)
    d = np.asarray(dy, dtype=np.float64).reshape(-1, km * jm * im)
    dW = np.zeros((d.shape[0], xs.shape[0], 27))
    for o, (di, dj, dk) in enumerate(_offsets()):
        dW[:, :, o] = d @ _shift(xs, dims, di, dj, dk).reshape(xs.shape[0], -1).T
    return dW


def forward(theta, x, dims, quantize=True):
    """Network output y [5, N] (FP32 when quantized) and the hidden activations.

    x: features [15 or 16, N] (channel 15, if present, is ignored)."""
    q = bf16 if quantize else (lambda a: np.asarray(a, np.float64))
    layers = unflatten(theta)
    a = q(np.asarray(x)[:15])
    acts = [a]
    for l, (W, b) in enumerate(layers):
        z = conv(a, q(W), b, dims)
        if l < len(layers) - 1:
            a = q(np.maximum(z, 0.0).astype(np.float32) if quantize else np.maximum(z, 0.0))
            acts.append(a)
        else:
            y = z.astype(np.float32) if quantize else z
    return y, acts


def loss_grad(theta, x, t, dims, quantize=True):
    """Mean squared error over the 5 N outputs and its gradient (flat, FP64)."""
    q = bf16 if quantize else (lambda a: np.asarray(a, np.float64))
    layers = unflatten(theta)
    y, acts = forward(theta, x, dims, quantize)
    t = np.asarray(t, np.float64).reshape(5, -1)
    err = np.asarray(y, np.float64) - t
    loss = float(np.mean(err ** 2))
    g = 2.0 / err.size
    d = q(err.astype(np.float32) if quantize else err)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        grads[l] = (g * conv_wgrad(acts[l], d, dims), g * np.asarray(d, np.float64).sum(axis=1))
        if l > 0:
            dx = conv_dgrad(d, q(W), dims) * (np.asarray(acts[l]) > 0)
            d = q(dx.astype(np.float32) if quantize else dx)
    return loss, flatten(grads)


def scales(qn, qnm1, qnm2):
    """Scales of three time levels ([5, N] FP64 arrays each): rs[16], the
    reciprocal RMS of the 15 feature channels, and s5[5], the RMS of
    (q^n - q^{n-1})_f.  A difference channel whose RMS is not above
    max(1e-12 RMS(q^n_f), 1e-30), or a field channel whose RMS is not above
    1e-30, is still: its rs (and s5) is zero."""
    rs = np.zeros(16, np.float32)
    s5 = np.zeros(5, np.float32)
    for f in range(5):
        rq = np.sqrt(np.sum(qn[f] * qn[f]) / qn[f].size)
        for c, v in enumerate((qn[f], qn[f] - qnm1[f], qnm1[f] - qnm2[f])):
            rms = np.sqrt(np.sum(v * v) / v.size)
            floor = 1e-30 if c == 0 else max(1e-12 * rq, 1e-30)
            if rms > floor:
                rs[3 * f + c] = np.float32(1.0 / rms)
                if c == 1:
                    s5[f] = np.float32(rms)
    return rs, s5


def features(qn, qnm1, qnm2, rs):
    """Scaled BF16 features [16, N] as float32, rounded as the CUDA path does
    (difference in FP64, to FP32, times the FP32 scale, to BF16)."""
    N = qn.shape[1]
    x = np.zeros((16, N), np.float32)
    for f in range(5):
        x[3 * f + 0] = qn[f].astype(np.float32) * rs[3 * f + 0]
        x[3 * f + 1] = (qn[f] - qnm1[f]).astype(np.float32) * rs[3 * f + 1]
        x[3 * f + 2] = (qnm1[f] - qnm2[f]).astype(np.float32) * rs[3 * f + 2]
    return bf16(x)


def target(q, qn, qnm1, rs):
    """(q^{n+1} - 2 q^n + q^{n-1}) / s_f with 1 / s_f = rs[3 f + 1], FP32."""
    rs5 = np.array([rs[3 * f + 1] for f in range(5)], np.float32)
    return ((q - 2.0 * qn + qnm1).astype(np.float32) * rs5[:, None]).astype(np.float32)


def blend(y, t, ymax=8.0):
    """Least-squares factor <y_f, t_f> / <y_f, y_f> of each field, limited to
    [0, 1] (0 when y_f is zero or the ratio is not finite), with y clipped to
    [-ymax, ymax] and non-finite outputs counted as zero."""
    y = np.asarray(y, np.float32)
    yc = np.where(np.isfinite(y), np.clip(y, np.float32(-ymax), np.float32(ymax)), 0.0).astype(np.float64)
    t = np.asarray(t, np.float64)
    a = np.zeros(5, np.float32)
    for f in range(5):
        yy = np.sum(yc[f] * yc[f])
        r = np.sum(yc[f] * t[f]) / yy if yy > 0 else 0.0
        a[f] = np.float32(min(max(r, 0.0), 1.0)) if np.isfinite(r) else 0.0
    return a


def guess(qn, qnm1, y, s5, ymax=8.0, alpha=None):
    """2 q^n - q^{n-1} + s_f alpha_f min(max(y_f, -ymax), ymax) (alpha = 1 by
    default); the linear extrapolation where y is not finite."""
    y = np.asarray(y, np.float32)
    a = np.ones(5, np.float32) if alpha is None else np.asarray(alpha, np.float32)
    sa = (np.asarray(s5, np.float32) * a).astype(np.float32)
    yc = np.clip(y, np.float32(-ymax), np.float32(ymax)).astype(np.float64)
    corr = np.where(np.isfinite(y), sa[:, None].astype(np.float64) * yc, 0.0)
    return 2.0 * qn - qnm1 + corr


def adam(theta, g, m, v, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba, 2015) with bias correction at step t >= 1."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v
