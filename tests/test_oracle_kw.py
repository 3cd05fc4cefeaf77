"""The k-omega restatement on the CPU (src/kw_eddy.F90 and its rhs_kw_*
routines; the reference builds none of it, so parity is unpinned).  These
identities pin what can be pinned without the reference:
- mirror equivariance: reflecting the problem in i (x -> -x with the node
  order reversed, u -> -u) must reflect kw_eddy's result, to round-off, on a
  channel with walls (wall values, wall-edge averages), periodic i faces and
  a perturbed state; a flux or stencil taken on the wrong side breaks it;
- the coefficients are Wilcox's (1994) low-Reynolds-number functions:
  alpha* = (beta0/3 + Re_t/6) / (1 + Re_t/6) with beta0 = 0.075, and
  nu_t = alpha* k / omega after every sub-iteration;
- wall faces get k = 0 and omega = 60 / (Re 0.075 y^2) from the adjacent
  node's wall distance.
"""
import numpy as np

from conftest import rel_l2
from desalm import abi, cases


def _kw_channel(seed=3, im=17, jm=21, km=13):
    case, grid, state = cases.channel(im=im, jm=jm, km=km, seed=seed)
    c, g, st, om = cases.with_kw(case, grid, state)
    rng = np.random.default_rng(seed)
    N = c.im * c.jm * c.km
    q = st["q"].reshape(N, 5)
    inner = q[:, 4] > 0
    q[inner, 4] *= np.exp(rng.normal(0, 0.3, inner.sum()))
    w = om["omega"] * np.exp(rng.normal(0, 0.3, N))
    st["q"] = q.reshape(-1)
    om = dict(omega=w, omega_n=w * 1.01, omega_nm1=w * 1.02)
    st["nut"] = cases.kw_coef_as(q[:, 4], w, c.ren) * q[:, 4] / w
    return c, g, st, om


def _run(oracle_mod, c, g, st, om):
    o = oracle_mod.OracleSolver(c)
    o.set_grid(g["x"], g["y"], g["z"], g.get("wd"))
    o.set_state(st["q"], st["qn"], st["qnm1"], st["nut"])
    o.set_omega(om["omega"], om["omega_n"], om["omega_nm1"])
    o.kw_eddy()
    return o.get_field(1, abi.F_Q + 4), o.get_omega()["omega"], o.get_field(1, abi.F_NUT)


def _mirror(a, c, comp=None, flip=()):
    """Reverse the i order of an (i, j, k) array or a (1:5, i, j, k) array."""
    if comp is None:
        return np.ascontiguousarray(a.reshape(c.km, c.jm, c.im)[:, :, ::-1]).reshape(-1)
    b = a.reshape(c.km, c.jm, c.im, comp)[:, :, ::-1, :].copy()
    for m in flip:
        b[..., m] = -b[..., m]
    return b.reshape(-1)


def test_kw_eddy_mirror_equivariance(oracle_mod):
    c, g, st, om = _kw_channel()
    c.itk = 2
    k1, w1, n1 = _run(oracle_mod, c, g, st, om)
    gm = dict(x=-_mirror(g["x"], c), y=_mirror(g["y"], c), z=_mirror(g["z"], c), wd=_mirror(g["wd"], c))
    stm = {key: _mirror(st[key], c, 5, flip=(1,)) for key in ("q", "qn", "qnm1")}
    stm["nut"] = _mirror(st["nut"], c)
    omm = {key: _mirror(om[key], c) for key in om}
    k2, w2, n2 = _run(oracle_mod, c, gm, stm, omm)
    assert rel_l2(_mirror(k2, c), k1) < 1e-12
    assert rel_l2(_mirror(w2, c), w1) < 1e-12
    assert rel_l2(_mirror(n2, c), n1) < 1e-12
    assert rel_l2(k1, st["q"].reshape(-1, 5)[:, 4]) > 1e-6    # the step did something


def test_kw_coefficients_and_walls(oracle_mod):
    c, g, st, om = _kw_channel(seed=5)
    c.itk = 1
    k, w, nut = _run(oracle_mod, c, g, st, om)
    rt = c.ren * k / w
    astar = (0.075 / 3 + rt / 6) / (1 + rt / 6)
    assert np.allclose(nut, astar * k / w, rtol=1e-12, atol=0)
    kk, ww = k.reshape(c.km, c.jm, c.im), w.reshape(c.km, c.jm, c.im)
    wd = g["wd"].reshape(c.km, c.jm, c.im)
    srenp = 60.0 / c.ren / 0.075
    # j = 1 and j = jm are walls; the i and k faces are periodic (no wall edges)
    assert np.all(kk[:, 0, :] == 0) and np.all(kk[:, -1, :] == 0)
    assert np.allclose(ww[:, 0, :], srenp / wd[:, 1, :] ** 2, rtol=1e-14)
    assert np.allclose(ww[:, -1, :], srenp / wd[:, -2, :] ** 2, rtol=1e-14)


def test_kw_wall_edges_average(oracle_mod):
    """A box with walls on every face: omega on each wall edge is the mean of
    its two face neighbours, edges in the reference's order."""
    case, grid, state = cases.cavity(n=13, seed=2)
    N = case.im * case.jm * case.km
    x, y, z = grid["x"], grid["y"], grid["z"]
    grid["wd"] = np.minimum.reduce([x, 1 - x, y, 1 - y, z, 1 - z]) + 1e-3
    case.btype[3] = abi.BC_WALL
    c, g, st, om = cases.with_kw(case, grid, state)
    c.itk = 1
    k, w, nut = _run(oracle_mod, c, g, st, om)
    W = w.reshape(c.km, c.jm, c.im)
    # edge (i = 1, j = 1) at an interior k: set after every face
    kk = c.km // 2
    assert np.isclose(W[kk, 0, 0], 0.5 * (W[kk, 0, 1] + W[kk, 1, 0]), rtol=1e-14)
    # the corner (1, 1, 1): last written by the edge (j = 1, k = 1)
    assert np.isclose(W[0, 0, 0], 0.5 * (W[0, 1, 0] + W[1, 0, 0]), rtol=1e-14)
