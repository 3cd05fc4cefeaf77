"""Known answers for the oracle's characteristics outlet (btype 5) on the CPU.

The reference ships no output for it either, so its restatement is pinned by
identities of the mathematics it implements:
  * the closed form of nonreflect_ibc (src/nonreflect_ibc.F90:139-240) is the
    outgoing part A+ = V diag(max(lambda, 0)) V^-1 of the beta = 1
    pseudo-compressibility flux Jacobian A in csi, applied to the one-sided
    difference q(im) - q(im-1) and divided by J: checked against numpy's
    eigen-decomposition of A on a sheared affine grid, for outflow (ucon > 0:
    three outgoing characteristics) and backflow (ucon < 0: one);
  * mg_brhs's 2D residual equals the interior residual of any plane when the
    state does not vary along i on an affine grid (every csi term and the
    LODI terms vanish then), which pins the brhs_* restatement on the
    interior residual's;
  * a uniform stream is a fixed point of a DAF step with the outlet solved;
  * rhs_sa_bcond's btype-5 rows extrapolate nu_tilde with the grid ratio
    (src/rhs_sa_bcond.F90:61-67, 98-104, 144-150, 181-187);
  * a btype-5 face other than i = im keeps its values (bcond_fm's case(5)
    branches are empty, src/bcond_fm.F90:104, 138-152, 196, 230, 264, 298).
"""
import numpy as np
import pytest

from desalm import abi, cases


def _affine_case(n=13):
    case, _, _ = cases.wake(im=n, jm=n, km=n, turbulence=0)
    s = np.arange(n, dtype=float) / (n - 1)
    K, J, I = np.meshgrid(s, s, s, indexing="ij")
    A = np.array([[2.0, 0.3, 0.1], [0.2, 1.5, -0.4], [0.1, 0.25, 3.0]])
    P = np.stack([I, J, K], -1) @ A.T
    grid = dict(x=P[..., 0].reshape(-1), y=P[..., 1].reshape(-1), z=P[..., 2].reshape(-1))
    return case, grid


def _jacobian_plus(c, vel):
    u, v, w = vel
    c1, c2, c3 = c
    ucon = c1 * u + c2 * v + c3 * w
    A = np.array([[0.0, c1, c2, c3],
                  [c1, ucon + c1 * u, c2 * u, c3 * u],
                  [c2, c1 * v, ucon + c2 * v, c3 * v],
                  [c3, c1 * w, c2 * w, ucon + c3 * w]])
    lam, V = np.linalg.eig(A)
    lam, V = lam.real, V.real
    return (V * np.maximum(lam, 0.0)) @ np.linalg.inv(V), ucon


@pytest.mark.parametrize("u0", [1.0, -0.5])
def test_lodi_is_the_outgoing_characteristic_part(u0, oracle_mod):
    n = 13
    case, grid = _affine_case(n)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    # a state that varies along i only and is steady: every eta / zeta term of
    # the plane's residual vanishes, only the LODI csi terms remain
    i = np.arange(n, dtype=float)
    q = np.zeros((n, n, n, 5))
    q[..., 0] = (0.01 + 0.003 * i)[None, None, :]
    q[..., 1] = (u0 + 0.02 * i)[None, None, :]
    q[..., 2] = (0.1 - 0.01 * i)[None, None, :]
    q[..., 3] = (-0.05 + 0.015 * i)[None, None, :]
    q = q.reshape(-1)
    o.set_state(q, q, q)
    rh = o.outlet_rhs()
    csi = np.array([o.get_field(1, abi.F_CSI + d).reshape(n, n, n)[5, 6, -1] for d in range(3)])
    aj = o.get_field(1, abi.F_AJ).reshape(n, n, n)[5, 6, -1]
    qq = q.reshape(n, n, n, 5)
    vel = qq[5, 6, -1, 1:4]
    dq = qq[5, 6, -1, :4] - qq[5, 6, -2, :4]
    Ap, ucon = _jacobian_plus(csi, vel)
    assert (ucon > 0) == (u0 > 0)
    want = Ap @ dq / aj
    got = rh[:, 5, 6]
    assert np.allclose(got, want, rtol=1e-10, atol=1e-12 * np.abs(want).max()), (got, want)
    # every interior node of the plane sees the same affine metrics and state
    inner = rh[:, 1:-1, 1:-1].reshape(4, -1)
    assert np.allclose(inner, got[:, None], rtol=1e-9, atol=1e-13)
    # and the plane's edges keep rh = 0
    assert not rh[:, 0, :].any() and not rh[:, :, 0].any()


def test_uniform_stream_is_a_fixed_point(oracle_mod):
    n = 13
    case, _, _ = cases.wake(im=n, jm=n, km=n, turbulence=0)
    s = np.linspace(0.0, 1.0, n)
    X, Y, Z = cases._mesh(1.5 * s, s, s)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(X.reshape(-1), Y.reshape(-1), Z.reshape(-1))
    q = np.zeros((n ** 3, 5))
    q[:, 1], q[:, 3] = 1.0, 0.3          # p = 0: bcond_fm subtracts p(ifix, jfix, kfix)
    q = q.reshape(-1)
    o.set_state(q, q, q)
    assert np.abs(o.outlet_rhs()).max() < 1e-12
    o.solver_daf(1, 0, 1)
    assert np.allclose(o.get_state()["q"], q, rtol=0, atol=1e-12)


def test_sa_btype5_extrapolation(oracle_mod):
    n = 13
    case, grid, state = cases.wake(im=n, jm=n, km=n, turbulence=1, side=abi.BC_OUTLET)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(grid["x"], grid["y"], grid["z"], grid["wd"])
    rng = np.random.default_rng(5)
    q = state["q"].reshape(-1, 5).copy()
    q[:, 4] *= 1.0 + 0.1 * rng.normal(size=q.shape[0])
    o.set_state(q.reshape(-1), state["qn"], state["qnm1"], state["nut"])
    o.des_eddy()
    q5 = o.get_state()["q"].reshape(n, n, n, 5)[..., 4]      # [k][j][i]
    x = grid["x"].reshape(n, n, n)
    y = grid["y"].reshape(n, n, n)
    # i = im face (before the j and k faces overwrite its edges)
    r = (x[:, :, -1] - x[:, :, -2]) / (x[:, :, -2] - x[:, :, -3])
    want = (1 + r) * q5[:, :, -2] - r * q5[:, :, -3]
    assert np.allclose(q5[1:-1, 1:-1, -1], want[1:-1, 1:-1], rtol=1e-13, atol=0)
    # j = 1 and j = jm faces (before the periodic k faces)
    for jb, j1, j2 in ((0, 1, 2), (-1, -2, -3)):
        r = (y[:, jb, :] - y[:, j1, :]) / (y[:, j1, :] - y[:, j2, :])
        want = (1 + r) * q5[:, j1, :] - r * q5[:, j2, :]
        assert np.allclose(q5[1:-1, jb, :], want[1:-1], rtol=1e-13, atol=0)


def test_btype5_side_faces_keep_their_values(oracle_mod):
    n = 13
    case, grid, state = cases.wake(im=n, jm=n, km=n, turbulence=0, side=abi.BC_OUTLET)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    o.set_state(state["q"], state["qn"], state["qnm1"])
    o.begin_step()
    o.pseudo_iteration()
    a = state["q"].reshape(n, n, n, 5)
    b = o.get_state()["q"].reshape(n, n, n, 5)
    for jb in (0, -1):   # velocities (bcond_fm shifts every pressure by p(ifix, jfix, kfix))
        assert np.array_equal(b[1:-1, jb, 1:-1, 1:4], a[1:-1, jb, 1:-1, 1:4])
    # the outlet plane is solved
    assert np.abs(b[1:-1, 1:-1, -1, 1:4] - a[1:-1, 1:-1, -1, 1:4]).max() > 1e-6


def test_plane_residual_equals_interior_residual_without_i_variation(oracle_mod):
    """mg_brhs's terms are the interior residual's eta and zeta terms: on an
    affine grid with a state that does not vary along i (so every csi term of
    the interior residual vanishes, and so do the LODI terms, dq = 0), the
    outlet plane's residual equals the interior residual of any plane."""
    n = 13
    case, grid = _affine_case(n)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    rng = np.random.default_rng(8)
    q = np.zeros((n, n, n, 5))                       # [k][j][i][m]
    q[..., :4] = rng.normal(0.0, 0.3, size=(n, n, 1, 4))
    q[..., 1] += 1.0
    qn = q.copy()
    qn[..., :4] += rng.normal(0.0, 1e-2, size=(n, n, 1, 4))
    qnm1 = qn.copy()
    qnm1[..., :4] += rng.normal(0.0, 1e-2, size=(n, n, 1, 4))
    o.set_state(q.reshape(-1), qn.reshape(-1), qnm1.reshape(-1))
    plane = o.outlet_rhs()                           # (4, km, jm)
    rh = np.stack([o.get_field(1, abi.F_RH + m).reshape(n, n, n) for m in range(4)])
    assert np.abs(plane).max() > 1e-3
    for i0 in (3, n // 2, n - 2):
        interior = rh[:, 1:-1, 1:-1, i0]
        assert np.allclose(plane[:, 1:-1, 1:-1], interior, rtol=1e-10, atol=1e-12 * np.abs(interior).max())
