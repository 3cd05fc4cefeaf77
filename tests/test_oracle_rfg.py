"""Synthetic inflow turbulence on the CPU: the oracle's random flow generator
(oracle/rfg_oracle.py) against its defining properties, and the library's
host-side mode tables (desalm_rfg_modes) against the oracle, bit for bit.
No GPU needed."""
import ctypes as C

import numpy as np
import pytest

import rfg_oracle
from desalm import abi
from desalm.solver import lib, rfg_modes


def _spd(rng, scale=1.0):
    B = rng.normal(size=(3, 3))
    R = B @ B.T + 0.3 * np.eye(3)
    R *= scale / np.trace(R)
    return np.array([R[0, 0], R[0, 1], R[0, 2], R[1, 1], R[1, 2], R[2, 2]])


def test_mode_tables_match_library_bit_for_bit():
    """desalm_rfg_modes and the oracle draw the same deviates in the same
    order (initialize_rfg, src/rfg.F90:75-90)."""
    for n, seed in ((1, 0), (257, 12345), (1000, -7)):
        lib_t = rfg_modes(n, seed)
        ora_t = rfg_oracle.modes(n, seed)
        for f in ("p", "q", "k", "omega"):
            assert np.array_equal(lib_t[f], ora_t[f]), (n, seed, f)


def test_mode_tables_distribution():
    """k ~ N(0, 0.5^2), omega ~ N(0, 1), p = zeta x k and q = xi x k are
    orthogonal to k with E[p_d^2] = E[q_d^2] = 2 (0.5)^2 = 0.5 (the sample
    mean of p_d^2 over 20000 modes has a standard error of 0.008)."""
    t = rfg_oracle.modes(20000, 3)
    assert abs(t["k"].std() - 0.5) < 0.01 and abs(t["k"].mean()) < 0.01
    assert abs(t["omega"].std() - 1.0) < 0.02 and abs(t["omega"].mean()) < 0.02
    for f in ("p", "q"):
        dots = np.einsum("nd,nd->n", t[f], t["k"])
        assert np.abs(dots).max() < 1e-12
        assert np.allclose((t[f] ** 2).mean(axis=0), 0.5, atol=0.04)  # 5 standard errors


def test_decompose_signs_and_order():
    """Eigenvalues ascending; every eigenvector's largest component positive;
    a diagonal tensor gives a permutation matrix (what LAPACK returns too)."""
    M, c = rfg_oracle.decompose([3.0, 0.0, 0.0, 1.0, 0.0, 2.0])
    assert np.array_equal(M, [[0.0, 0.0, 1.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    assert np.allclose(c, np.sqrt([1.0, 2.0, 3.0]))
    M, c = rfg_oracle.decompose([0.25, 0.0, 0.0, 0.25, 0.0, 0.25])
    assert np.array_equal(M, np.eye(3)) and np.array_equal(c, [0.5, 0.5, 0.5])
    rng = np.random.default_rng(0)
    for _ in range(50):
        r = _spd(rng)
        M, c = rfg_oracle.decompose(r)
        assert np.all(np.diff(c) >= 0)
        assert np.allclose(M @ np.diag(c ** 2) @ M.T, rfg_oracle.sym(r), atol=1e-14)
        for col in range(3):
            assert M[np.argmax(np.abs(M[:, col])), col] > 0


def test_generated_velocity_reproduces_the_correlation_tensor():
    """The generator's defining property (Smirnov et al. 2001, eqs. 8-9):
    over points and times far apart, the fluctuations have zero mean and the
    covariance M diag(c) C diag(c) M^T, C = (1/N) sum (p p^T + q q^T) the
    tables' own isotropic covariance, which tends to I as N grows; hence the
    prescribed tensor r_ij."""
    rng = np.random.default_rng(1)
    tab = rfg_oracle.modes(2000, 11)
    r = _spd(rng, scale=3 * 0.05 ** 2)
    tau, eta = 0.3, 0.2
    dec = rfg_oracle.decompose(r)
    P = 4000
    xs = rng.uniform(0.0, 200.0 * eta, size=(P, 3))
    ts = rng.uniform(0.0, 200.0 * tau, size=P)
    v = np.array([rfg_oracle.rfg_vel(ts[i], xs[i], tau, eta, r, tab, dec) for i in range(P)])
    cov = np.cov(v.T, bias=True)
    M, c = dec
    Ciso = (tab["p"].T @ tab["p"] + tab["q"].T @ tab["q"]) / len(tab["omega"])
    expect = M @ np.diag(c) @ Ciso @ np.diag(c) @ M.T
    R = rfg_oracle.sym(r)
    assert np.linalg.norm(Ciso - np.eye(3)) < 0.15
    assert np.linalg.norm(cov - expect) < 0.08 * np.linalg.norm(expect)
    assert np.linalg.norm(cov - R) < 0.15 * np.linalg.norm(R)
    assert np.abs(v.mean(axis=0)).max() < 0.1 * np.sqrt(np.trace(R) / 3)


def test_inlet_forcing_touches_only_the_inflow_plane():
    """rfg_mpi_inlet_forcing writes q(2:4) of i = 1, j = 2..jm-1, k = 2..km-1
    (src/rfg_inlet.F90:121-161); nothing else changes."""
    from desalm import cases
    case, grid, state = cases.wake(im=9, jm=11, km=7, itmax=2, turbulence=0)
    spec = cases.rfg_inflow(case, nmodes=64, seed=5, tables=rfg_oracle.modes(64, 5))
    q0 = state["q"].reshape(case.km, case.jm, case.im, 5).copy()
    q1 = rfg_oracle.inlet_forcing(q0.copy(), grid, (case.im, case.jm, case.km), 0.25, spec)
    changed = q1 != q0
    assert not changed[:, :, 1:, :].any() and not changed[..., 0].any() and not changed[..., 4].any()
    assert not changed[0].any() and not changed[-1].any() and not changed[:, 0].any() and not changed[:, -1].any()
    assert changed[1:-1, 1:-1, 0, 1:4].all()


def test_rfg_entry_points_reject_bad_arguments_without_gpu():
    L = lib()
    d = C.POINTER(C.c_double)
    buf = np.zeros(30)
    p = buf.ctypes.data_as(d)
    assert L.desalm_rfg_modes(0, 1, p, p, p, p) == abi.DESALM_EINVAL
    assert L.desalm_rfg_modes((1 << 20) + 1, 1, p, p, p, p) == abi.DESALM_EINVAL
    assert L.desalm_rfg_modes(3, 1, None, p, p, p) == abi.DESALM_EINVAL
    assert L.desalm_rfg_set(None, None) == abi.DESALM_EINVAL
    assert L.desalm_rfg_inlet(None, 0.0) == abi.DESALM_EINVAL
