"""Known-answer checks that pin the CPU oracle without reference output.
The check_* functions take the solver class, so that the same identities run
on the GPU path too (tests/test_gpu_identities.py).

The reference ships no tests or golden data, so the restatement is pinned by
mathematical identities of the routines it restates:
  * SGTSV restatement == dense solve (with and without row interchanges)
  * Ma^-1 Ma = I, Mb^-1 Mb = I, Mc^-1 Mc = I; N1^-1 = Mb^-1 Ma, N2^-1 = Mc^-1 Mb
  * the 27-point restriction weights sum to one (16/16)
  * metrics of an affine map are exact
  * a uniform flow on a Cartesian grid has zero residual (free stream)
  * a linear velocity field on an affine grid has the exact convective and
    divergence residual (QUICK and the central differences are exact on it)
  * so does a quadratic one, with the full-stress viscous term
  * on a coarse level the convection is first-order upwind, whose error on a
    quadratic field is known exactly
  * the BDF2 time derivative of a flow uniform in space
  * the SA eddy viscosity nu_t = nu_tilde f_v1 and the nu_tilde floor
  * the convergence norm of mg_residual over the interior nodes
  * the local pseudo-time step of rhs_daf_dtau on a curvilinear grid
  * bcond_fm's extrapolation, wall and symmetry rows and the pressure fix
  * prolongation of a linear coarse correction is exact on interior nodes
  * the FP32 mirror stays within FP32 round-off of the FP64 oracle
"""
import numpy as np
import pytest

from conftest import rel_l2
from desalm import abi, cases


def test_gtsv_matches_dense_no_pivot(oracle_mod):
    rng = np.random.default_rng(0)
    n = 40
    dl = rng.uniform(-1, 1, n - 1)
    du = rng.uniform(-1, 1, n - 1)
    d = 3.0 + rng.uniform(0, 1, n)
    b = rng.normal(size=n)
    x, info, piv = oracle_mod.gtsv(dl, d, du, b)
    A = np.diag(d) + np.diag(dl, -1) + np.diag(du, 1)
    assert info == 0 and piv == 0
    assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-13, atol=1e-13)


def test_gtsv_matches_dense_with_pivots(oracle_mod):
    rng = np.random.default_rng(1)
    n = 33
    dl = rng.uniform(-3, 3, n - 1)
    du = rng.uniform(-3, 3, n - 1)
    d = rng.uniform(-0.5, 0.5, n)
    b = rng.normal(size=(4, n))
    x, info, piv = oracle_mod.gtsv(dl, d, du, b)
    A = np.diag(d) + np.diag(dl, -1) + np.diag(du, 1)
    assert info == 0 and piv > 0
    for r in range(4):
        assert rel_l2(x[r], np.linalg.solve(A, b[r])) < 1e-10


def test_gtsv_zero_pivot_reports_info(oracle_mod):
    d = np.array([0.0, 1.0, 1.0])
    x, info, _ = oracle_mod.gtsv(np.zeros(2), d, np.zeros(2), np.ones(3))
    assert info == 1


def test_modal_inverses(oracle_mod):
    rng = np.random.default_rng(2)
    for _ in range(50):
        csi, eta, zet = rng.normal(size=3), rng.normal(size=3), rng.normal(size=3)
        sigma = rng.uniform(0.5, 2.0)
        mai, n1i, n2i, mc, ma, mb, mci = oracle_mod.modal(csi, eta, zet, sigma)
        I = np.eye(4)
        assert np.allclose(mai @ ma, I, atol=1e-12)
        assert np.allclose(mci @ mc, I, atol=1e-12)
        mbi = n1i @ np.linalg.inv(ma)
        assert np.allclose(mbi @ mb, I, atol=1e-10)
        assert np.allclose(n2i, mci @ mb, atol=1e-13)


def test_restriction_weights_sum_to_one(oracle_mod):
    case, grid, state = cases.cavity(n=17, seed=0)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    o.set_state(state["q"])
    N = 17 ** 3
    one = np.ones(N).reshape(17, 17, 17)
    one[0], one[-1], one[:, 0], one[:, -1], one[:, :, 0], one[:, :, -1] = (0.0,) * 6
    for m in range(4):
        o.set_field(1, abi.F_RH + m, np.ones(N))
    o.mg_nlevel(2)
    pk = o.get_field(2, abi.F_PK).reshape(9, 9, 9)
    assert np.allclose(pk[1:-1, 1:-1, 1:-1], 1.0, rtol=0, atol=1e-15)
    assert np.all(pk[0] == 0) and np.all(pk[:, :, -1] == 0)


def _cartesian(n, h=None):
    case, _, _ = cases.cavity(n=n, seed=0)
    s = np.linspace(0.0, 1.0, n)
    X = np.broadcast_to(s[None, None, :], (n, n, n))
    Y = np.broadcast_to(s[None, :, None], (n, n, n))
    Z = np.broadcast_to(s[:, None, None], (n, n, n))
    return case, X, Y, Z


def test_affine_metrics_exact(oracle_mod):
    n = 17
    case, X, Y, Z = _cartesian(n)
    A = np.array([[2.0, 0.3, 0.1], [0.2, 1.5, -0.4], [0.0, 0.25, 3.0]])
    P = np.stack([X, Y, Z], -1) @ A.T
    o = oracle_mod.OracleSolver(case)
    o.set_grid(P[..., 0].reshape(-1), P[..., 1].reshape(-1), P[..., 2].reshape(-1))
    h = 1.0 / (n - 1)
    J = np.linalg.inv(A * h)           # d(xi)/d(x) per unit index
    for d, f in enumerate((abi.F_CSI, abi.F_ETA, abi.F_ZET)):
        for c in range(3):
            v = o.get_field(1, f + c)
            assert np.allclose(v, J[d, c], rtol=1e-12, atol=1e-12)
    aj = o.get_field(1, abi.F_AJ)
    assert np.allclose(aj, 1.0 / np.linalg.det(A * h), rtol=1e-12)


def check_uniform_flow_has_zero_residual(make):
    n = 17
    case, X, Y, Z = _cartesian(n)
    for b in range(6):
        case.btype[b] = abi.BC_FREESTREAM   # first-order extrapolation keeps a uniform field
    o = make(case)
    o.set_grid(X.reshape(-1), Y.reshape(-1), Z.reshape(-1))
    q = np.zeros((n ** 3, 5))
    q[:, 1], q[:, 2], q[:, 3] = 0.7, -0.2, 0.4
    q[:, 0] = 0.1
    o.set_state(q.reshape(-1), q.reshape(-1), q.reshape(-1))
    o.solver_daf(1, 1, 1)
    for m in range(4):
        assert np.max(np.abs(o.get_field(1, abi.F_RH + m))) < 1e-12
    qq = o.get_state()["q"].reshape(-1, 5)
    assert np.allclose(qq[:, 1:4], q[:, 1:4], atol=1e-12)


def test_uniform_flow_has_zero_residual(oracle_mod):
    check_uniform_flow_has_zero_residual(oracle_mod.OracleSolver)


def check_linear_velocity_residual_is_exact(make):
    """On an affine grid (constant metrics) a linear velocity field u = u0 + G x
    with uniform pressure and q = q^n = q^{n-1} has the residual
      rh(1)   = (div u) / J                     (rhs_flux_sans_convec: central
                                                 differences of U/J,
                                                 src/rhs_flux_sans_convec.F90:124-133)
      rh(m+1) = (u . grad) u_m / J, m = 1..3    (rhs_convec_quick: QUICK,
                                                 (3, 3, -7, 1)/8 with the
                                                 U+/U- split, adds +fv,
                                                 src/rhs_convec_quick.F90:90-198)
    exactly: QUICK and the central differences reproduce the index derivative
    of a linear field, the viscous terms and the pressure terms vanish, and so
    do the BDF2 terms.  cfl1 = vnn1 = 0 makes dtau = 0, so the DAF update is
    zero and the recalculated residual is that of the field as set.  Checked
    on nodes 4..n-3, whose stencils do not reach the boundary nodes that
    bcond_fm rewrites."""
    n = 17
    case, X, Y, Z = _cartesian(n)
    case.cfl1 = case.vnn1 = 0.0
    A = np.array([[2.0, 0.3, 0.1], [0.2, 1.5, -0.4], [0.0, 0.25, 3.0]])
    P = np.stack([X, Y, Z], -1) @ A.T
    o = make(case)
    o.set_grid(P[..., 0].reshape(-1), P[..., 1].reshape(-1), P[..., 2].reshape(-1))
    G = np.array([[0.3, -0.2, 0.1], [0.15, 0.05, -0.25], [-0.1, 0.2, 0.12]])
    centre = A @ np.full(3, 0.5)
    u0 = np.array([0.05, -0.03, 0.02]) - G @ centre
    U = u0 + P @ G.T                              # (n, n, n, 3): every component changes sign
    inner = (slice(3, n - 3),) * 3                # inside the checked nodes (both QUICK branches)
    assert all((U[inner][..., c] > 0).any() and (U[inner][..., c] < 0).any() for c in range(3))
    q = np.zeros((n, n, n, 5))
    q[..., 0] = 0.1
    q[..., 1:4] = U
    o.set_state(q.reshape(-1), q.reshape(-1), q.reshape(-1))
    o.solver_daf(1, 1, 1)
    aj = o.get_field(1, abi.F_AJ).reshape(n, n, n)
    want = [np.trace(G) / aj] + [np.einsum("kjic,c->kji", U, G[m]) / aj for m in range(3)]
    for m in range(4):
        got = o.get_field(1, abi.F_RH + m).reshape(n, n, n)
        scale = np.abs(want[m][inner]).max()
        assert np.abs(got[inner] - want[m][inner]).max() <= 1e-12 * scale, m
    assert np.array_equal(o.get_state()["q"].reshape(n, n, n, 5)[inner][..., 1:4], U[inner])


def test_linear_velocity_residual_is_exact(oracle_mod):
    check_linear_velocity_residual_is_exact(oracle_mod.OracleSolver)


def check_quadratic_velocity_residual_is_exact(make):
    """QUICK is exact up to quadratics ((3, 3, -7, 1)/8 of i^2 is 2i), and so
    are the central and face differences of the viscous and pressure terms.
    On an affine grid quadratic velocity and pressure fields therefore have
      rh(1)   = (div u) / J
      rh(m+1) = [(u . grad) u_m + d_m p - nu (lap u_m + d_m div u)] / J,
    the viscous term in the full-stress form nu div(grad u + grad u^T) that
    rhs_viscous's face fluxes build (the a . (du/dx) terms beside the
    c11, c12, c13 ones, src/rhs_viscous.F90:126-162).  A Laplacian-only
    viscous term would miss by nu d_m div u / J, 1.4e-5 to 2.1e-4 here, against
    a tolerance of 1e-12 of each field's largest value.  Same set-up as the
    linear case (dtau = 0, which also zeroes the pressure dissipation
    diss(1); nodes 4..n-3)."""
    n = 17
    case, X, Y, Z = _cartesian(n)
    case.cfl1 = case.vnn1 = 0.0
    case.ren = 10.0
    A = np.array([[2.0, 0.3, 0.1], [0.2, 1.5, -0.4], [0.0, 0.25, 3.0]])
    P = np.stack([X, Y, Z], -1) @ A.T
    o = make(case)
    o.set_grid(P[..., 0].reshape(-1), P[..., 1].reshape(-1), P[..., 2].reshape(-1))
    rng = np.random.default_rng(3)
    G = rng.normal(0.0, 0.2, (3, 3))
    H = rng.normal(0.0, 0.1, (3, 3, 3))
    H = 0.5 * (H + H.transpose(0, 2, 1))       # u_m = ... + sum_ab H[m, a, b] D_a D_b
    D = P - A @ np.full(3, 0.5)
    U = np.array([0.05, -0.03, 0.02]) + D @ G.T + np.einsum("mab,...a,...b->...m", H, D, D)
    gp = np.array([0.2, -0.1, 0.05])
    Kp = np.array([[0.1, 0.02, -0.03], [0.02, -0.05, 0.01], [-0.03, 0.01, 0.08]])
    q = np.zeros((n, n, n, 5))
    q[..., 0] = 0.1 + D @ gp + np.einsum("ab,...a,...b->...", Kp, D, D)
    q[..., 1:4] = U
    o.set_state(q.reshape(-1), q.reshape(-1), q.reshape(-1))
    o.solver_daf(1, 1, 1)
    aj = o.get_field(1, abi.F_AJ).reshape(n, n, n)
    dp = gp + 2.0 * D @ Kp                                      # dp / dx_m (rhs_flux_sans_convec)
    grad = G + 2.0 * np.einsum("mcb,...b->...mc", H, D)          # du_m / dx_c
    div = np.einsum("...mm->...", grad)
    conv = np.einsum("...c,...mc->...m", U, grad)
    lap = 2.0 * np.einsum("mcc->m", H)
    graddiv = 2.0 * np.einsum("ccm->m", H)
    nu = 1.0 / case.ren
    inner = (slice(3, n - 3),) * 3
    want = [div / aj] + [(conv[..., m] + dp[..., m] - nu * (lap[m] + graddiv[m])) / aj for m in range(3)]
    assert np.abs(nu * graddiv).max() > 1e-6
    for m in range(4):
        got = o.get_field(1, abi.F_RH + m).reshape(n, n, n)
        scale = np.abs(want[m][inner]).max()
        assert np.abs(got[inner] - want[m][inner]).max() <= 1e-12 * scale, m


def test_quadratic_velocity_residual_is_exact(oracle_mod):
    check_quadratic_velocity_residual_is_exact(oracle_mod.OracleSolver)


def check_sa_eddy_viscosity_closure(make):
    """With a zero turbulence time step (cfl2 = vnn2 = 0: dtev = 0), des_eddy
    changes no interior nu_tilde except by the floor, and leaves
      nu_t = nu_tilde f_v1,  f_v1 = chi^3 / (chi^3 + 357.911),
      chi = nu_tilde Re,  nu_tilde >= 1e-7
    on every interior node (rhs_sa_bcond, src/rhs_sa_bcond.F90:282-286; cv1^3
    from src/des_eddy.F90:72).  nu_tilde spans 1e-9..1e-1, across the floor
    and the range where f_v1 turns from chi^3 / cv1^3 to one."""
    case, grid, state = cases.channel(im=17, jm=17, km=17, seed=0, itmax=2)
    case.cfl2 = case.vnn2 = 0.0
    o = make(case)
    o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    q = state["q"].reshape(-1, 5).copy()
    nt = 10.0 ** np.random.default_rng(0).uniform(-9.0, -1.0, size=q.shape[0])
    q[:, 4] = nt
    o.set_state(q.reshape(-1), q.reshape(-1), q.reshape(-1), state["nut"])
    o.des_eddy()
    inner = np.zeros((17, 17, 17), bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.reshape(-1)
    floor = np.maximum(1e-7, nt)[inner]
    assert (nt[inner] < 1e-7).any()
    q5 = o.get_state()["q"].reshape(-1, 5)[inner, 4]
    assert np.array_equal(q5, floor)
    chi3 = (floor * case.ren) ** 3
    want = floor * (chi3 / (chi3 + 357.911))
    nut = o.get_field(1, abi.F_NUT)[inner]
    assert np.abs(nut - want).max() <= 1e-14 * np.abs(want).max()


def test_sa_eddy_viscosity_closure(oracle_mod):
    check_sa_eddy_viscosity_closure(oracle_mod.OracleSolver)


def check_coarse_levels_convect_first_order_upwind(make):
    """On coarse levels the convection is first-order upwind
    (decide_upwind = 1, src/rhs_convec_quick.F90:90-161): for a quadratic
    field its error is exactly -1/2 dxi |U/J| times the second difference
    along each direction, so the level-2 residual of the quadratic case equals
      [(u . grad) u_m - nu (lap u_m + d_m div u)] / J
        - sum_d 1/2 dxi_d |U_d / J| (q_{I+1} - 2 q_I + q_{I-1})_d,
    with dxi = 1/2 there.  The FAS forcing pk is zero and itr = 2, so rhs_pk
    only adds it (src/rhs_pk.F90:35-67)."""
    n, nc = 17, 9
    case, X, Y, Z = _cartesian(n)
    case.cfl1 = case.vnn1 = 0.0
    case.ren = 10.0
    A = np.array([[2.0, 0.3, 0.1], [0.2, 1.5, -0.4], [0.0, 0.25, 3.0]])
    P = np.stack([X, Y, Z], -1) @ A.T
    o = make(case)
    o.set_grid(P[..., 0].reshape(-1), P[..., 1].reshape(-1), P[..., 2].reshape(-1))
    rng = np.random.default_rng(3)
    G = rng.normal(0.0, 0.2, (3, 3))
    H = rng.normal(0.0, 0.1, (3, 3, 3))
    H = 0.5 * (H + H.transpose(0, 2, 1))
    D = P[::2, ::2, ::2] - A @ np.full(3, 0.5)     # the coarse nodes (injection)
    U = np.array([0.05, -0.03, 0.02]) + D @ G.T + np.einsum("mab,...a,...b->...m", H, D, D)
    qc = np.zeros((nc, nc, nc, 5))
    qc[..., 0] = 0.1
    qc[..., 1:4] = U
    for m in range(5):
        for f in (abi.F_Q, abi.F_QN, abi.F_QNM1, abi.F_QOLD):
            o.set_field(2, f + m, qc[..., m].reshape(-1))
    for m in range(4):
        o.set_field(2, abi.F_PK + m, np.zeros(nc ** 3))
    o.solver_daf(2, 1, 2)
    aj = o.get_field(2, abi.F_AJ).reshape(nc, nc, nc)
    met = [np.stack([o.get_field(2, f + c).reshape(nc, nc, nc) for c in range(3)], -1)
           for f in (abi.F_CSI, abi.F_ETA, abi.F_ZET)]
    grad = G + 2.0 * np.einsum("mcb,...b->...mc", H, D)
    div = np.einsum("...mm->...", grad)
    conv = np.einsum("...c,...mc->...m", U, grad)
    lap = 2.0 * np.einsum("mcc->m", H)
    graddiv = 2.0 * np.einsum("ccm->m", H)
    nu, dxi = 1.0 / case.ren, 0.5
    inner = (slice(2, nc - 2),) * 3
    got = o.get_field(2, abi.F_RH).reshape(nc, nc, nc)
    assert np.abs(got - div / aj)[inner].max() <= 1e-12 * np.abs(div / aj)[inner].max()
    for m in range(3):
        want = (conv[..., m] - nu * (lap[m] + graddiv[m])) / aj
        for d, ax in enumerate((2, 1, 0)):            # xi along i (last axis), eta along j, zeta along k
            Ud = np.einsum("...c,...c->...", met[d], U) / aj
            q = U[..., m]
            want = want - 0.5 * dxi * np.abs(Ud) * (np.roll(q, -1, ax) - 2.0 * q + np.roll(q, 1, ax))
        got = o.get_field(2, abi.F_RH + 1 + m).reshape(nc, nc, nc)
        assert np.abs(got - want)[inner].max() <= 1e-12 * np.abs(want[inner]).max(), m


def test_coarse_levels_convect_first_order_upwind(oracle_mod):
    check_coarse_levels_convect_first_order_upwind(oracle_mod.OracleSolver)


def check_bdf2_term_of_a_uniform_accelerating_flow(make):
    """A flow uniform in space that changes linearly in time, q^{n-1} = a - 2 b dt,
    q^n = a - b dt, q = a: every spatial term vanishes and the residual is the
    BDF2 time derivative (3 q - 4 q^n + q^{n-1}) / (2 dt J) = b / J
    (rhs_unst_visc_diss, src/rhs_unst_visc_diss.F90:35-50, e_source = 1),
    which pins its coefficients, sign and scale; rh(1) = 0."""
    n = 17
    case, X, Y, Z = _cartesian(n)
    case.cfl1 = case.vnn1 = 0.0
    for b in range(6):
        case.btype[b] = abi.BC_FREESTREAM   # the extrapolation keeps a uniform field uniform
    A = np.array([[2.0, 0.3, 0.1], [0.2, 1.5, -0.4], [0.0, 0.25, 3.0]])
    P = np.stack([X, Y, Z], -1) @ A.T
    o = make(case)
    o.set_grid(P[..., 0].reshape(-1), P[..., 1].reshape(-1), P[..., 2].reshape(-1))
    a_ = np.array([0.1, 0.7, -0.2, 0.4, 0.0])
    b_ = np.array([0.0, 0.3, 0.5, -0.25, 0.0])
    dt = case.delti
    Q = lambda v: np.broadcast_to(v, (n ** 3, 5)).reshape(-1).copy()
    o.set_state(Q(a_), Q(a_ - b_ * dt), Q(a_ - 2.0 * b_ * dt))
    o.solver_daf(1, 1, 1)
    aj = o.get_field(1, abi.F_AJ).reshape(n, n, n)
    inner = (slice(1, n - 1),) * 3
    assert np.abs(o.get_field(1, abi.F_RH).reshape(n, n, n)[inner]).max() < 1e-12
    for m in range(1, 4):
        got = o.get_field(1, abi.F_RH + m).reshape(n, n, n)[inner]
        want = b_[m] / aj[inner]
        assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max(), m


def test_bdf2_term_of_a_uniform_accelerating_flow(oracle_mod):
    check_bdf2_term_of_a_uniform_accelerating_flow(oracle_mod.OracleSolver)


def check_boundary_extrapolation_and_walls(make):
    """bcond_fm (src/bcond_fm.F90:80-310) with the coefficients of
    src/init.F90:482-509 on the face nodes away from edges: an extrapolating
    face (btype 3) sets q_b = 4/3 q_1 - 1/3 q_2 (a zero normal derivative to
    second order: exact for a quadratic with zero slope at the face), a wall
    (btype 1) sets u = v = w = 0 and extrapolates p, a symmetry plane (btype 2)
    zeroes its bdir component only; then p(ifix, jfix, kfix) is subtracted
    from p everywhere (src/bcond_fm.F90:316-322)."""
    n = 17
    case, X, Y, Z = _cartesian(n)
    bt = [abi.BC_FREESTREAM, abi.BC_WALL, abi.BC_SYMMETRY, abi.BC_FREESTREAM, abi.BC_WALL, abi.BC_SYMMETRY]
    for b in range(6):
        case.btype[b] = bt[b]
    case.ifix, case.jfix, case.kfix = 5, 6, 7
    o = make(case)
    o.set_grid(X.reshape(-1), Y.reshape(-1), Z.reshape(-1))
    q = np.random.default_rng(6).normal(size=(n, n, n, 5))
    o.set_state(q.reshape(-1))
    o.bcond_fm()
    got = o.get_state()["q"].reshape(n, n, n, 5)
    pfix = q[case.kfix - 1, case.jfix - 1, case.ifix - 1, 0]
    mid = slice(1, n - 1)
    # faces in the reference's order: i = 1, i = im, j = 1, j = jm, k = 1, k = km
    faces = [lambda a: a[mid, mid, 0], lambda a: a[mid, mid, -1], lambda a: a[mid, 0, mid],
             lambda a: a[mid, -1, mid], lambda a: a[0, mid, mid], lambda a: a[-1, mid, mid]]
    inner1 = [lambda a: a[mid, mid, 1], lambda a: a[mid, mid, -2], lambda a: a[mid, 1, mid],
              lambda a: a[mid, -2, mid], lambda a: a[1, mid, mid], lambda a: a[-2, mid, mid]]
    inner2 = [lambda a: a[mid, mid, 2], lambda a: a[mid, mid, -3], lambda a: a[mid, 2, mid],
              lambda a: a[mid, -3, mid], lambda a: a[2, mid, mid], lambda a: a[-3, mid, mid]]
    for b in range(6):
        g, q1, q2 = faces[b](got), inner1[b](q), inner2[b](q)
        ext = 4.0 / 3.0 * q1 - 1.0 / 3.0 * q2
        assert np.allclose(g[..., 0], ext[..., 0] - pfix, rtol=0, atol=1e-14), b
        for m in (1, 2, 3):
            if bt[b] == abi.BC_WALL or (bt[b] == abi.BC_SYMMETRY and case.bdir[b] == m):
                want = np.zeros_like(ext[..., m])
            else:
                want = ext[..., m]
            assert np.allclose(g[..., m], want, rtol=0, atol=1e-14), (b, m)
    assert np.allclose(got[1:-1, 1:-1, 1:-1, 0], q[1:-1, 1:-1, 1:-1, 0] - pfix, rtol=0, atol=1e-15)


def test_boundary_extrapolation_and_walls(oracle_mod):
    check_boundary_extrapolation_and_walls(oracle_mod.OracleSolver)


def check_local_pseudo_time_step(make):
    """rhs_daf_dtau (src/rhs_daf_dtau.F90:30-84) on a curvilinear grid with an
    eddy viscosity: per node, with g_d = |grad xi_d|^2,
      dtau = min_d min( cfl1 / sqrt(g_d) / dxi_d,
                        vnn1 / (1/Re + nu_t) / dxi_d^2 / g_d ),
    the convective and viscous limits of the three directions."""
    case, grid, state = cases.channel(im=17, jm=17, km=17, seed=1, itmax=2)
    o = make(case)
    o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
    o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
    o.solver_daf(1, 0, 1)
    nut = o.get_field(1, abi.F_NUT)
    assert np.ptp(nut) > 0
    ret = 1.0 / case.ren + nut
    lim = []
    for f in (abi.F_CSI, abi.F_ETA, abi.F_ZET):     # dc = de = dz = 1 on the fine level
        g = sum(o.get_field(1, f + c) ** 2 for c in range(3))
        lim += [case.cfl1 / np.sqrt(g), case.vnn1 / ret / g]
    want = np.minimum.reduce(lim)
    got = o.get_field(1, abi.F_DTAU)
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()
    assert len(set(np.argmin(np.stack(lim), axis=0).tolist())) > 1   # more than one limit is active


def test_local_pseudo_time_step(oracle_mod):
    check_local_pseudo_time_step(oracle_mod.OracleSolver)


def check_residual_norm_definition(make):
    """mg_residual (src/mg_residual.F90:32-84): per field, log10 of the sum of
    |q - qold_mg| over the interior nodes divided by (im-2)(jm-2)(km-2);
    boundary nodes do not count."""
    case, grid, state = cases.cavity(n=17, seed=4)
    o = make(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    rng = np.random.default_rng(5)
    N = 17 ** 3
    q = rng.normal(size=(N, 5))
    qold = rng.normal(size=(N, 5))
    o.set_state(q.reshape(-1))
    for m in range(5):
        o.set_field(1, abi.F_QOLD + m, qold[:, m])
    got = o.mg_residual(1)
    d = np.abs(q - qold).reshape(17, 17, 17, 5)[1:-1, 1:-1, 1:-1]
    want = np.log10(d.reshape(-1, 5).sum(axis=0) / 15 ** 3)
    assert np.allclose(got, want, rtol=0, atol=1e-13)


def test_residual_norm_definition(oracle_mod):
    check_residual_norm_definition(oracle_mod.OracleSolver)


def check_prolongation_of_linear_correction_is_exact(make):
    case, grid, state = cases.cavity(n=17, seed=1)
    case.ep[1][0] = case.ep[1][1] = case.ep[1][2] = 0.0   # no smoothing: pure interpolation
    o = make(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    o.set_state(state["q"])
    c = np.arange(9, dtype=float)
    K, J, I = np.meshgrid(c, c, c, indexing="ij")
    lin = 0.01 * (1.0 + 2.0 * I - 0.5 * J + 0.25 * K)
    q0 = o.get_field(1, abi.F_Q + 1)
    for m in range(4):
        o.set_field(2, abi.F_QOLD + m, np.zeros(9 ** 3))
        o.set_field(2, abi.F_Q + m, lin.reshape(-1))
    o.mg_prolong(1)
    f = np.arange(17, dtype=float) / 2.0
    Kf, Jf, If = np.meshgrid(f, f, f, indexing="ij")
    want = 0.01 * (1.0 + 2.0 * If - 0.5 * Jf + 0.25 * Kf)
    got = (o.get_field(1, abi.F_Q + 1) - q0).reshape(17, 17, 17)
    assert np.allclose(got[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1], atol=1e-15)
    assert np.all(got[0] == 0)


def test_prolongation_of_linear_correction_is_exact(oracle_mod):
    check_prolongation_of_linear_correction_is_exact(oracle_mod.OracleSolver)


def test_fp32_mirror_tracks_fp64(oracle_mod):
    case, grid, state = cases.cavity(n=17, seed=2)
    a = oracle_mod.OracleSolver(case, 8)
    b = oracle_mod.OracleSolver(case, 4)
    for s in (a, b):
        s.set_grid(grid["x"], grid["y"], grid["z"])
        s.set_state(state["q"], state["qn"], state["qnm1"])
        s.begin_step()
        for _ in range(3):
            s.pseudo_iteration()
    for m in range(4):
        e = rel_l2(b.get_field(1, abi.F_Q + m), a.get_field(1, abi.F_Q + m))
        assert e < 1e-4, (m, e)


def test_oracle_cavity_converges(oracle_mod):
    case, grid, state = cases.cavity(n=17, seed=3, itmax=30)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(grid["x"], grid["y"], grid["z"])
    o.set_state(state["q"], state["qn"], state["qnm1"])
    o.begin_step()
    r0 = np.array(o.pseudo_iteration()["residual"])
    for _ in range(20):
        r = np.array(o.pseudo_iteration()["residual"])
    assert max(r[1:4] - r0[1:4]) < -0.3
