"""Known answer for the oracle's actuator-line projection (rhs_lines,
src/rhs_lines.F90:382-448) on the CPU.

The reference spreads each element's force with the 3D Gaussian
exp(-r^2 / eps^2) / (eps^3 pi^(3/2)), eps = 2 dV^(1/3), which integrates to
one.  On a uniform grid of spacing h (eps = 2h) whose kernel nodes reach four
eps past every element, the grid sum of the Gaussian times dV is one to
rounding (the sampled Gaussian's aliasing error is about exp(-4 pi^2) and its
truncation erfc(4)), so the force field, times J dV and summed over the
kernel nodes, must give back the elements' forces times the element length
and the nondimensional scale ls / (rho V^2) (:433-446).
"""
import numpy as np

from desalm import abi, cases


def test_projection_conserves_the_element_forces(oracle_mod):
    n, h = 41, 0.1
    case, _, _ = cases.wake(im=n, jm=n, km=n, turbulence=0)
    s = h * np.arange(n)
    X, Y, Z = cases._mesh(s, s, s)
    # rotor centre off the grid lines, so that no kernel node sits on the axis
    tur, polars = cases.alm_rotor(s, s, s, (2.0, 2.03, 1.97), 0.8, hub_frac=0.0, ker_cells=8, seed=3)
    spec = dict(turbines=[tur], polars=polars, vel_infty=0.1, length_scale=1.0)
    o = oracle_mod.OracleSolver(case)
    o.set_grid(X.reshape(-1), Y.reshape(-1), Z.reshape(-1))
    rng = np.random.default_rng(2)
    q = np.zeros((n ** 3, 5))
    q[:, 1] = 1.0 + 0.05 * rng.normal(size=n ** 3)
    q[:, 2:4] = 0.05 * rng.normal(size=(n ** 3, 2))
    o.set_state(q.reshape(-1), q.reshape(-1), q.reshape(-1))
    o.alm_set(spec)
    o.solver_daf(1, 0, 1)
    F = o.alm_get(abi.ALM_FORCES)                  # (elements, 6): x, y, z, fx, fy, fz
    field = o.alm_get(abi.ALM_FIELD)               # (3, N)
    aj = o.get_field(1, abi.F_AJ)
    I, J, K = tur["ker_index"].T
    l = (I - 1) + n * ((J - 1) + n * (K - 1))
    dV = tur["ker_dat"][:, 3]
    got = (field[:, l] * aj[l] * dV).sum(axis=1)
    rho, ls = 1178.62, 1.0
    vel = case.ren * 1e-6 / ls
    deltar = abs(tur["tur_rad"] - tur["hub_rad"]) / tur["nelems"]
    want = F[:, 3:6].sum(axis=0) * deltar * ls / (rho * vel * vel)
    assert np.abs(want).max() > 0
    assert np.allclose(got, want, rtol=1e-6, atol=1e-6 * np.abs(want).max()), (got, want)
