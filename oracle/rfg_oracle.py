"""Synthetic inflow turbulence on the CPU: the random flow generator of
Smirnov, Shi & Celik (ASME J. Fluids Eng. 123, 2001) as the reference runs it.

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the library's
desalm_rfg_* entry points; the product never loads it.

- modes() restates initialize_rfg (src/rfg.F90:42-96): the draws of zeta, xi
  (N(0, 1)), k (N(0, 0.5^2)) and omega (N(0, 1)) in its call order, then
  p = zeta x k and q = xi x k (cross_product, src/rfg.F90:115-124).  The
  normal deviates are the polar method's (the reference's box_muller,
  src/rfg.F90:126-173: the second deviate of a pair is returned first, the
  first kept for the next call) over the uniform stream the library uses
  (splitmix64), in plain Python floats, so that the tables match the
  library's desalm_rfg_modes bit for bit.  The reference's own uniform
  generator (src/rfg.F90:176-236) is not restated: its samples cannot be
  pinned without its seed file, which the reference does not ship.
- decompose() restates diagonalize (src/rfg.F90:286-313) with LAPACK's
  symmetric eigen-solver (numpy.linalg.eigh; the reference calls ssyev),
  eigenvalues ascending, then signs every eigenvector so that its component of
  largest magnitude (the first of equal ones) is positive, as the library
  does (the reference keeps LAPACK's signs).
- rfg_vel() restates rfg_vel, get_iso_velocity and anti_diagonalize
  (src/rfg.F90:238-284,315-374) in the reference's operation order.
- inlet_forcing() restates rfg_mpi_inlet_forcing (src/rfg_inlet.F90:107-173)
  on one block without MPI neighbours: nodes j = 2..jm-1, k = 2..km-1 of the
  plane i = 1.
"""
import math

import numpy as np

MASK64 = (1 << 64) - 1


class Gauss:
    """Polar-method normal deviates over a splitmix64 uniform stream."""

    def __init__(self, seed):
        self.s = seed & MASK64
        self.have = False
        self.kept = 0.0

    def uniform(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        z ^= z >> 31
        return (float(z >> 11) + 0.5) * (1.0 / 9007199254740992.0)

    def next(self, mean, stdev):
        if self.have:
            self.have = False
            g = self.kept
        else:
            while True:
                v1 = 2.0 * self.uniform() - 1.0
                v2 = 2.0 * self.uniform() - 1.0
                rsq = v1 * v1 + v2 * v2
                if not (rsq >= 1.0 or rsq == 0.0):
                    break
            fac = math.sqrt(-2.0 * math.log(rsq) / rsq)
            self.kept = v1 * fac
            self.have = True
            g = v2 * fac
        return mean + stdev * g


def _cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def modes(nmodes, seed):
    g = Gauss(seed)
    N = nmodes
    zet = np.zeros((N, 3))
    csi = np.zeros((N, 3))
    k = np.zeros((N, 3))
    for arr, sd in ((zet, 1.0), (csi, 1.0), (k, 0.5)):
        for d in range(3):
            for i in range(N):
                arr[i, d] = g.next(0.0, sd)
    omega = np.array([g.next(0.0, 1.0) for _ in range(N)])
    return dict(p=_cross(zet, k), q=_cross(csi, k), k=k, omega=omega)


def sym(r6):
    r = np.asarray(r6, dtype=np.float64)
    return np.array([[r[0], r[1], r[2]], [r[1], r[3], r[4]], [r[2], r[4], r[5]]])


def decompose(r6):
    """(M, c): M's columns the eigenvectors, c = sqrt(eigenvalues), ascending."""
    w, V = np.linalg.eigh(sym(r6))
    for col in range(3):
        big = int(np.argmax(np.abs(V[:, col])))
        if V[big, col] < 0.0:
            V[:, col] = -V[:, col]
    return V, np.sqrt(w)


def rfg_vel(t, x, tau, eta, r6, tab, dec=None):
    """Velocity fluctuation at point x (3,) and time t."""
    m, c = decompose(r6) if dec is None else dec
    t1 = t / tau
    x1 = np.asarray(x, dtype=np.float64) / eta
    upsilon = eta / tau
    k_scale = tab["k"] * upsilon / c
    term1 = k_scale @ x1 + tab["omega"] * t1
    sum1 = (tab["p"] * np.cos(term1)[:, None] + tab["q"] * np.sin(term1)[:, None]).sum(axis=0)
    const = math.sqrt(2.0 / float(len(tab["omega"])))
    v = const * sum1
    v = c * v
    return m @ v


def inlet_forcing(q, grid, dims, time, spec):
    """q: the state, shape (km, jm, im, 5) (Fortran q(1:5, i, j, k)), changed
    in place; grid: x, y, z flat arrays; spec: the desalm_rfg tables with um
    (km, jm, 3), uij (km, jm, 6), t_ts and t_ls (km, jm)."""
    im, jm, km = dims
    X = grid["x"].reshape(km, jm, im)
    Y = grid["y"].reshape(km, jm, im)
    Z = grid["z"].reshape(km, jm, im)
    tab = dict(p=np.asarray(spec["p"]).reshape(-1, 3), q=np.asarray(spec["q"]).reshape(-1, 3),
               k=np.asarray(spec["k"]).reshape(-1, 3), omega=np.asarray(spec["omega"]).reshape(-1))
    um = np.asarray(spec["um"]).reshape(km, jm, 3)
    uij = np.asarray(spec["uij"]).reshape(km, jm, 6)
    ts = np.asarray(spec["t_ts"]).reshape(km, jm)
    ls = np.asarray(spec["t_ls"]).reshape(km, jm)
    for k in range(1, km - 1):
        for j in range(1, jm - 1):
            x = (X[k, j, 0], Y[k, j, 0], Z[k, j, 0])
            v = rfg_vel(time, x, ts[k, j], ls[k, j], uij[k, j], tab)
            q[k, j, 0, 1:4] = um[k, j] + v
    return q
