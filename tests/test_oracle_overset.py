"""The overset donor exchange restated on the CPU (oracle/overset_oracle.py,
mg_bintp_mom / mg_bintp_tur).  Pins: the seeded donor maps place every donee
node inside its host cell (fractions in [0, 1], hosts inside the other block),
and trilinear interpolation reproduces a field linear in x, y and z exactly on
these product grids, so every donee node receives the field's own value."""
import numpy as np

from desalm import abi, cases


def test_donor_maps_are_inside_their_host_cells():
    blocks, ov = cases.overset_pair()
    n = ov["n"]
    d = ov["donee"].reshape(n, 4)
    h = ov["host"].reshape(n, 4)
    c = ov["coef"].reshape(n, 3)
    assert n == 21 * 17 + 17 * 21
    assert ((c >= 0) & (c <= 1)).all()
    for e in range(n):
        hc = blocks[h[e, 0]][0]
        assert h[e, 0] != d[e, 0]
        assert 1 <= h[e, 1] <= hc.im - 1 and 1 <= h[e, 2] <= hc.jm - 1 and 1 <= h[e, 3] <= hc.km - 1


def test_exchange_is_exact_for_linear_fields(oracle_mod):
    import overset_oracle as oo
    blocks, ov = cases.overset_pair(turbulence=0)
    solvers = []
    for case, grid, state in blocks:
        o = oracle_mod.OracleSolver(case)
        o.set_grid(grid["x"], grid["y"], grid["z"])
        N = case.im * case.jm * case.km
        q = np.zeros((N, 5))
        for m in range(4):
            q[:, m] = 0.3 + (m + 1) * 0.7 * grid["x"] - 0.4 * grid["y"] + 0.25 * (m - 1) * grid["z"]
        o.set_state(q.reshape(-1), q.reshape(-1), q.reshape(-1), np.zeros(N))
        solvers.append(o)
    before = [[s.get_field(1, abi.F_Q + m) for m in range(4)] for s in solvers]
    oo.exchange(solvers, ov, [0, 1, 2, 3])
    n = ov["n"]
    d = ov["donee"].reshape(n, 4)
    for b, (case, grid, _) in enumerate(blocks):
        for m in range(4):
            got = solvers[b].get_field(1, abi.F_Q + m)
            want = before[b][m]
            sel = np.zeros(case.im * case.jm * case.km, bool)
            for e in np.nonzero(d[:, 0] == b)[0]:
                _, i, j, k = d[e]
                sel[(i - 1) + case.im * ((j - 1) + case.jm * (k - 1))] = True
            assert sel.sum() > 0
            assert np.allclose(got[sel], want[sel], rtol=0, atol=1e-13)   # the linear field's own values
            assert np.array_equal(got[~sel], want[~sel])                   # nothing else moves
