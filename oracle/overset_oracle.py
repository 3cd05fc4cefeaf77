"""Overset blocks on the CPU oracle: the donor exchange and the multi-zone
physical step, and one rank's exchange of a sharded run (DistExchange).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the library's
desalm_overset_* entry points; the product never loads it.

exchange() restates mg_bintp_mom (src/mg_bintp_mom.F90:60-160) and
mg_bintp_tur (src/mg_bintp_tur.F90): every donee value is the trilinear
interpolation of its host cell's eight corners, with the weights and in the
summation order of the reference, all values gathered before any is written
(the reference fills its send buffer, then mpi_alltoallv, then writes).
mg_driver() runs the reference's mg_driver loop (src/mg_driver.F90:42-316)
over several OracleSolver blocks through their fine-grained entry points,
exchanging after each fine-level turbulence update and DAF step
(src/mg_driver.F90:164-183,237-244), with the convergence norm summed over
every block and divided by block 0's interior count (src/mg_residual.F90:
31,64-80).
"""
import numpy as np

from desalm import abi

TURB_FIELDS = {0: [], 1: [4], 2: [4, "omega"]}


def _weights(c):
    x, y, z = c[:, 0], c[:, 1], c[:, 2]
    one = 1.0
    return [(one - x) * (one - y) * (one - z), x * (one - y) * (one - z), (one - x) * y * (one - z),
            (one - x) * (one - y) * z, x * (one - y) * z, (one - x) * y * z, x * y * (one - z), x * y * z]


def _get(block, f):
    if f == "omega":
        return block.get_omega()["omega"]
    return block.get_field(1, abi.F_Q + f)


def _set(block, f, v):
    if f == "omega":
        om = block.get_omega()
        block.set_omega(v, om["omega_n"], om["omega_nm1"])
    else:
        block.set_field(1, abi.F_Q + f, v)


def exchange(blocks, ov, fields):
    """Donor exchange of the given fields (q indices 0..4, or "omega")."""
    n = int(ov["n"])
    if n == 0 or not fields:
        return
    d = np.asarray(ov["donee"]).reshape(n, 4)
    h = np.asarray(ov["host"]).reshape(n, 4)
    c = np.asarray(ov["coef"], np.float64).reshape(n, 3)
    w = _weights(c)
    dims = [(b.case.im, b.case.jm, b.case.km) for b in blocks]
    # corner offsets in the reference's order: 000 100 010 001 101 011 110 111
    offs = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 0), (1, 1, 1)]
    vals = {}
    for f in fields:
        data = [_get(b, f) for b in blocks]
        out = np.zeros(n)
        for e in range(n):
            hb, ih, jh, kh = h[e]
            im, jm, km = dims[hb]
            v = data[hb]
            acc = 0.0
            for t, (a, bb, cc) in enumerate(offs):
                acc = acc + v[(ih - 1 + a) + im * ((jh - 1 + bb) + jm * (kh - 1 + cc))] * w[t][e]
            out[e] = acc
        vals[f] = out
    for f in fields:
        data = [_get(b, f) for b in blocks]
        for e in range(n):
            db, i, j, k = d[e]
            im, jm, km = dims[db]
            data[db][(i - 1) + im * ((j - 1) + jm * (k - 1))] = vals[f][e]
        for b, blk in enumerate(blocks):
            _set(blk, f, data[b])


def mg_driver(blocks, ov):
    """One physical step of every block in lockstep; returns the combined
    report (iterations, converged, residual, init_residual)."""
    c = blocks[0].case
    turb = TURB_FIELDS[c.turbulence]
    for b in blocks:
        b.begin_step()
    ng = c.ng
    tnu0 = (c.im - 2) * (c.jm - 2) * (c.km - 2)
    init = None
    itc = 0
    conv = False
    res = None
    while not conv and itc < c.itmax:
        itc += 1
        recalc = 0
        for b in blocks:
            b.save_qold()
        for n in range(ng):
            if n > 0:
                for b in blocks:
                    b.mg_nlevel(n + 1)
            for itr in range(1, c.iter[n] + 1):
                if n != ng - 1:
                    recalc = 0 if itr != c.iter[n] else 1
                rc_eff = 0 if n == ng - 1 else recalc
                if n == 0 and c.turbulence:
                    for b in blocks:
                        b.des_eddy() if c.turbulence == 1 else b.kw_eddy()
                    exchange(blocks, ov, turb)
                for b in blocks:
                    b.solver_daf(n + 1, rc_eff, itr)
                    if n == 0 and c.wall_functions:
                        b.wall_functions()
                if n == 0:
                    exchange(blocks, ov, [0, 1, 2, 3])
        for n in range(ng - 1, 0, -1):
            for b in blocks:
                b.mg_prolong(n)
        for b in blocks:
            b.bcond_fm()
        total = np.zeros(5)
        for b in blocks:
            bc = b.case
            tnu = (bc.im - 2) * (bc.jm - 2) * (bc.km - 2)
            total += 10.0 ** np.asarray(b.mg_residual(1)) * tnu
        with np.errstate(divide="ignore"):
            res = np.log10(total / tnu0)
        if itc == 1:
            init = res.copy()
        eomax = res[1:4].max()
        ermax = (res[1:4] - init[1:4]).max()
        conv = (itc > c.it_min and ermax < c.er_min) or (itc > c.it_min and eomax < c.eo_min)
    return {"iterations": itc, "converged": conv, "residual": list(res), "init_residual": list(init)}


class DistExchange:
    """exchange() for one rank of a sharded run (desalm.overset_dist): the
    values this rank's host cells owe to each rank, interpolated with the
    weights and in the summation order of exchange(), packed point-major in
    the Partition's send order, crossed by overset_dist.transfer (gloo), and
    written into this rank's donee nodes.  blocks: this rank's oracle
    blocks in part.local_blocks order."""

    def __init__(self, part, blocks, dist):
        self.part, self.blocks, self.dist = part, blocks, dist
        self.turbulence = blocks[0].case.turbulence

    def __call__(self, what):
        import torch
        from desalm.overset_dist import transfer
        fields = [0, 1, 2, 3] if what == 0 else TURB_FIELDS[self.turbulence]
        nf = len(fields)
        if nf == 0:
            return
        part, blocks = self.part, self.blocks
        gp, gc = part.gather_pts, part.gather_coef
        w = _weights(gc) if len(gc) else []
        offs = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 0), (1, 1, 1)]
        send = np.zeros(max(1, len(gp) * nf))
        for fi, f in enumerate(fields):
            data = [_get(b, f) for b in blocks]
            for e in range(len(gp)):
                lb, ih, jh, kh = gp[e]
                c = blocks[lb].case
                v = data[lb]
                acc = 0.0
                for t, (a, bb, cc) in enumerate(offs):
                    acc = acc + v[(ih - 1 + a) + c.im * ((jh - 1 + bb) + c.jm * (kh - 1 + cc))] * w[t][e]
                send[e * nf + fi] = acc
        sp = part.scatter_pts
        st = torch.from_numpy(send)
        rt = torch.zeros(max(1, len(sp) * nf), dtype=torch.float64)
        transfer(self.dist, part, st, rt, nf)
        recv = rt.numpy()
        for fi, f in enumerate(fields):
            data = [_get(b, f) for b in blocks]
            for e in range(len(sp)):
                lb, i, j, k = sp[e]
                c = blocks[lb].case
                data[lb][(i - 1) + c.im * ((j - 1) + c.jm * (k - 1))] = recv[e * nf + fi]
            for lb, blk in enumerate(blocks):
                _set(blk, f, data[lb])
