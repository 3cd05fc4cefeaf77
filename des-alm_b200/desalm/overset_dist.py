"""Overset blocks sharded across ranks (one process per GPU).

Each rank steps the blocks it owns; the donor exchange crosses ranks the way
the reference's does (src/mg_bintp_mom.F90:60-160, src/mg_bintp_tur.F90):
every rank interpolates the values its host cells owe to each destination
into one send buffer (point-major, destinations in rank order), the buffers
cross (the reference's mpi_alltoallv; here torch.distributed point-to-point
transfers, NCCL between GPUs), and every rank writes what it received into
its donee nodes.  All values are gathered before any is written, as in the
reference and in desalm_overset_exchange.

Partition: for every ordered pair of ranks (src, dst), the donees in map
order whose host cell lies on a block of src and whose node lies on a block
of dst.  The sender and the receiver enumerate the same global map, so the
receive buffer from src holds exactly the points src packed for it, in the
same order, without any index travelling.

mg_driver() is the lockstep physical step of desalm_overset_mg_driver and of
the reference's mg_driver over several blocks (src/mg_driver.F90:42-316):
the blocks' fine-level turbulence sub-iterations, exchange of the turbulence
scalars, their fine-level DAF steps, exchange of q(1..4), the coarse levels,
prolongation, boundary conditions, then the convergence norm summed over all
blocks of all ranks in global block order and divided by block 0's interior
count (src/mg_residual.F90:31,64-80), the same on every rank, so every rank
takes the same number of pseudo-iterations.  It is written over the blocks'
fine-grained entry points, so it steps GPU Solver blocks (with GpuExchange)
or any objects with the same methods and an exchange of their own.
"""
import numpy as np


class Partition:
    """One rank's share of a donor map.

    ov: {"n", "donee" [n][4], "host" [n][4], "coef" [n][3]} with global block
    ids (0-based) and 1-based nodes; block_rank[b]: the rank owning block b;
    local_blocks: this rank's blocks in the order of its block list.
    """

    def __init__(self, ov, block_rank, rank, nranks):
        n = int(ov["n"])
        d = np.asarray(ov["donee"], np.int64).reshape(n, 4)
        h = np.asarray(ov["host"], np.int64).reshape(n, 4)
        c = np.asarray(ov["coef"], np.float64).reshape(n, 3)
        self.block_rank = [int(r) for r in block_rank]
        self.rank, self.nranks = int(rank), int(nranks)
        self.local_blocks = [b for b, r in enumerate(self.block_rank) if r == self.rank]
        loc = {b: i for i, b in enumerate(self.local_blocks)}
        hr = np.array([self.block_rank[b] for b in h[:, 0]], np.int64) if n else np.zeros(0, np.int64)
        dr = np.array([self.block_rank[b] for b in d[:, 0]], np.int64) if n else np.zeros(0, np.int64)
        # points this rank sends to dst (its host cells), and receives from src (its donees)
        self.send_idx = [np.nonzero((hr == self.rank) & (dr == r))[0] for r in range(self.nranks)]
        self.recv_idx = [np.nonzero((dr == self.rank) & (hr == r))[0] for r in range(self.nranks)]
        self.send_counts = [len(x) for x in self.send_idx]
        self.recv_counts = [len(x) for x in self.recv_idx]
        gi = np.concatenate(self.send_idx) if n else np.zeros(0, np.int64)
        si = np.concatenate(self.recv_idx) if n else np.zeros(0, np.int64)
        # gather points: (local host block, i, j, k) + weights; scatter points: (local donee block, i, j, k)
        self.gather_pts = np.array([[loc[h[e, 0]], h[e, 1], h[e, 2], h[e, 3]] for e in gi], np.int32).reshape(-1, 4)
        self.gather_coef = c[gi].reshape(-1, 3)
        self.scatter_pts = np.array([[loc[d[e, 0]], d[e, 1], d[e, 2], d[e, 3]] for e in si], np.int32).reshape(-1, 4)
        self.send_map_index = gi     # map entries in send-buffer order
        self.recv_map_index = si     # map entries in receive-buffer order


def transfer(dist, part, send, recv, nf):
    """The buffers cross: send (rank-ordered chunks of send_counts[r] * nf
    values) to recv (chunks of recv_counts[r] * nf), point-to-point between
    ranks (batched, so NCCL groups them), this rank's own chunk copied."""
    so = [int(v) * nf for v in np.concatenate([[0], np.cumsum(part.send_counts)])]
    ro = [int(v) * nf for v in np.concatenate([[0], np.cumsum(part.recv_counts)])]
    me = part.rank
    recv[ro[me]:ro[me + 1]] = send[so[me]:so[me + 1]]
    if part.nranks == 1:
        return
    ops = []
    for r in range(part.nranks):
        if r == me:
            continue
        if part.send_counts[r]:
            ops.append(dist.P2POp(dist.isend, send[so[r]:so[r + 1]], r))
        if part.recv_counts[r]:
            ops.append(dist.P2POp(dist.irecv, recv[ro[r]:ro[r + 1]], r))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class GpuExchange:
    """The exchange of GPU Solver blocks: desalm_ov_list gathers into and
    scatters from device buffers (torch tensors on the blocks' GPU), which
    cross ranks by transfer()."""

    def __init__(self, part, solvers, dist=None):
        import torch
        from .solver import OvList
        self.part, self.dist, self.torch = part, dist, torch
        self.glist = OvList(solvers, part.gather_pts, part.gather_coef)
        self.slist = OvList(solvers, part.scatter_pts, None)
        dev = torch.device("cuda", torch.cuda.current_device())
        self.send = torch.zeros(max(1, 4 * self.glist.n), dtype=torch.float64, device=dev)
        self.recv = torch.zeros(max(1, 4 * self.slist.n), dtype=torch.float64, device=dev)

    def __call__(self, what):
        nf = self.glist.fields(what)
        if nf == 0:
            return
        if self.glist.n:
            self.glist.gather(what, self.send.data_ptr())
        self.torch.cuda.synchronize()
        transfer(self.dist, self.part, self.send, self.recv, nf)
        self.torch.cuda.synchronize()
        if self.slist.n:
            self.slist.scatter(what, self.recv.data_ptr())

    def close(self):
        self.glist.close()
        self.slist.close()


def combined_norm(dist, part, local_terms, nblocks):
    """sum over every block, in global block order, of its mean |q - qold|
    times its interior count; local_terms[i] belongs to part.local_blocks[i].
    Each block's term travels alone (one nonzero per slot of an all-reduce),
    so the sum is the same on every rank and for every partition."""
    terms = np.zeros((nblocks, 5))
    for i, b in enumerate(part.local_blocks):
        terms[b] = local_terms[i]
    if dist is not None and part.nranks > 1:
        import torch
        t = torch.from_numpy(terms)
        if dist.get_backend() == "nccl":
            t = t.cuda()
        dist.all_reduce(t)
        terms = t.cpu().numpy()
    total = np.zeros(5)
    for b in range(nblocks):
        total += terms[b]
    return total


def mg_driver(blocks, part, exchange, dist, nblocks, tnu0):
    """One physical step of this rank's blocks in lockstep with every other
    rank's; returns (iterations, converged, residual, init_residual).
    blocks: this rank's block objects in part.local_blocks order; tnu0: the
    interior node count of global block 0."""
    c = blocks[0].case
    for b in blocks:
        b.begin_step()
    ng = c.ng
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
                    exchange(1)
                for b in blocks:
                    b.solver_daf(n + 1, rc_eff, itr)
                    if n == 0 and c.wall_functions:
                        b.wall_functions()
                if n == 0:
                    exchange(0)
        for n in range(ng - 1, 0, -1):
            for b in blocks:
                b.mg_prolong(n)
        for b in blocks:
            b.bcond_fm()
        local = []
        for b in blocks:
            bc = b.case
            tnu = (bc.im - 2) * (bc.jm - 2) * (bc.km - 2)
            local.append(10.0 ** np.asarray(b.mg_residual(1)) * tnu)
        total = combined_norm(dist, part, local, nblocks)
        with np.errstate(divide="ignore"):
            res = np.log10(total / tnu0)
        if itc == 1:
            init = res.copy()
        eomax = res[1:4].max()
        ermax = (res[1:4] - init[1:4]).max()
        conv = (itc > c.it_min and ermax < c.er_min) or (itc > c.it_min and eomax < c.eo_min)
    return {"iterations": itc, "converged": conv, "residual": list(res), "init_residual": list(init)}
