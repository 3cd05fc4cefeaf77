"""Overset blocks sharded across ranks (desalm.overset_dist): the partition of
a donor map into per-rank-pair send and receive lists, and the lockstep
multi-block physical step with the exchange crossing ranks, run here on the
CPU oracle's blocks with two gloo ranks.  The sharded run must take the same
pseudo-iterations, report the same combined residual and leave every block
with the same values, bit for bit, as the single-process oracle driver
(oracle/overset_oracle.py mg_driver) on the same blocks: the exchange writes
the same interpolated values and the combined norm is summed in global block
order whatever the partition.  The k-omega case moves omega across ranks with
k (mg_bintp_tur's turbulence fields)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from desalm import cases
from desalm.overset_dist import Partition

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_pairs_senders_with_receivers():
    """Every map entry is sent by exactly one rank and received by exactly one,
    and the receiver's list from a source equals the source's list for it."""
    blocks, ov = cases.overset_chain(3)
    n = ov["n"]
    for owner in ([0, 1, 0], [0, 0, 1], [1, 0, 1], [0, 0, 0]):
        world = max(owner) + 1
        parts = [Partition(ov, owner, r, world) for r in range(world)]
        sent = np.concatenate([np.concatenate(p.send_idx) for p in parts])
        got = np.concatenate([np.concatenate(p.recv_idx) for p in parts])
        assert sorted(sent.tolist()) == list(range(n)) and sorted(got.tolist()) == list(range(n))
        for src in range(world):
            for dst in range(world):
                assert np.array_equal(parts[src].send_idx[dst], parts[dst].recv_idx[src])
        d = ov["donee"].reshape(n, 4)
        h = ov["host"].reshape(n, 4)
        for p in parts:
            assert len(p.gather_pts) == sum(p.send_counts) and len(p.scatter_pts) == sum(p.recv_counts)
            for row, e in zip(p.gather_pts, p.send_map_index):
                assert p.local_blocks[row[0]] == h[e, 0] and tuple(row[1:]) == tuple(h[e, 1:])
            for row, e in zip(p.scatter_pts, p.recv_map_index):
                assert p.local_blocks[row[0]] == d[e, 0] and tuple(row[1:]) == tuple(d[e, 1:])


def _oracle_blocks(oracle_mod, specs):
    out = []
    for case, grid, state, om in specs:
        o = oracle_mod.OracleSolver(case)
        o.set_grid(grid["x"], grid["y"], grid["z"], grid.get("wd"))
        o.set_state(state["q"], state["qn"], state["qnm1"], state["nut"])
        if om is not None:
            o.set_omega(om["omega"], om["omega_n"], om["omega_nm1"])
        out.append(o)
    return out


def _spec(nblocks, turbulence, itmax):
    """([(case, grid, state, omega or None)], map); turbulence 2 is the
    SA chain with the k-omega model (cases.with_kw)."""
    specs, ov = cases.overset_chain(nblocks, seed=5, turbulence=min(turbulence, 1), itmax=itmax)
    out = []
    for c, g, st in specs:
        om = None
        if turbulence == 2:
            c, g, st, om = cases.with_kw(c, g, st)
        c.iter[0], c.iter[1], c.iter[2] = 1, 1, 1
        out.append((c, g, st, om))
    return out, ov


def _worker(rank, world, port, owner, nblocks, turbulence, itmax, q):
    import sys
    import datetime
    for p in (ROOT, os.path.join(ROOT, "des-alm_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    import oracle
    import overset_oracle as oo
    from desalm.overset_dist import Partition, mg_driver
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        oracle.lib()
        specs, ov = _spec(nblocks, turbulence, itmax)
        part = Partition(ov, owner, rank, world)
        mine = _oracle_blocks(oracle, [specs[b] for b in part.local_blocks])
        c0 = specs[0][0]
        tnu0 = (c0.im - 2) * (c0.jm - 2) * (c0.km - 2)
        rep = mg_driver(mine, part, oo.DistExchange(part, mine, dist), dist, nblocks, tnu0)
        states = {b: (mine[i].get_state()["q"], mine[i].get_omega()["omega"] if turbulence == 2 else None)
                  for i, b in enumerate(part.local_blocks)}
        q.put((rank, rep, states))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("owner,turbulence", [([0, 1], 1), ([0, 1, 0], 1), ([0, 0, 1], 0), ([1, 0, 0], 2)])
def test_sharded_step_equals_single_process(owner, turbulence, oracle_mod):
    import overset_oracle as oo
    nblocks, itmax = len(owner), 3
    world = max(owner) + 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, owner, nblocks, turbulence, itmax, q))
             for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    # the single-process run on the same blocks
    specs, ov = _spec(nblocks, turbulence, itmax)
    blocks = _oracle_blocks(oracle_mod, specs)
    ref = oo.mg_driver(blocks, ov)
    for rank, rep, states in out:
        assert rep["iterations"] == ref["iterations"]
        assert rep["residual"] == ref["residual"] and rep["init_residual"] == ref["init_residual"]
        for b, (qv, wv) in states.items():
            assert np.array_equal(qv, blocks[b].get_state()["q"]), b
            if wv is not None:
                assert np.array_equal(wv, blocks[b].get_omega()["omega"]), b
