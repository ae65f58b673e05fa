"""Owner-computes sharding of a contraction across processes (CPU; no GPU needed).

tb_mult_owned gives each rank its output blocks under the FLOP-balanced owner rule
(every rank derives the same assignment from the operands alone).  Checked: the
shares of 1..4 ranks are disjoint, cover every admitted output block and stay within
25 % of a perfect balance; and two gloo ranks that each compute only their own
blocks (with the oracle) and all-reduce a zero-initialised output reproduce the
single-process result bit for bit."""
import os
import socket

import numpy as np
import pytest

import tamm_b200 as tb
from tamm_b200 import workloads as W
from tamm_b200.tamm import mult_info, mult_owned


def _ladder(oa=4, va=13, seed=3):
    rng = np.random.default_rng(seed)
    occ, virt = W.random_tiles(oa, 3, 6, rng), W.random_tiles(va, 3, 6, rng)
    MO = W.mo_tiled(oa, va, occ, virt)
    O, V = MO("occ"), MO("virt")
    v = tb.Tensor([V, V, V, V], spin=(2, 2))
    t2 = tb.Tensor([V, V, O, O], spin=(2, 2))
    r2 = tb.Tensor([V, V, O, O], spin=(2, 2))
    a, b, c, d = V.labels(4)
    i, j = O.labels(2)
    return v, t2, r2, (r2(a, b, i, j), v(a, b, c, d), t2(c, d, i, j))


@pytest.mark.parametrize("nranks", [1, 2, 3, 4])
def test_shares_cover_disjoint_balanced(nranks):
    _, _, r2, (lhs, a, b) = _ladder()
    ngroups, _, total = mult_info(lhs, a, b)
    shares = [mult_owned(lhs, a, b, r, nranks) for r in range(nranks)]
    offs = np.concatenate([s[0] for s in shares])
    assert len(offs) == ngroups and len(set(offs.tolist())) == ngroups
    assert set(offs.tolist()) == set(mult_owned(lhs, a, b, 0, 1)[0].tolist())
    loads = np.array([s[1] for s in shares])
    assert abs(loads.sum() - total) <= 1e-9 * total
    assert loads.max() <= 1.25 * total / nranks


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import torch
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v, t2, r2, (lhs, a, b) = _ladder()
        ob = lambda t: O.BlockTensor([s.tile_sizes for s in t.spaces], [s.tile_spins for s in t.spaces],
                                     [0, 0, 1, 1])
        ov, ot, full = ob(v), ob(t2), ob(r2)
        O.fill_uniform(ov.data[:ov.total], 5)
        O.fill_normal(ot.data[:ot.total], 6, 0, 0.0, 1e-2)
        O.mult_bufacc(full, [1, 2, 5, 6], 1.0, ov, [1, 2, 3, 4], ot, [3, 4, 5, 6])
        # this rank's blocks only, then the sum over ranks
        mine = np.zeros(full.total)
        ends = dict(zip(full.offsets.tolist(), list(full.offsets[1:].tolist()) + [full.total]))
        owned, _ = mult_owned(lhs, a, b, rank, world)
        for off in owned.tolist():
            mine[off:ends[off]] = full.data[off:ends[off]]
        x = torch.from_numpy(mine)
        dist.all_reduce(x)
        shares = [None] * world
        dist.all_gather_object(shares, owned.tolist())
        if rank == 0:
            out.put((np.array_equal(x.numpy(), full.data[:full.total]), shares, len(full.offsets)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reassemble_the_contraction():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    equal, shares, nblocks = out.get(timeout=60)
    assert equal
    assert not set(shares[0]) & set(shares[1]) and len(shares[0]) + len(shares[1]) == nblocks
