"""Multi-rank beam sharding on CPU (gloo, world size 2): the partition and the
reductions of beamax_b200.sharding, with the oracle's C summation as each
rank's local operator.  The sharded forward (all-reduce of the ranks' partial
fields) and transpose (all-reduce of the zero-padded per-coefficient
gradients) equal the unsharded oracle results."""

import os
import socket

import numpy as np
import pytest

from beamax_b200.sharding import ShardingStrategy, shard_range


def test_shard_range_partitions_every_item_once():
    for n in (0, 1, 7, 64, 1001):
        for world in (1, 2, 3, 8):
            ranges = [shard_range(n, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [hi - lo for lo, hi in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_strategy_rejects_uneven_beam_counts_like_the_reference():
    s = ShardingStrategy()
    s.world, s.rank = 4, 1
    with pytest.raises(ValueError, match="not divisible by 4 devices"):
        s.shard(3)  # 6 beams over 4 ranks
    assert s.shard(8) == (2, 4)


def _case():
    from oracle import msgb as om

    N = (64, 64)
    dom = om.Dom(N=N, dx=(1e-4, 1e-4), periodic=(False, False), cfl=0.3, c=1500.0)
    ow = om.Wpt(om.Decomp(2, N, (4, 8), (1, 1)), 2, "rectangular_mirror")
    rng = np.random.default_rng(0)
    p0 = rng.standard_normal(N)
    mask = np.zeros(N)
    mask[0, :] = 1
    mask[:, 0] = 1
    sens = om.sensor_positions_from_mask(dom, mask)
    ts = dom.generate_time_domain()[::8]
    bm = om.select_beams(p0, dom, ow, 96)
    return dom, sens, ts, bm


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from beamax_b200.sharding import ShardingStrategy, assemble_shards, reduce_partials
    from oracle import build as ob
    from oracle import msgb as om

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dom, sens, ts, bm = _case()
        tab = om.beam_table(bm, 1500.0)
        n = bm.idx.size
        strat = ShardingStrategy()
        lo, hi = strat.shard(n)
        sub = {k: v[lo:hi] for k, v in tab.items()}
        part = ob.sum_hom(sub, 1500.0, ts, sens, dom.grid_size, dom.periodic)
        y = reduce_partials(torch.from_numpy(part)).numpy()
        data = np.random.default_rng(7).standard_normal(y.shape)
        g = ob.adj_hom(sub, bm.a0_unit[lo:hi], 1500.0, ts, sens, dom.grid_size, dom.periodic, data)
        g_all = assemble_shards(torch.from_numpy(g), n, lo).numpy()
        if rank == 0:
            y_ref = ob.sum_hom(tab, 1500.0, ts, sens, dom.grid_size, dom.periodic)
            g_ref = ob.adj_hom(tab, bm.a0_unit, 1500.0, ts, sens, dom.grid_size, dom.periodic, data)
            np.savez(out, y=y, y_ref=y_ref, g=g_all, g_ref=g_ref, lo=lo, hi=hi)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_forward_and_transpose_equal_unsharded_on_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    from oracle import build as ob

    ob.build()
    out = str(tmp_path / "r0.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    r = np.load(out)
    assert (int(r["lo"]), int(r["hi"])) == (0, 48)
    assert np.linalg.norm(r["y"] - r["y_ref"]) <= 1e-12 * np.linalg.norm(r["y_ref"])
    assert np.linalg.norm(r["g"] - r["g_ref"]) <= 1e-12 * np.linalg.norm(r["g_ref"])
