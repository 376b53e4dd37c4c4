"""Set-level sharding of the batched and served forms (host logic, CPU only): the packing
rules, and the per-rank reductions over a world_size-2 gloo process group."""
import os
import socket

import numpy as np
import pytest

from cosmosphere_b200 import shard


def ensemble_sizes(nsets=256, seed=42):
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(1e4), np.log(5e5), nsets))).astype(int)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_pack_sets_is_a_balanced_partition(world):
    sizes = ensemble_sizes()
    shares = shard.pack_sets(sizes, world)
    assert len(shares) == world
    flat = sorted(k for s in shares for k in s)
    assert flat == list(range(len(sizes)))
    assert all(s == sorted(s) for s in shares)
    # longest-processing-time packing: within the largest set of the mean load
    loads = [sizes[s].sum() for s in shares]
    assert max(loads) - min(loads) <= sizes.max()
    assert shard.imbalance(sizes, shares) < 1.1


def test_pack_sets_edge_cases():
    assert shard.pack_sets([], 3) == [[], [], []]
    assert shard.pack_sets([5], 2) == [[0], []]
    with pytest.raises(ValueError):
        shard.pack_sets([1, 2], 0)


def test_continuations_follow_their_set():
    reqs = [{"kind": "new", "n": 100}, {"kind": "new", "n": 50}, {"kind": "cont", "of": 0},
            {"kind": "new", "n": 70}, {"kind": "cont", "of": 1}, {"kind": "cont", "of": 3}]
    rank = shard.pack_requests(reqs, 2)
    assert rank[2] == rank[0] and rank[4] == rank[1] and rank[5] == rank[3]
    assert sorted({rank[0], rank[1]}) == [0, 1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sizes, out):
    import datetime

    import torch.distributed as td
    td.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=60))
    try:
        shares = shard.pack_sets(sizes, world)
        mine = shares[rank]
        load = float(sum(sizes[k] for k in mine))
        total = shard.reduce_scalar(td, load, "sum")
        worst = shard.reduce_scalar(td, load, "max")
        every = shard.gather_floats(td, [float(k) for k in mine], world)
        out.put((rank, load, total, worst, every))
    finally:
        td.destroy_process_group()


def test_two_rank_reductions_over_gloo():
    import torch.multiprocessing as mp
    sizes = [int(v) for v in ensemble_sizes(64)]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, sizes, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    loads = [r[1] for r in res]
    for _, _, total, worst, every in res:
        assert total == pytest.approx(sum(sizes))
        assert worst == max(loads)
        assert sorted(int(v) for v in every) == list(range(len(sizes)))
