"""The halo exchange of a set decomposed over ranks (host logic, CPU only, a world_size-2
gloo process group): every rank receives every other rank's particle within the halo
radius of one of its own, and only particles in the dilated occupancy of its own."""
import socket

import numpy as np
import pytest

from cosmosphere_b200 import halo


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def make_set(n, seed, periodic):
    rng = np.random.default_rng(seed)
    x, y, z = (rng.uniform(0.0, 1.0, n) for _ in range(3))
    if not periodic:           # a clustered set: the halo crosses a dense region
        x, y, z = (0.5 + 0.25 * rng.standard_normal(n) for _ in range(3))
    own = {"gid": np.arange(n, dtype=np.int64), "x": x, "y": y, "z": z}
    for f in halo.FIELDS[3:]:
        own[f] = rng.uniform(0.5, 1.5, n)
    return own


def _rank_main(rank, world, port, n, seed, periodic, radius, out):
    import datetime

    import torch.distributed as td
    td.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=60))
    try:
        full = make_set(n, seed, periodic)
        part = full["x"] < np.median(full["x"]) if rank == 0 else full["x"] >= np.median(full["x"])
        own = {k: v[part] for k, v in full.items()}
        if periodic:
            ext = np.array([0.0, 1.0, 0.0, 1.0, 0.0, 1.0])
        else:
            ext = halo.global_extents(own["x"], own["y"], own["z"])
        lo, span = ext[0::2], ext[1::2] - ext[0::2]
        got, sent = halo.select_halo(own, lo, span, radius, periodic)
        out.put((rank, got[:, 0].astype(np.int64), [s.tolist() for s in sent]))
    finally:
        td.destroy_process_group()


@pytest.mark.parametrize("periodic", [False, True])
def test_two_rank_halo_exchange_over_gloo(periodic):
    import torch.multiprocessing as mp
    n, seed, radius = 4000, 7, 0.08
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, n, seed, periodic, radius, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([out.get(timeout=120) for _ in procs], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = make_set(n, seed, periodic)
    pos = np.stack([full["x"], full["y"], full["z"]], 1)
    med = np.median(full["x"])
    parts = [np.nonzero(full["x"] < med)[0], np.nonzero(full["x"] >= med)[0]]
    for rank, got, _ in res:
        mine, other = parts[rank], parts[1 - rank]
        d = pos[other][:, None, :] - pos[mine][None, :, :]
        if periodic:
            d = d - np.round(d)
        near = np.min(np.sqrt((d ** 2).sum(-1)), axis=1) < radius
        need = set(other[near].tolist())
        have = set(got.tolist())
        assert need <= have                       # nothing within the radius is missing
        assert have <= set(other.tolist())        # only the other rank's particles
        assert len(have) == got.size              # each once
    # what one rank sent is what the other received
    assert sorted(np.asarray(parts[0])[res[0][2][1]].tolist()) == sorted(res[1][1].tolist())
    assert sorted(np.asarray(parts[1])[res[1][2][0]].tolist()) == sorted(res[0][1].tolist())
