"""One set decomposed over two ranks (here two processes sharing the GPU, gloo between
them): each rank solves its particles with a halo of the other's, fixed, in the whole
set's key order, then takes the halo's converged values from its owner for the force
pass.  Every rank's particles must come out with the same h, rho, gradh, gradient outputs
and forces, bit for bit, as from one solve of the whole set."""
import socket

import numpy as np
import pytest

from cosmosphere_b200 import capi, halo, inputs

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600, method="thread")]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def workload(case):
    """(fields by name, pmass, box, quintic)"""
    if case == "lattice":
        p = inputs.lattice100_workload(20)
        box, quintic = None, False
    elif case == "plummer":
        p = inputs.plummer(20000, lnsigma=0.3, vfrac=0.5, seed=31)
        th = inputs._thermo(p, 0.05, hfact=1.0)
        p["pro2"], p["cs"], p["alpha"], p["u"] = th
        box, quintic = None, True
    else:
        p = inputs.uniform_box(16000, seed=33)
        n = p.n
        p["vx"], p["vy"], p["vz"] = (inputs.gaussian(n, 0.0, 0.05, 40 + k) for k in range(3))
        th = inputs._thermo(p, 1.0)
        p["pro2"], p["cs"], p["alpha"], p["u"] = th
        box, quintic = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0], False
    n = p.n
    f = {"gid": np.arange(n, dtype=np.int64)}
    for k in halo.FIELDS:
        f[k] = np.asarray(p[k], dtype=np.float64) if k in p else np.zeros(n)
    return f, float(p["pmass"]), box, quintic


def _rank_main(rank, world, port, case, path, out):
    import datetime

    import torch.distributed as td
    td.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=300))
    try:
        full, pmass, box, quintic = workload(case)
        med = np.median(full["x"])
        part = full["x"] < med if rank == 0 else full["x"] >= med
        own = {k: v[part] for k, v in full.items()}
        res = halo.HaloStep(quintic).step(own, pmass, box=box)
        np.savez(path + f"_{rank}.npz", gid=own["gid"], **{k: v for k, v in res.items()})
        out.put((rank, int(res["halo"]), float(res["radius"])))
    finally:
        td.destroy_process_group()


def whole(case):
    full, pmass, box, quintic = workload(case)
    n = full["x"].size
    c = capi.Cosmo(quintic)
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([full["x"], full["y"], full["z"]]))
    c.upload(capi.HSML, full["h"])
    c.upload(capi.VEL, np.stack([full["vx"], full["vy"], full["vz"]]))
    c.upload(capi.ACCEL, np.stack([full["ax"], full["ay"], full["az"]]))
    c.density(n, pmass, periodic_box=box, hfact=1.0 if quintic else 1.2)
    c.upload(capi.THERMO, np.stack([full["pro2"], full["cs"], full["alpha"], full["u"]]), sorted_=True)
    c.force(n, pmass, beta=2.0, alphau=0.0)
    dens, grad = c.download(capi.DENS_OUT, n), c.download(capi.GRAD_OUT, n)
    return {"h": c.download(capi.HSML, n)[0], "rho": dens[0], "gradh": dens[1], "divv": grad[0],
            "xi": grad[1], "ddivvdt": grad[2], "force": c.download(capi.FORCE_OUT, n)}


@pytest.mark.parametrize("case", ["lattice", "plummer", "periodic"])
def test_two_rank_decomposition_equals_whole_set(case, tmp_path):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    path = str(tmp_path / "rank")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, case, path, out)) for r in range(2)]
    for p in procs:
        p.start()
    info = sorted([out.get(timeout=480) for _ in procs])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ref = whole(case)
    n = ref["h"].size
    seen = np.zeros(n, dtype=bool)
    for rank, nhalo, radius in info:
        assert 0 < nhalo < n
        r = np.load(path + f"_{rank}.npz")
        g = r["gid"]
        seen[g] = True
        for k in ("h", "rho", "gradh", "divv", "xi", "ddivvdt"):
            np.testing.assert_array_equal(r[k], ref[k][g], err_msg=f"rank {rank} {k}")
        np.testing.assert_array_equal(r["force"], ref["force"][:, g], err_msg=f"rank {rank} force")
    assert seen.all()
