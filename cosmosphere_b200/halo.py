"""One particle set decomposed over several GPUs, one process per GPU.

The reference runs a set on one GPU (include/gpu_state.hpp:25).  Here a set larger than
one GPU is split among ranks -- any partition; a Hilbert-range one keeps the halos small
-- and a density + force step on a rank goes:

1. the whole set's extents, by all-reduce (open boundaries), so that every rank's keys and
   sort order are the whole set's (``cosmo_x_set_key_extent``);
2. a halo radius D from the largest h of the set;
3. the halo: the other ranks' particles within D of this rank's, found on a coarse
   occupancy grid of the set's box dilated by D, exchanged pairwise;
4. the density solve of own + halo particles with the halo fixed (``cosmo_x_set_frozen``):
   an own particle's sums run over the same neighbours, in the same order, as in a solve
   of the whole set, so its h, rho, gradh and gradient outputs are the same bits;
5. the coverage check: the largest h any sum used (``hmaxSeen``) and the largest converged
   h of the set must lie within D / R, otherwise the step is redone with a larger D;
6. the halo's converged h, rho and gradh from their owners (``cosmo_upload_sorted``,
   ``cosmo_x_refresh_h``), then the force pass: an own particle's symmetric pairs see
   every neighbour with its converged values, so its forces are the same bits as well.

Collectives go through ``torch.distributed`` (NCCL between GPUs, gloo on the CPU); the
halo exchange is one send/receive per pair of ranks and step plus one for the converged
values.  The solves run through the C-ABI (``capi``), the library's own CUDA path.
"""
from __future__ import annotations

import math

import numpy as np

GRID = 64                 # occupancy cells per axis of the set's box
FIELDS = ("x", "y", "z", "h", "vx", "vy", "vz", "ax", "ay", "az", "pro2", "cs", "alpha", "u")


def _dist():
    import torch.distributed as dist
    return dist


def _device():
    dist = _dist()
    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def _tensor(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a)).to(_device())


def _numpy(t):
    return t.cpu().numpy()


def global_extents(x, y, z):
    """min and max of every coordinate over all ranks: (xmin, xmax, ymin, ymax, zmin, zmax)."""
    dist = _dist()
    v = np.array([-np.min(x) if x.size else -np.inf, np.max(x) if x.size else -np.inf,
                  -np.min(y) if y.size else -np.inf, np.max(y) if y.size else -np.inf,
                  -np.min(z) if z.size else -np.inf, np.max(z) if z.size else -np.inf])
    t = _tensor(v)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    m = _numpy(t)
    return np.array([-m[0], m[1], -m[2], m[3], -m[4], m[5]])


def global_max(v: float) -> float:
    dist = _dist()
    t = _tensor(np.array([v], dtype=np.float64))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(_numpy(t)[0])


def _cells(x, y, z, lo, span):
    c = []
    for a, l0, s0 in ((x, lo[0], span[0]), (y, lo[1], span[1]), (z, lo[2], span[2])):
        c.append(np.clip(np.floor((a - l0) / s0 * GRID).astype(np.int64), 0, GRID - 1))
    return c


def occupancy(x, y, z, lo, span, radius, periodic):
    """Cells of the set's box (GRID per axis) within `radius` of a cell holding one of
    these particles: the occupied cells, dilated by ceil(radius / cell) cells on every
    axis (a cube around each cell, so it holds the ball of that radius)."""
    from scipy.ndimage import maximum_filter1d
    occ = np.zeros((GRID, GRID, GRID), dtype=np.uint8)
    if x.size:
        cx, cy, cz = _cells(x, y, z, lo, span)
        occ[cx, cy, cz] = 1
    for axis in range(3):
        k = int(math.ceil(radius / (span[axis] / GRID)))
        k = min(k, GRID)
        if k > 0:
            occ = maximum_filter1d(occ, size=2 * k + 1, axis=axis, mode="wrap" if periodic else "constant", cval=0)
    return occ


def _exchange(send: list, counts_only=False):
    """Pairwise exchange: send[r] is the float64 matrix (rows) for rank r; returns the
    matrices received from every rank (own slot empty)."""
    import torch
    dist = _dist()
    world, rank = dist.get_world_size(), dist.get_rank()
    ncol = next((m.shape[1] for m in send if m is not None and m.ndim == 2), 0)
    ncol = int(global_max(float(ncol)))
    cnt = np.array([0 if (r == rank or send[r] is None) else send[r].shape[0] for r in range(world)], dtype=np.int64)
    allc = [_tensor(np.zeros(world, dtype=np.int64)) for _ in range(world)]
    dist.all_gather(allc, _tensor(cnt))
    counts = np.stack([_numpy(t) for t in allc])          # counts[src, dst]
    recv = [np.zeros((0, ncol)) for _ in range(world)]
    reqs = []
    bufs = {}
    for r in range(world):
        if r == rank:
            continue
        if counts[rank, r] > 0:
            reqs.append(dist.isend(_tensor(np.ascontiguousarray(send[r], dtype=np.float64)), dst=r))
        if counts[r, rank] > 0:
            bufs[r] = torch.empty((int(counts[r, rank]), ncol), dtype=torch.float64, device=_device())
            reqs.append(dist.irecv(bufs[r], src=r))
    for q in reqs:
        q.wait()
    for r, b in bufs.items():
        recv[r] = _numpy(b)
    return recv


def select_halo(own: dict, lo, span, radius, periodic):
    """The pairwise halo exchange: every rank sends the others its particles lying in
    their occupancy within `radius`.  Returns (halo rows received, what was sent to each
    rank as row indices of `own`).  Rows: gid then FIELDS."""
    dist = _dist()
    world, rank = dist.get_world_size(), dist.get_rank()
    occ = occupancy(own["x"], own["y"], own["z"], lo, span, radius, periodic)
    maps = [_tensor(np.zeros_like(occ)) for _ in range(world)]
    dist.all_gather(maps, _tensor(occ))
    maps = [_numpy(m) for m in maps]
    cx, cy, cz = _cells(own["x"], own["y"], own["z"], lo, span)
    sent_idx, send = [], []
    rows = np.stack([own["gid"].astype(np.float64)] + [own[f] for f in FIELDS], axis=1) if own["x"].size else \
        np.zeros((0, 1 + len(FIELDS)))
    for r in range(world):
        if r == rank:
            sent_idx.append(np.zeros(0, dtype=np.int64))
            send.append(None)
            continue
        sel = np.nonzero(maps[r][cx, cy, cz])[0] if own["x"].size else np.zeros(0, dtype=np.int64)
        sent_idx.append(sel)
        send.append(rows[sel])
    recv = _exchange(send)
    halo = np.concatenate([m for m in recv if m.size] or [np.zeros((0, 1 + len(FIELDS)))], axis=0)
    return halo, sent_idx


class HaloStep:
    """Density + force steps of one rank's part of a decomposed set."""

    def __init__(self, quintic: bool = False):
        from . import capi
        self.c = capi.Cosmo(quintic)
        self.quintic = quintic
        self.R = float(self.c.L.cosmo_kernel_radius())

    def step(self, own: dict, pmass: float, *, box=None, tolh=1e-4, hfact=None, beta=2.0, alphau=0.0,
             disc=0, pdv=1, shock=1, max_iter=100, radius_factor=1.3):
        """own: gid (global index, int64) and FIELDS of this rank's particles.  Returns
        this rank's outputs in its own order (h, rho, gradh, divv, xi, ddivvdt, force),
        the halo size and the radius used."""
        from . import capi
        c = self.c
        hfact = hfact if hfact is not None else (1.0 if self.quintic else 1.2)
        n = own["x"].size
        periodic = box is not None
        if periodic:
            ext = np.asarray(box, dtype=np.float64)
        else:
            ext = global_extents(own["x"], own["y"], own["z"])
        lo = ext[0::2]
        span = np.maximum(ext[1::2] - ext[0::2], 1e-300) * (1.0 if periodic else 1.0 + 1e-12)
        hlive = own["h"][np.isfinite(own["h"]) & (own["h"] > 0)]
        hmax = global_max(float(hlive.max()) if hlive.size else 0.0)
        D = self.R * hmax * radius_factor
        for _attempt in range(8):
            halo, sent = select_halo(own, lo, span, D, periodic)
            nh = halo.shape[0]
            gid = np.concatenate([own["gid"].astype(np.int64), halo[:, 0].astype(np.int64)])
            cols = {f: np.concatenate([own[f], halo[:, 1 + k]]) for k, f in enumerate(FIELDS)}
            perm = np.argsort(gid, kind="stable")     # the whole set's order among equal keys
            inv = np.empty_like(perm)
            inv[perm] = np.arange(perm.size)
            cols = {f: v[perm] for f, v in cols.items()}
            frozen = np.zeros(perm.size, dtype=np.int32)
            frozen[inv[n:]] = 1
            nc = perm.size
            c.arrays_init(nc)
            c.upload(capi.POS, np.stack([cols["x"], cols["y"], cols["z"]]))
            c.upload(capi.HSML, cols["h"])
            c.upload(capi.VEL, np.stack([cols["vx"], cols["vy"], cols["vz"]]))
            c.upload(capi.ACCEL, np.stack([cols["ax"], cols["ay"], cols["az"]]))
            c.set_key_extent(None if periodic else ext)
            c.set_frozen(frozen)
            try:
                st = c.density_status(nc, pmass, periodic_box=box, tolh=tolh, hfact=hfact, max_iter=max_iter,
                                      with_gradients=True)
                seen = c.scalar("hmaxSeen")
            finally:
                c.set_frozen(None)
                c.set_key_extent(None)
            h_c = c.download(capi.HSML, nc)[0]
            mine = inv[:n]
            hfin = h_c[mine]
            hf = hfin[np.isfinite(hfin) & (hfin > 0)]
            need = self.R * global_max(max(seen, float(hf.max()) if hf.size else 0.0))
            ok = global_max(0.0 if need <= D else 1.0) == 0.0
            if ok:
                break
            D = need * 1.05
        else:
            raise RuntimeError("halo radius did not settle")
        if st not in (0,):
            raise RuntimeError(f"density solve status {st}")
        dens = c.download(capi.DENS_OUT, nc)
        grad = c.download(capi.GRAD_OUT, nc)
        # the halo's converged h, rho, gradh from their owners, in the order they were sent
        vals = np.stack([hfin, dens[0][mine], dens[1][mine]], axis=1)
        back = _exchange([None if s.size == 0 else vals[s] for s in sent])
        hv = np.concatenate([m for m in back if m.size] or [np.zeros((0, 3))], axis=0)
        h_all, rho_all, gh_all = h_c.copy(), dens[0].copy(), dens[1].copy()
        hal = inv[n:]
        h_all[hal], rho_all[hal], gh_all[hal] = hv[:, 0], hv[:, 1], hv[:, 2]
        c.upload(capi.HSML, h_all, sorted_=True)
        c.upload(capi.DENS_OUT, np.stack([rho_all, gh_all]), sorted_=True)
        if c.refresh_h() != 0:
            raise RuntimeError("refresh after the halo's converged values failed")
        c.upload(capi.THERMO, np.stack([cols["pro2"], cols["cs"], cols["alpha"], cols["u"]]), sorted_=True)
        c.force(nc, pmass, beta=beta, alphau=alphau, disc=disc, pdv=pdv, shock=shock)
        force = c.download(capi.FORCE_OUT, nc)
        return {"h": hfin, "rho": dens[0][mine], "gradh": dens[1][mine], "divv": grad[0][mine],
                "xi": grad[1][mine], "ddivvdt": grad[2][mine], "force": force[:, mine],
                "halo": nh, "radius": D}
