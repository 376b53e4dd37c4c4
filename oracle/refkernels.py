"""The reference's own physics kernels as a parity checker (test infrastructure only).

oracle/_ref/libref_physics_{cubic,quintic}.so holds the reference's
sphDensityKernelJList (src/density_base.cu:237-334), sphGradientsKernel + xiLimiter
(:511-714), forcePrepKernel and sphForceKernelJList (src/force.cu:92-383), compiled for
sm_100a from the reference's sources by `make -C oracle ref` (ref_pin/physics_probe.cu).
Only tests use this module.

`solve` runs the reference's density / smoothing-length pipeline as its host code does
(src/density_base.cu:790-886 and :936-975; src/force.cu:385-455) on a particle order,
leaf layout and leaf geometry handed in (this library's tree): each Newton iteration
takes hmax over the active leaves, j-leaf lists, one launch of the reference's kernel
over the still-active particles, and the stable compaction of the unconverged ones;
then the gradient sweep at the converged h over the full-tree gather lists, and the
force pass over the symmetric lists.

The j-leaf lists are built here in numpy with the reference's leaf-level accept tests
(include/tree.cuh:228-252: the i-leaf box inflated by radkernel*hmax overlapping the
candidate's box for gather; box distance within radkernel*max(hmax_i, hmax_j) for the
symmetric lists), with a relative margin of 1e-9 so they are supersets, in ascending
leaf order.  The kernels test every pair exactly, so a superset in ascending order gives
the same accepted pairs, summed in the same (ascending j) order, as the exact lists.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_libs: dict = {}


def lib_path(quintic: bool = False) -> str:
    return os.path.join(HERE, "_ref", "libref_physics_quintic.so" if quintic else "libref_physics_cubic.so")


def available(quintic: bool = False) -> bool:
    return os.path.exists(lib_path(quintic))


def _load(quintic: bool):
    if quintic not in _libs:
        L = ctypes.CDLL(lib_path(quintic))
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ref_density_step.argtypes = [I, P, I, I, P, P, P, P, P, P, P, P, D, P, I, P, P, P, I, P, D, D]
        L.ref_density_step.restype = I
        L.ref_gradients.argtypes = [I, P, I, P, P, P, P, P, P, P, P, P, P, P, D, P, I, P, P, P, I, P]
        L.ref_gradients.restype = I
        L.ref_force.argtypes = [I, P, I, P, P, P, P, P, P, P, P, D, D, D, D, I, I, I, P, I, P, P, P, I, P]
        L.ref_force.restype = I
        _libs[quintic] = L
    return _libs[quintic]


def _p(a):
    return a.ctypes.data


class LeafGeometry:
    """Leaf cubes (centre, half-size) and particle layout of one tree, in leaf order."""

    def __init__(self, layout, centers, halves, particle_leaf, box=None):
        self.layout = np.ascontiguousarray(layout, dtype=np.uint32)
        self.c = np.ascontiguousarray(centers, dtype=np.float64)       # (nL, 3)
        self.s = np.ascontiguousarray(halves, dtype=np.float64)        # (nL, 3)
        self.pleaf = np.ascontiguousarray(particle_leaf, dtype=np.int32)
        self.nL = self.c.shape[0]
        self.box = None if box is None else np.asarray(box, dtype=np.float64)
        self.L = None if box is None else np.array([box[1] - box[0], box[3] - box[2], box[5] - box[4]])

    def hmax(self, h):
        """Largest finite h in each leaf (include/tree.cuh:177-191)."""
        lay = self.layout.astype(np.int64)
        hf = np.where(np.isfinite(h), h, 0.0)
        out = np.zeros(self.nL)
        nonempty = lay[1:] > lay[:-1]
        out[nonempty] = np.maximum.reduceat(hf[: lay[-1]], lay[:-1][nonempty])
        return np.maximum(out, 0.0)

    def _gaps(self, rows):
        d = np.abs(self.c[rows, None, :] - self.c[None, :, :])
        if self.L is not None:
            d = np.minimum(d, self.L[None, None, :] - d)
        return np.maximum(d - (self.s[rows, None, :] + self.s[None, :, :]), 0.0)

    def lists(self, leaves, hmax, R, symmetric):
        """CSR j-leaf lists (ascending) for `leaves`; other leaves get empty lists."""
        jcount = np.zeros(self.nL, dtype=np.int32)
        rows_out = {}
        margin = 1.0 + 1e-9
        for k in range(0, len(leaves), 256):
            rows = np.asarray(leaves[k:k + 256])
            g = self._gaps(rows)
            if symmetric:
                rs = R * np.maximum(hmax[rows, None], hmax[None, :]) * margin
                ok = np.sum(g * g, axis=2) <= rs * rs
            else:
                ok = np.all(g <= (R * hmax[rows] * margin)[:, None, None], axis=2)
            for r, row in zip(rows, ok):
                js = np.nonzero(row)[0].astype(np.int32)
                rows_out[int(r)] = js
                jcount[r] = js.size
        joff = np.zeros(self.nL + 1, dtype=np.int32)
        joff[1:] = np.cumsum(jcount)
        jlist = np.zeros(max(int(joff[-1]), 1), dtype=np.int32)
        for r, js in rows_out.items():
            jlist[joff[r]:joff[r] + js.size] = js
        return joff, jcount, jlist


def solve(quintic, geo: LeafGeometry, x, y, z, h0, pmass, n_alive, *, tolh=1e-4, hfact=None, max_iter=100,
          vel=None, acc=None, thermo=None, beta=2.0, alphau=0.0, disc=0, pdv=1, shock=1):
    """Run the reference's kernels through the reference's solve sequence on one
    Hilbert-ordered particle set.  Returns a dict of Hilbert-order outputs and the
    per-iteration active counts."""
    L = _load(bool(quintic))
    R = 3.0 if quintic else 2.0
    if hfact is None:
        hfact = 1.0 if quintic else 1.2
    n = x.size
    x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
    h = np.ascontiguousarray(h0, dtype=np.float64).copy()
    rho = np.zeros(n)
    gradh = np.zeros(n)
    conv = np.zeros(n, dtype=np.int32)
    periodic = 1 if geo.box is not None else 0
    box6 = np.ascontiguousarray(geo.box if periodic else np.zeros(6))
    pleaf = np.zeros(n, dtype=np.int32)
    pleaf[:n_alive] = geo.pleaf[:n_alive]
    active = np.arange(n_alive, dtype=np.int32)
    per_iter = []
    hm = np.zeros(geo.nL)
    for _ in range(max_iter):
        act_leaves = np.unique(pleaf[active])
        hm[act_leaves] = geo.hmax(h)[act_leaves]
        joff, jcnt, jl = geo.lists(act_leaves, hm, R, symmetric=False)
        rc = L.ref_density_step(periodic, _p(box6), n, active.size, _p(active), _p(x), _p(y), _p(z), _p(h), _p(rho),
                                _p(gradh), _p(conv), pmass, _p(pleaf), geo.nL, _p(joff), _p(jcnt), _p(jl), jl.size,
                                _p(geo.layout), tolh, hfact)
        assert rc == 0, "reference density kernel failed"
        per_iter.append(active.size)
        active = active[conv[active] == 0]
        if active.size == 0:
            break
    out = {"h": h, "nr_rho": rho.copy(), "nr_gradh": gradh.copy(), "activePerIter": np.array(per_iter),
           "unconverged": int(active.size)}
    if vel is None:
        return out
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    acc = np.ascontiguousarray(acc, dtype=np.float64)
    hmax_all = geo.hmax(h)
    all_leaves = np.arange(geo.nL)
    joff, jcnt, jl = geo.lists(all_leaves, hmax_all, R, symmetric=False)
    g = {k: np.zeros(n) for k in ("rho", "gradh", "divv", "xi", "ddivvdt")}
    rc = L.ref_gradients(periodic, _p(box6), n, _p(x), _p(y), _p(z), _p(vel), _p(acc), _p(h), _p(g["rho"]),
                         _p(g["gradh"]), _p(g["divv"]), _p(g["xi"]), _p(g["ddivvdt"]), pmass, _p(pleaf), geo.nL,
                         _p(joff), _p(jcnt), _p(jl), jl.size, _p(geo.layout))
    assert rc == 0, "reference gradient kernel failed"
    out.update(g)
    if thermo is None:
        return out
    thermo = np.ascontiguousarray(thermo, dtype=np.float64)
    joff, jcnt, jl = geo.lists(all_leaves, hmax_all, R, symmetric=True)
    f = np.zeros(6 * n)
    rc = L.ref_force(periodic, _p(box6), n, _p(x), _p(y), _p(z), _p(vel), _p(h), _p(g["gradh"]), _p(thermo), _p(f),
                     pmass, beta, alphau, hfact, disc, pdv, shock, _p(pleaf), geo.nL, _p(joff), _p(jcnt), _p(jl),
                     jl.size, _p(geo.layout))
    assert rc == 0, "reference force kernels failed"
    f = f.reshape(6, n)
    for k, name in enumerate(("fx", "fy", "fz", "f4", "vsigmax", "divvF")):
        out[name] = f[k]
    return out
