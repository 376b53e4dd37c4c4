"""Seeded synthetic particle sets (csrc/inputs.cpp): the reference driver's lattice and
jiggle, and the generators of the measured workloads.  Host-only."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .capi import LIBDIR

_L = None


def _lib():
    global _L
    if _L is None:
        path = os.path.join(LIBDIR, "libcosmo_inputs.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build with make -C cosmosphere_b200")
        L = ctypes.CDLL(path)
        P, I, D, U64, LNG = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_long
        L.cin_lattice_count.argtypes = [I]
        L.cin_lattice_count.restype = LNG
        L.cin_lattice.argtypes = [I, P, P, P, P]
        L.cin_lattice.restype = D
        L.cin_jiggle_ref.argtypes = [LNG, P, ctypes.c_uint]
        L.cin_jiggle_ref.restype = LNG
        L.cin_jiggle_frac.argtypes = [LNG, P, D, D, D, U64]
        L.cin_jiggle_frac.restype = LNG
        L.cin_gaussian.argtypes = [LNG, P, D, D, U64]
        L.cin_uniform.argtypes = [LNG, P, D, D, U64]
        L.cin_uniform_box.argtypes = [LNG, P, P, P, P, D, D, D, U64]
        L.cin_uniform_box.restype = D
        L.cin_plummer.argtypes = [LNG, P, P, P, P, P, P, P, D, D, D, D, D, D, U64]
        L.cin_plummer.restype = D
        _L = L
    return _L


def _p(a):
    return a.ctypes.data


class Particles(dict):
    """x, y, z, h (and optionally vx, vy, vz, u) as float64 arrays, plus n and pmass."""

    @property
    def n(self):
        return int(self["x"].size)


def lattice(npartx: int) -> Particles:
    """The reference driver's close-packed lattice (src/main.cu:84-109)."""
    L = _lib()
    n = L.cin_lattice_count(npartx)
    x, y, z, h = (np.empty(n) for _ in range(4))
    pm = L.cin_lattice(npartx, _p(x), _p(y), _p(z), _p(h))
    return Particles(x=x, y=y, z=z, h=h, pmass=pm)


def jiggle_ref(h: np.ndarray, seed: int = 42) -> int:
    """The reference driver's jiggle (src/main.cu:47-63), in place."""
    return int(_lib().cin_jiggle_ref(h.size, _p(h), seed))


def jiggle_frac(h: np.ndarray, frac=0.01, lo=0.65, hi=1.35, seed: int = 42) -> int:
    """round(frac*n) particles picked uniformly, h scaled by U[lo, hi], in place."""
    return int(_lib().cin_jiggle_frac(h.size, _p(h), frac, lo, hi, seed))


def gaussian(n, mean=0.0, sigma=1.0, seed=42) -> np.ndarray:
    a = np.empty(n)
    _lib().cin_gaussian(n, _p(a), mean, sigma, seed)
    return a


def uniform(n, lo=0.0, hi=1.0, seed=42) -> np.ndarray:
    a = np.empty(n)
    _lib().cin_uniform(n, _p(a), lo, hi, seed)
    return a


def uniform_box(n, hfac=1.2, hlo=0.8, hhi=1.2, seed=42) -> Particles:
    x, y, z, h = (np.empty(n) for _ in range(4))
    pm = _lib().cin_uniform_box(n, _p(x), _p(y), _p(z), _p(h), hfac, hlo, hhi, seed)
    return Particles(x=x, y=y, z=z, h=h, pmass=pm)


def plummer(n, rmax=20.0, hfact=1.0, lnsigma=0.3, ulo=1.0, uhi=1.0, vfrac=0.5, seed=42) -> Particles:
    """Plummer sphere (a=1, M=1, G=1) truncated at rmax; h from the local density times a
    log-normal factor (lnsigma > 0) or U[ulo, uhi]; |v| = vfrac * circular speed."""
    a = [np.empty(n) for _ in range(7)]
    pm = _lib().cin_plummer(n, *(_p(v) for v in a), rmax, hfact, lnsigma, ulo, uhi, vfrac, seed)
    x, y, z, h, vx, vy, vz = a
    return Particles(x=x, y=y, z=z, h=h, vx=vx, vy=vy, vz=vz, pmass=pm)


def lattice100_workload(npartx: int = 100, seed: int = 42, vsigma=0.1, u=1.0, gamma=5.0 / 3.0,
                        alpha=1.0, hfact=1.2) -> Particles:
    """The lattice-with-jiggle density + force workload: the close-packed lattice, 1% of
    particles with h scaled by U[0.65, 1.35], velocities N(0, vsigma^2) per component,
    u = 1, gamma = 5/3, alpha_AV = 1.  Thermodynamics use rho = pmass (hfact/h)^3 of the
    initial h: P = (gamma-1) rho u, pro2 = P/rho^2, cs = sqrt(gamma (gamma-1) u)."""
    p = lattice(npartx)
    jiggle_frac(p["h"], 0.01, 0.65, 1.35, seed)
    n = p.n
    p["vx"] = gaussian(n, 0.0, vsigma, seed + 1)
    p["vy"] = gaussian(n, 0.0, vsigma, seed + 2)
    p["vz"] = gaussian(n, 0.0, vsigma, seed + 3)
    rho = p["pmass"] * (hfact / p["h"]) ** 3
    p["pro2"] = (gamma - 1.0) * u / rho
    p["cs"] = np.full(n, np.sqrt(gamma * (gamma - 1.0) * u))
    p["alpha"] = np.full(n, alpha)
    p["u"] = np.full(n, u)
    return p


def ensemble_sizes(nsets: int = 256, nmin: float = 1e4, nmax: float = 5e5, seed: int = 42) -> np.ndarray:
    """Particle counts of the batched-ensemble sets: log-uniform in [nmin, nmax], seeded."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax), nsets))).astype(np.int64)


def ensemble_sets(nsets: int = 256, nmin: float = 1e4, nmax: float = 5e5, seed: int = 42, only=None):
    """The batched-ensemble workload: nsets independent sets with sizes log-uniform in
    [nmin, nmax] (seeded); even sets uniform random in the unit periodic box, odd sets
    Plummer spheres (a = 1, r < 20); h = 1.2 x the local mean spacing x U[0.8, 1.2]
    (the spacing from the mean density for the box, from the Plummer density profile
    for the spheres); pmass = 1/N.  With only (set indices), just those sets, each the
    same as in the full ensemble."""
    sizes = ensemble_sizes(nsets, nmin, nmax, seed)
    keep = set(range(nsets)) if only is None else set(int(k) for k in only)
    sets = []
    for k, n in enumerate(sizes):
        if k not in keep:
            continue
        if k % 2 == 0:
            p = uniform_box(int(n), hfac=1.2, hlo=0.8, hhi=1.2, seed=seed + 1000 + k)
            p["box"] = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
        else:
            p = plummer(int(n), rmax=20.0, hfact=1.2, lnsigma=0.0, ulo=0.8, uhi=1.2, seed=seed + 1000 + k)
        sets.append(p)
    return sets


def _thermo(p, u, gamma=5.0 / 3.0, alpha=1.0, hfact=1.2):
    """pro2, cs, alpha, u of an ideal gas at internal energy u, with rho estimated from
    the initial h: rho = pmass (hfact/h)^3."""
    n = p.n
    rho = p["pmass"] * (hfact / p["h"]) ** 3
    uu = np.broadcast_to(np.asarray(u, dtype=np.float64), (n,))
    return np.ascontiguousarray(np.stack([(gamma - 1.0) * uu / rho, np.sqrt(gamma * (gamma - 1.0) * uu),
                                          np.full(n, alpha), uu]))


def served_requests(nreq: int = 96, nmin: float = 5e3, nmax: float = 2e6, pcont: float = 0.3, seed: int = 42,
                    only=None):
    """The served-stream request list: particle counts log-uniform in [nmin, nmax]
    (seeded), each new set drawn from the lattice-with-jiggle, periodic-uniform-box or
    Plummer generator; with probability pcont a request instead continues an earlier set
    by one step of dt = 0.1 min(h/c_s) over that set's initial h.

    Each entry is a dict: kind "new" with n and, when generated, the particle set p (x,
    y, z, h, vx, vy, vz, pmass, optional box), pos3 (3, n), vel3 (3, n), thermo4 (4, n)
    component-major and dt; or kind "cont" with "of" (the index of the set's first
    request) and, when its set is generated, dt.  With only (request indices), just the
    sets of those requests are generated (each the same as in the full stream)."""
    rng = np.random.default_rng(seed)
    out = []
    firsts = []
    for k in range(nreq):
        if firsts and rng.uniform() < pcont:
            out.append({"kind": "cont", "of": int(rng.choice(firsts))})
            continue
        n = int(np.rint(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        g = int(rng.integers(3))
        out.append({"kind": "new", "n": n, "gen_id": g, "seed": seed + 7919 * (k + 1)})
        firsts.append(k)
    keep = set(range(nreq)) if only is None else set(int(k) for k in only)
    for k, e in enumerate(out):
        if e["kind"] != "new" or k not in keep:
            continue
        n, g, s = e["n"], e["gen_id"], e["seed"]
        if g == 0:
            npx = max(4, int(round((n / 1.403) ** (1.0 / 3.0))))
            p = lattice100_workload(npx, seed=s)
            th = np.ascontiguousarray(np.stack([p["pro2"], p["cs"], p["alpha"], p["u"]]))
            gen = f"lattice {npx} + jiggle"
        elif g == 1:
            p = uniform_box(n, hfac=1.2, hlo=0.8, hhi=1.2, seed=s)
            p["box"] = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
            p["vx"], p["vy"], p["vz"] = (gaussian(n, 0.0, 0.1, s + a) for a in (1, 2, 3))
            th = _thermo(p, 1.0)
            gen = "periodic uniform box"
        else:
            p = plummer(n, rmax=20.0, hfact=1.2, lnsigma=0.3, vfrac=0.5, seed=s)
            th = _thermo(p, 0.05)
            gen = "Plummer"
        e.update({"p": p, "gen": gen, "n": p.n, "dt": 0.1 * float(np.min(p["h"] / th[1])),
                  "pos3": np.ascontiguousarray(np.stack([p["x"], p["y"], p["z"]])),
                  "vel3": np.ascontiguousarray(np.stack([p["vx"], p["vy"], p["vz"]])),
                  "thermo4": th})
    for e in out:
        if e["kind"] == "cont" and "dt" in out[e["of"]]:
            e["dt"] = out[e["of"]]["dt"]
    return out
