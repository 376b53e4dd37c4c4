"""ctypes front end of the CPU oracle (oracle/sph_oracle.cpp).

Test infrastructure only: the parity checker for the CUDA library and the timed CPU
baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use it.
Parity status is stated at the top of sph_oracle.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libsph_oracle.so")

_DT = {0: np.float64, 1: np.int32, 2: np.uint32, 3: np.uint64, 4: np.int64}
_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with the committed Makefile (g++ + OpenMP)."""
    if force or not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB)
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_create.restype = P
        L.orc_create.argtypes = [I]
        L.orc_destroy.argtypes = [P]
        L.orc_set_threads.argtypes = [I]
        L.orc_max_threads.restype = I
        L.orc_density.restype = I
        L.orc_density.argtypes = [P, I, D, I, P, D, D, I, I, P, P, P, P, P, P]
        L.orc_force.restype = I
        L.orc_force.argtypes = [P, D, D, I, I, I, P, P]
        L.orc_scalar.restype = D
        L.orc_scalar.argtypes = [P, ctypes.c_char_p]
        L.orc_array.restype = ctypes.c_long
        L.orc_array.argtypes = [P, ctypes.c_char_p, P, ctypes.POINTER(I)]
        L.orc_hilbert_encode.restype = ctypes.c_uint64
        L.orc_hilbert_encode.argtypes = [ctypes.c_uint32] * 3 + [I]
        L.orc_hilbert_decode.argtypes = [ctypes.c_uint64, I, P]
        L.orc_kernel_eval.argtypes = [I, I, P, P, P]
        L.orc_kernel_consts.argtypes = [I, P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Oracle:
    """One oracle state: a restated GpuState on the CPU, for one kernel (cubic/quintic)."""

    def __init__(self, quintic: bool = False, threads: int = 0):
        self._L = lib()
        if threads:
            self._L.orc_set_threads(int(threads))
        self._s = self._L.orc_create(1 if quintic else 0)
        self.quintic = quintic

    def __del__(self):
        try:
            self._L.orc_destroy(self._s)
        except Exception:
            pass

    def density(self, x, y, z, h, pmass, *, periodic_box=None, tolh=1e-4, hfact=-1.0,
                max_iter=100, with_gradients=True, vel=None, acc=None) -> int:
        """Tree + Newton-Raphson density solve (+ gradient sweep). Returns the status:
        0 ok, 1 unconverged, 2 periodic support reaches half the box."""
        x, y, z, h = (_f64(a) for a in (x, y, z, h))
        n = x.size
        box = _f64(periodic_box) if periodic_box is not None else np.zeros(6)
        v3 = _f64(vel).reshape(-1) if vel is not None else None
        a3 = _f64(acc).reshape(-1) if acc is not None else None
        self._keep = (x, y, z, h, box, v3, a3)
        return self._L.orc_density(self._s, n, float(pmass), 1 if periodic_box is not None else 0,
                                   _ptr(box), float(tolh), float(hfact), int(max_iter),
                                   1 if with_gradients else 0, _ptr(x), _ptr(y), _ptr(z), _ptr(h),
                                   _ptr(v3), _ptr(a3))

    def force(self, thermo4, *, beta=2.0, alphau=0.0, disc=0, pdv=1, shock=1, vel=None) -> int:
        """Force pass on the last density solve's tree.  thermo4 = (pro2, cs, alpha, u)
        component-major in the caller's order; vel likewise (None: the solve's)."""
        t = _f64(thermo4).reshape(-1)
        v = _f64(vel).reshape(-1) if vel is not None else None
        self._keep2 = (t, v)
        return self._L.orc_force(self._s, float(beta), float(alphau), int(disc), int(pdv),
                                 int(shock), _ptr(t), _ptr(v))

    def scalar(self, name: str) -> float:
        return self._L.orc_scalar(self._s, name.encode())

    def array(self, name: str) -> np.ndarray:
        dt = ctypes.c_int(0)
        n = self._L.orc_array(self._s, name.encode(), None, ctypes.byref(dt))
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=_DT[dt.value])
        self._L.orc_array(self._s, name.encode(), _ptr(out), ctypes.byref(dt))
        return out

    def unsorted(self, name: str) -> np.ndarray:
        """A per-particle sorted array scattered back to the caller's order."""
        a = self.array(name)
        out = np.empty_like(a)
        out[self.array("order")] = a
        return out


def hilbert_encode(ix, iy, iz, bits=21) -> int:
    return int(lib().orc_hilbert_encode(int(ix), int(iy), int(iz), int(bits)))


def hilbert_decode(key, bits=21):
    out = np.zeros(3, dtype=np.uint32)
    lib().orc_hilbert_decode(int(key), int(bits), out.ctypes.data)
    return tuple(int(v) for v in out)


def kernel_eval(q, quintic=False):
    q = _f64(q)
    w = np.empty_like(q)
    dw = np.empty_like(q)
    lib().orc_kernel_eval(1 if quintic else 0, q.size, _ptr(q), _ptr(w), _ptr(dw))
    return w, dw


def kernel_consts(quintic=False):
    out = np.zeros(4)
    lib().orc_kernel_consts(1 if quintic else 0, out.ctypes.data)
    return out


def max_threads() -> int:
    return int(lib().orc_max_threads())
