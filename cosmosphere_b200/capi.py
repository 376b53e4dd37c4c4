"""ctypes binding of libcosmoSPHere's C-ABI (include/cosmosphere.h).

Every call goes to the CUDA library; nothing here computes.  The library aborts the
process with a "FATAL:" line on misuse, exactly as the reference's C-ABI does, so tests
of those paths run it in a child process.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

POS, HSML, VEL, ACCEL, DENS_OUT, GRAD_OUT, THERMO, FORCE_OUT = range(1, 9)
NCOMP = {POS: 3, HSML: 1, VEL: 3, ACCEL: 3, DENS_OUT: 2, GRAD_OUT: 3, THERMO: 4, FORCE_OUT: 6}

EXPORTS = [
    "cosmo_arrays_init", "cosmo_slot_ncomp", "cosmo_upload", "cosmo_upload_sorted", "cosmo_download",
    "cosmo_pin_host", "cosmo_unpin_host", "cosmo_kernel_radius", "densityiterate_gpu_c", "force_gpu_c",
    "cosmo_x_set_max_iter", "cosmo_x_density", "cosmo_x_sync", "cosmo_x_scalar", "cosmo_x_array",
    "cosmo_x_stats_line", "cosmo_x_set_option", "cosmo_x_set_wait_limit", "cosmo_x_get_wait_limit", "cosmo_x_wait_test",
    "cosmo_x_set_key_extent", "cosmo_x_refresh_h", "cosmo_x_set_frozen", "cosmo_batch_set_staging",
    "cosmo_x_set_device", "cosmo_x_mark", "cosmo_x_mark_elapsed", "cosmo_x_launches", "cosmo_x_fp64_peak",
    "cosmo_hilbert_order_noalloc", "cosmo_set_precision", "cosmo_get_precision",
    "cosmo_batch_init", "cosmo_batch_set_params", "cosmo_batch_set_bucket", "cosmo_batch_set_tuning",
    "cosmo_batch_upload",
    "cosmo_batch_density", "cosmo_batch_download", "cosmo_batch_scalar",
    "cosmo_serve_start", "cosmo_serve_submit", "cosmo_serve_continue", "cosmo_serve_wait",
    "cosmo_serve_request_stat", "cosmo_serve_release", "cosmo_serve_stat", "cosmo_serve_stop",
]

_DT = {0: np.float64, 1: np.int32, 2: np.uint32, 3: np.uint64, 4: np.int64}


def lib_path(quintic: bool = False) -> str:
    return os.path.join(LIBDIR, "libcosmoSPHere_quintic.so" if quintic else "libcosmoSPHere.so")


def _bind(L: ctypes.CDLL) -> ctypes.CDLL:
    I, D, P = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    L.cosmo_arrays_init.argtypes = [I]
    L.cosmo_slot_ncomp.argtypes = [I]
    L.cosmo_slot_ncomp.restype = I
    for f in (L.cosmo_upload, L.cosmo_upload_sorted, L.cosmo_download):
        f.argtypes = [I, P, I]
    L.cosmo_pin_host.argtypes = [P, ctypes.c_size_t]
    L.cosmo_unpin_host.argtypes = [P]
    L.cosmo_kernel_radius.restype = D
    L.densityiterate_gpu_c.argtypes = [I, D, I, P, D, D]
    L.force_gpu_c.argtypes = [I, D, D, D, I, I, I]
    L.cosmo_x_set_max_iter.argtypes = [I]
    L.cosmo_x_density.argtypes = [I, D, I, P, D, D, I, I]
    L.cosmo_x_density.restype = I
    L.cosmo_x_scalar.argtypes = [ctypes.c_char_p]
    L.cosmo_x_stats_line.argtypes = [I, P, ctypes.c_char_p, I]
    L.cosmo_x_stats_line.restype = I
    L.cosmo_x_set_option.argtypes = [ctypes.c_char_p, I]
    L.cosmo_x_set_option.restype = I
    L.cosmo_x_set_key_extent.argtypes = [ctypes.c_void_p]
    L.cosmo_x_refresh_h.restype = I
    L.cosmo_batch_set_staging.argtypes = [I]
    L.cosmo_x_set_frozen.argtypes = [ctypes.c_void_p, I]
    L.cosmo_x_set_frozen.restype = I
    L.cosmo_x_set_wait_limit.argtypes = [ctypes.c_longlong]
    L.cosmo_x_get_wait_limit.restype = ctypes.c_longlong
    L.cosmo_x_wait_test.argtypes = [I, I]
    L.cosmo_x_wait_test.restype = I
    L.cosmo_x_scalar.restype = D
    L.cosmo_x_array.argtypes = [ctypes.c_char_p, P, ctypes.POINTER(I)]
    L.cosmo_x_array.restype = ctypes.c_long
    L.cosmo_x_set_device.argtypes = [I]
    L.cosmo_x_mark.argtypes = [I]
    L.cosmo_x_mark_elapsed.argtypes = [I, I]
    L.cosmo_x_mark_elapsed.restype = D
    L.cosmo_x_launches.restype = ctypes.c_ulonglong
    L.cosmo_x_fp64_peak.restype = D
    L.cosmo_hilbert_order_noalloc.argtypes = [I, P, P, P, P, I, P, P, P]
    L.cosmo_hilbert_order_noalloc.restype = I
    L.cosmo_set_precision.argtypes = [I]
    L.cosmo_get_precision.restype = I
    L.cosmo_batch_init.argtypes = [I, P]
    L.cosmo_batch_init.restype = I
    L.cosmo_batch_set_params.argtypes = [P, P, P]
    L.cosmo_batch_set_bucket.argtypes = [P]
    L.cosmo_batch_set_tuning.argtypes = [P, P, P, P]
    L.cosmo_batch_set_tuning.restype = I
    L.cosmo_batch_upload.argtypes = [P, P, P, P]
    L.cosmo_batch_density.argtypes = [D, D, I, I]
    L.cosmo_batch_density.restype = I
    L.cosmo_batch_download.argtypes = [P, P, P]
    L.cosmo_batch_scalar.argtypes = [ctypes.c_char_p]
    L.cosmo_batch_scalar.restype = D
    LNG = ctypes.c_long
    L.cosmo_serve_start.argtypes = [I, D]
    L.cosmo_serve_start.restype = I
    L.cosmo_serve_submit.argtypes = [I, D, I, P, D, D, P, P, P, P, D, D, I]
    L.cosmo_serve_submit.restype = LNG
    L.cosmo_serve_continue.argtypes = [LNG, D, P, I]
    L.cosmo_serve_continue.restype = LNG
    L.cosmo_serve_wait.argtypes = [LNG, P, P, P, P]
    L.cosmo_serve_wait.restype = I
    L.cosmo_serve_request_stat.argtypes = [LNG, ctypes.c_char_p]
    L.cosmo_serve_request_stat.restype = D
    L.cosmo_serve_release.argtypes = [LNG]
    L.cosmo_serve_release.restype = I
    L.cosmo_serve_stat.argtypes = [ctypes.c_char_p]
    L.cosmo_serve_stat.restype = D
    L.cosmo_serve_stop.restype = I
    return L


_libs: dict = {}


def load(quintic: bool = False) -> ctypes.CDLL:
    """Load the CUDA library; raises if it has not been built (no fallback)."""
    key = bool(quintic)
    if key not in _libs:
        path = lib_path(quintic)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with __graft_entry__.build() "
                               "(make -C cosmosphere_b200); there is no CPU fallback")
        _libs[key] = _bind(ctypes.CDLL(path))
    return _libs[key]


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Cosmo:
    """The C-ABI, one call per method; arrays are numpy float64, slots component-major."""

    def __init__(self, quintic: bool = False):
        self.L = load(quintic)
        self.quintic = quintic

    def arrays_init(self, n: int):
        self.L.cosmo_arrays_init(int(n))

    def slot_ncomp(self, slot: int) -> int:
        return int(self.L.cosmo_slot_ncomp(int(slot)))

    def upload(self, slot: int, data, n: int | None = None, sorted_: bool = False):
        a = _c(data).reshape(-1)
        n = a.size // NCOMP[slot] if n is None else n
        f = self.L.cosmo_upload_sorted if sorted_ else self.L.cosmo_upload
        f(int(slot), a.ctypes.data, int(n))

    def download(self, slot: int, n: int, out=None) -> np.ndarray:
        nc = NCOMP[slot]
        if out is None:
            out = np.empty((nc, n), dtype=np.float64)
        self.L.cosmo_download(int(slot), out.ctypes.data, int(n))
        return out

    def density(self, n, pmass, *, periodic_box=None, tolh=1e-4, hfact=-1.0):
        box = _c(periodic_box if periodic_box is not None else np.zeros(6))
        self.L.densityiterate_gpu_c(int(n), float(pmass), 1 if periodic_box is not None else 0,
                                    box.ctypes.data, float(tolh), float(hfact))

    def density_status(self, n, pmass, *, periodic_box=None, tolh=1e-4, hfact=-1.0, max_iter=0,
                       with_gradients=True) -> int:
        box = _c(periodic_box if periodic_box is not None else np.zeros(6))
        return int(self.L.cosmo_x_density(int(n), float(pmass), 1 if periodic_box is not None else 0,
                                          box.ctypes.data, float(tolh), float(hfact), int(max_iter),
                                          1 if with_gradients else 0))

    def force(self, n, pmass, *, beta=2.0, alphau=0.0, disc=0, pdv=1, shock=1):
        self.L.force_gpu_c(int(n), float(pmass), float(beta), float(alphau), int(disc), int(pdv), int(shock))

    def stats_line(self, which: int, values) -> str:
        """One statistics line (0 COSMO_STATS, 1 COSMO_FORCE, 2 COSMO_MEM) formatted by the
        library from the given values, as its entry points print it."""
        v = _c(values)
        buf = ctypes.create_string_buffer(1024)
        n = self.L.cosmo_x_stats_line(which, v.ctypes.data, buf, len(buf))
        if n < 0:
            raise ValueError(which)
        return buf.value.decode()

    def set_option(self, name: str, value: int) -> int:
        return int(self.L.cosmo_x_set_option(name.encode(), int(value)))

    def set_key_extent(self, ext6=None):
        """Open boundaries: the extents (xmin, xmax, ymin, ymax, zmin, zmax) the solves' box
        and keys are made from; None returns to the uploaded particles' own."""
        if ext6 is None:
            self.L.cosmo_x_set_key_extent(None)
        else:
            self._ext = np.ascontiguousarray(np.asarray(ext6, dtype=np.float64))
            self.L.cosmo_x_set_key_extent(self._ext.ctypes.data)

    def refresh_h(self) -> int:
        return int(self.L.cosmo_x_refresh_h())

    def set_frozen(self, mask=None) -> int:
        """Particles the next solves take as neighbours only (caller order); None clears."""
        if mask is None:
            return int(self.L.cosmo_x_set_frozen(None, 0))
        m = np.ascontiguousarray(np.asarray(mask, dtype=np.int32))
        return int(self.L.cosmo_x_set_frozen(m.ctypes.data, int(m.size)))

    def set_wait_limit(self, ns: int):
        self.L.cosmo_x_set_wait_limit(int(ns))

    def wait_limit(self) -> int:
        return int(self.L.cosmo_x_get_wait_limit())

    def wait_test(self, kind: int, fatal: bool = False) -> int:
        return int(self.L.cosmo_x_wait_test(int(kind), 1 if fatal else 0))

    def kernel_radius(self) -> float:
        return float(self.L.cosmo_kernel_radius())

    def pin(self, a: np.ndarray):
        self.L.cosmo_pin_host(a.ctypes.data, a.nbytes)

    def unpin(self, a: np.ndarray):
        self.L.cosmo_unpin_host(a.ctypes.data)

    def set_max_iter(self, m: int):
        self.L.cosmo_x_set_max_iter(int(m))

    def sync(self):
        self.L.cosmo_x_sync()

    def hilbert_order_noalloc(self, n: int, d_x: int, d_y: int, d_z: int, d_h: int, d_keys: int, d_order: int,
                              periodic_box=None) -> int:
        """The allocation-free keys + sort entry point; all pointers are device addresses."""
        box = _c(periodic_box if periodic_box is not None else np.zeros(6))
        return int(self.L.cosmo_hilbert_order_noalloc(int(n), d_x, d_y, d_z, d_h,
                                                      1 if periodic_box is not None else 0, box.ctypes.data,
                                                      d_keys, d_order))

    def set_precision(self, mixed: bool):
        self.L.cosmo_set_precision(1 if mixed else 0)

    def precision(self) -> int:
        return int(self.L.cosmo_get_precision())

    def set_device(self, dev: int):
        self.L.cosmo_x_set_device(int(dev))

    def mark(self, i: int):
        self.L.cosmo_x_mark(int(i))

    def elapsed(self, a: int, b: int) -> float:
        return float(self.L.cosmo_x_mark_elapsed(int(a), int(b)))

    def launches(self) -> int:
        return int(self.L.cosmo_x_launches())

    def fp64_peak_tflops(self) -> float:
        return float(self.L.cosmo_x_fp64_peak())

    def scalar(self, name: str) -> float:
        return float(self.L.cosmo_x_scalar(name.encode()))

    def array(self, name: str) -> np.ndarray:
        dt = ctypes.c_int(0)
        n = self.L.cosmo_x_array(name.encode(), None, ctypes.byref(dt))
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=_DT[dt.value])
        self.L.cosmo_x_array(name.encode(), out.ctypes.data if n else None, ctypes.byref(dt))
        return out


class Batch:
    """The batched form: many independent sets, one segmented sort and forest, one
    density launch per Newton iteration for all of them."""

    def __init__(self, sets, quintic: bool = False, bucket=None):
        """sets: list of dicts with x, y, z, h, pmass and optional box (periodic)."""
        self.L = load(quintic)
        self.sizes = [int(np.asarray(s["x"]).size) for s in sets]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int32)
        self.n = int(self.offsets[-1])
        rc = self.L.cosmo_batch_init(len(sets), self.offsets.ctypes.data)
        if rc != 0:
            raise ValueError("cosmo_batch_init rejected the set sizes")
        pm = np.array([s["pmass"] for s in sets], dtype=np.float64)
        per = np.array([1 if s.get("box") is not None else 0 for s in sets], dtype=np.int32)
        box = np.array([s["box"] if s.get("box") is not None else [0.0] * 6 for s in sets], dtype=np.float64)
        self.L.cosmo_batch_set_params(pm.ctypes.data, per.ctypes.data, box.ctypes.data)
        if bucket is not None:
            b = np.ascontiguousarray(np.broadcast_to(np.asarray(bucket, dtype=np.int32), (len(sets),)))
            self.L.cosmo_batch_set_bucket(b.ctypes.data)
        self._keep = (pm, per, box)
        cat = lambda k: np.ascontiguousarray(np.concatenate([np.asarray(s[k], dtype=np.float64) for s in sets]))
        self.x, self.y, self.z, self.h = cat("x"), cat("y"), cat("z"), cat("h")

    def set_staging(self, on: bool):
        """The batched Newton kernel's j-stream feed: staged by bulk copies or direct."""
        self.L.cosmo_batch_set_staging(1 if on else 0)

    def set_tuning(self, bucket=None, list_margin=None, split_stream=None, split_work=None):
        """Per-set launch parameters (each a scalar or one value per set; None keeps it)."""
        ns = len(self.sizes)

        def arr(v, dt):
            return None if v is None else np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=dt), (ns,)))

        a = [arr(bucket, np.int32), arr(list_margin, np.float64), arr(split_stream, np.int32),
             arr(split_work, np.int32)]
        rc = self.L.cosmo_batch_set_tuning(*[x.ctypes.data if x is not None else None for x in a])
        if rc != 0:
            raise ValueError("cosmo_batch_set_tuning rejected a value")

    def upload(self):
        self.L.cosmo_batch_upload(self.x.ctypes.data, self.y.ctypes.data, self.z.ctypes.data, self.h.ctypes.data)

    def density(self, tolh=1e-4, hfact=-1.0, max_iter=100, graph=True, final_rho=False) -> int:
        flags = (1 if graph else 0) | (2 if final_rho else 0)
        return int(self.L.cosmo_batch_density(float(tolh), float(hfact), int(max_iter), flags))

    def download(self):
        h, rho, gh = (np.empty(self.n) for _ in range(3))
        self.L.cosmo_batch_download(h.ctypes.data, rho.ctypes.data, gh.ctypes.data)
        o = self.offsets
        split = lambda a: [a[o[k]:o[k + 1]] for k in range(len(self.sizes))]
        return split(h), split(rho), split(gh)

    def scalar(self, name: str) -> float:
        return float(self.L.cosmo_batch_scalar(name.encode()))


class Server:
    """The served form: continuous batching of density + force requests over worker
    slots, with device-resident sets and an HBM budget."""

    def __init__(self, slots: int = 4, budget_gb: float = 150.0, quintic: bool = False):
        self.L = load(quintic)
        if self.L.cosmo_serve_start(int(slots), float(budget_gb)) != 0:
            raise RuntimeError("cosmo_serve_start failed (already running?)")
        self.n = {}

    def submit(self, p, thermo, *, box=None, tolh=1e-4, hfact=-1.0, beta=2.0, alphau=0.0, keep=True) -> int:
        n = int(np.asarray(p["x"]).size)
        pos = np.ascontiguousarray(np.stack([p["x"], p["y"], p["z"]]), dtype=np.float64)
        h = np.ascontiguousarray(p["h"], dtype=np.float64)
        vel = (np.ascontiguousarray(np.stack([p["vx"], p["vy"], p["vz"]]), dtype=np.float64)
               if "vx" in p else None)
        th = np.ascontiguousarray(thermo, dtype=np.float64)
        b = _c(box if box is not None else np.zeros(6))
        rid = int(self.L.cosmo_serve_submit(n, float(p["pmass"]), 1 if box is not None else 0, b.ctypes.data,
                                            float(tolh), float(hfact), pos.ctypes.data, h.ctypes.data,
                                            vel.ctypes.data if vel is not None else None, th.ctypes.data,
                                            float(beta), float(alphau), 1 if keep else 0))
        if rid < 0:
            raise RuntimeError("submit rejected")
        self.n[rid] = n
        return rid

    def cont(self, set_id: int, dt: float, thermo=None, keep=True) -> int:
        th = np.ascontiguousarray(thermo, dtype=np.float64) if thermo is not None else None
        rid = int(self.L.cosmo_serve_continue(int(set_id), float(dt), th.ctypes.data if th is not None else None,
                                              1 if keep else 0))
        if rid < 0:
            raise RuntimeError("continue rejected: set not resident")
        self.n[rid] = self.n[set_id]
        return rid

    def wait(self, rid: int):
        n = self.n[rid]
        h, dens, grad, force = np.empty(n), np.empty((2, n)), np.empty((3, n)), np.empty((6, n))
        st = int(self.L.cosmo_serve_wait(int(rid), h.ctypes.data, dens.ctypes.data, grad.ctypes.data,
                                         force.ctypes.data))
        return st, {"h": h, "dens": dens, "grad": grad, "force": force}

    def stat(self, rid: int, name: str) -> float:
        return float(self.L.cosmo_serve_request_stat(int(rid), name.encode()))

    def server_stat(self, name: str) -> float:
        return float(self.L.cosmo_serve_stat(name.encode()))

    def release(self, set_id: int) -> int:
        return int(self.L.cosmo_serve_release(int(set_id)))

    def stop(self):
        self.L.cosmo_serve_stop()
