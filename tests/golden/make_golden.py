"""Regenerate the golden fixtures in this directory from the reference's own code.

Run in a container that has the reference checkout, given as the argument or by the
environment variable COSMO_REFERENCE_DIR:
    python tests/golden/make_golden.py [REF]
It compiles, where they lie, the reference's include/kernel.hpp (both kernels) and its
standalone driver src/main.cu (against a recording stub of the C-ABI), through
oracle/Makefile's `ref` target, then records:
  ref_kernel.npz            W(q), dW/dq of the reference's M4 and M6 kernels on a q grid,
                            and their constants (radkernel, radk2, cnormk, hfact_default)
  ref_driver_lattice8.npz   what the reference driver uploads for `lattice 8`, with and
                            without its jiggle: n, pmass, x, y, z, h
  ref_io.npz                a particle file written by cosmosphere_b200.dumpio (its bytes),
                            what the reference's reader (include/io.hpp) parses from it, and
                            the reference's h.txt text for the same h
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
ORACLE = os.path.join(REPO, "oracle")


def main(ref=None):
    ref = ref or os.environ.get("COSMO_REFERENCE_DIR")
    if not ref:
        sys.exit("give the reference checkout as the argument or in COSMO_REFERENCE_DIR")
    subprocess.run(["make", "-s", "-C", ORACLE, "ref", f"REF={ref}"], check=True)
    q = np.linspace(0.0, 3.2, 2049)
    out = {"q": q}
    for name in ("cubic", "quintic"):
        L = ctypes.CDLL(os.path.join(ORACLE, "_ref", f"libref_kernel_{name}.so"))
        w, dw, c = np.empty_like(q), np.empty_like(q), np.empty(4)
        L.ref_kernel_eval(ctypes.c_int(q.size), q.ctypes.data_as(ctypes.c_void_p),
                          w.ctypes.data_as(ctypes.c_void_p), dw.ctypes.data_as(ctypes.c_void_p))
        L.ref_kernel_consts(c.ctypes.data_as(ctypes.c_void_p))
        out[f"{name}_w"], out[f"{name}_dw"], out[f"{name}_consts"] = w, dw, c
    np.savez(os.path.join(HERE, "ref_kernel.npz"), **out)

    drv = os.path.join(ORACLE, "_ref", "ref_driver_capture")
    rec = {}
    for tag, extra in (("plain", []), ("jiggle", ["jiggle"])):
        cap = os.path.join(ORACLE, "_ref", f"capture_{tag}.bin")
        env = dict(os.environ, COSMO_CAPTURE=cap)
        subprocess.run([drv, "lattice", "8", "no_output"] + extra, check=True, env=env,
                       stdout=subprocess.DEVNULL)
        raw = np.fromfile(cap, dtype=np.float64)
        n = int(raw[0])
        rec[f"{tag}_n"] = n
        rec[f"{tag}_pmass"] = raw[1]
        pos = raw[2:2 + 3 * n]
        rec[f"{tag}_x"], rec[f"{tag}_y"], rec[f"{tag}_z"] = pos[:n], pos[n:2 * n], pos[2 * n:]
        rec[f"{tag}_h"] = raw[2 + 3 * n:2 + 4 * n]
    np.savez(os.path.join(HERE, "ref_driver_lattice8.npz"), **rec)

    sys.path.insert(0, REPO)
    from cosmosphere_b200 import dumpio, inputs
    p = inputs.lattice(5)
    inputs.jiggle_ref(p["h"], 42)
    fpath = os.path.join(ORACLE, "_ref", "io_case.dat")
    dumpio.write_particles(fpath, p["x"], p["y"], p["z"], p["h"], p["pmass"])
    L = ctypes.CDLL(os.path.join(ORACLE, "_ref", "libref_io.so"))
    n, pm, err = ctypes.c_int(0), ctypes.c_double(0), ctypes.create_string_buffer(256)
    assert L.ref_read_particles(fpath.encode(), ctypes.byref(n), ctypes.byref(pm), None, err, 256) == 0, err.value
    xyzh = np.empty(4 * n.value)
    L.ref_read_particles(fpath.encode(), ctypes.byref(n), ctypes.byref(pm), xyzh.ctypes.data_as(ctypes.c_void_p),
                         err, 256)
    hpath = os.path.join(ORACLE, "_ref", "io_case_h.txt")
    h = np.ascontiguousarray(xyzh[3 * n.value:])
    assert L.ref_write_h(hpath.encode(), n, h.ctypes.data_as(ctypes.c_void_p)) == 0
    with open(fpath, "rb") as f:
        fbytes = np.frombuffer(f.read(), dtype=np.uint8)
    with open(hpath, "rb") as f:
        htext = np.frombuffer(f.read(), dtype=np.uint8)
    np.savez(os.path.join(HERE, "ref_io.npz"), file_bytes=fbytes, n=n.value, pmass=pm.value,
             x=xyzh[:n.value], y=xyzh[n.value:2 * n.value], z=xyzh[2 * n.value:3 * n.value], h=h,
             h_txt=htext)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main(*sys.argv[1:])
