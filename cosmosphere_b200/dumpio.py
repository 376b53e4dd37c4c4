"""Particle files in the reference's Fortran unformatted sequential layout, and its h.txt.

A file holds three records, each wrapped in 4-byte length markers before and after the
payload (the layout Fortran's sequential unformatted WRITE produces):

    [int32 4]  ngas (int32)                 [int32 4]
    [int32 8]  pmass (float64)              [int32 8]
    [int32 L]  xyzh(4, ngas) (float64)      [int32 L]     L = 32 ngas

xyzh is column-major, so the file interleaves x1 y1 z1 h1 x2 y2 ...  Reading checks every
marker as the reference's reader does (include/io.hpp:32-127) and raises ValueError on a
mismatch or a short file.  write_h writes one smoothing length per line in "%.15e" (the
reference's h.txt, include/io.hpp:130-139).  Host-only.
"""
from __future__ import annotations

import os
import struct

import numpy as np

from .inputs import Particles


def _record(f, nbytes: int, what: str) -> bytes:
    head = f.read(4)
    if len(head) != 4:
        raise ValueError(f"{what}: file ends before the record start marker")
    (before,) = struct.unpack("<i", head)
    if before != nbytes:
        raise ValueError(f"{what}: record start marker {before}, expected {nbytes}")
    body = f.read(nbytes)
    if len(body) != nbytes:
        raise ValueError(f"{what}: file ends inside the record payload")
    tail = f.read(4)
    if len(tail) != 4:
        raise ValueError(f"{what}: file ends before the record end marker")
    (after,) = struct.unpack("<i", tail)
    if after != before:
        raise ValueError(f"{what}: record end marker {after} differs from the start marker {before}")
    return body


def read_particles(path: str | os.PathLike) -> Particles:
    """ngas, pmass and x, y, z, h (float64 arrays) of a particle file."""
    with open(path, "rb") as f:
        (ngas,) = struct.unpack("<i", _record(f, 4, "ngas"))
        if ngas < 0:
            raise ValueError(f"ngas: negative particle count {ngas}")
        (pmass,) = struct.unpack("<d", _record(f, 8, "pmass"))
        xyzh = np.frombuffer(_record(f, 32 * ngas, "xyzh"), dtype="<f8").reshape(ngas, 4)
    return Particles(x=np.ascontiguousarray(xyzh[:, 0]), y=np.ascontiguousarray(xyzh[:, 1]),
                     z=np.ascontiguousarray(xyzh[:, 2]), h=np.ascontiguousarray(xyzh[:, 3]), pmass=float(pmass))


def write_particles(path: str | os.PathLike, x, y, z, h, pmass: float) -> None:
    """Write x, y, z, h (ngas each) and pmass as a particle file."""
    x, y, z, h = (np.asarray(a, dtype="<f8").ravel() for a in (x, y, z, h))
    n = x.size
    if not (y.size == z.size == h.size == n):
        raise ValueError("x, y, z and h must have the same length")
    if 32 * n > 0x7FFFFFFF:
        raise ValueError(f"{n} particles exceed a 32-bit record length")
    xyzh = np.stack([x, y, z, h], axis=1)
    with open(path, "wb") as f:
        for payload in (struct.pack("<i", n), struct.pack("<d", float(pmass)), xyzh.tobytes()):
            marker = struct.pack("<i", len(payload))
            f.write(marker)
            f.write(payload)
            f.write(marker)


def write_h(path: str | os.PathLike, h) -> None:
    """One smoothing length per line, "%.15e"."""
    with open(path, "w") as f:
        for v in np.asarray(h, dtype=np.float64).ravel():
            f.write("%.15e\n" % v)
