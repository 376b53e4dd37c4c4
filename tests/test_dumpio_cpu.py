"""Particle files in the reference's Fortran record layout (CPU only), pinned to the
reference's own reader and h.txt writer (include/io.hpp) through tests/golden/ref_io.npz:
the bytes of a file written here, what the reference parsed from them, and the text the
reference writes for the same h."""
import os
import struct

import numpy as np
import pytest

from cosmosphere_b200 import dumpio, inputs

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_io.npz"))


def test_reader_matches_the_reference_reader(tmp_path):
    f = tmp_path / "case.dat"
    f.write_bytes(GOLD["file_bytes"].tobytes())
    p = dumpio.read_particles(f)
    assert p.n == int(GOLD["n"])
    assert p["pmass"] == float(GOLD["pmass"])
    for k in "xyzh":
        np.testing.assert_array_equal(p[k], GOLD[k])


def test_writer_reproduces_the_file_bytes(tmp_path):
    f = tmp_path / "case.dat"
    dumpio.write_particles(f, GOLD["x"], GOLD["y"], GOLD["z"], GOLD["h"], float(GOLD["pmass"]))
    assert f.read_bytes() == GOLD["file_bytes"].tobytes()


def test_h_text_matches_the_reference_writer(tmp_path):
    f = tmp_path / "h.txt"
    dumpio.write_h(f, GOLD["h"])
    assert f.read_bytes() == GOLD["h_txt"].tobytes()


def test_round_trip(tmp_path):
    p = inputs.plummer(1234, seed=3)
    f = tmp_path / "p.dat"
    dumpio.write_particles(f, p["x"], p["y"], p["z"], p["h"], p["pmass"])
    q = dumpio.read_particles(f)
    for k in "xyzh":
        np.testing.assert_array_equal(p[k], q[k])
    assert q["pmass"] == p["pmass"]


@pytest.mark.parametrize("cut", ["short_marker", "short_payload", "bad_start", "bad_end"])
def test_malformed_files_raise(tmp_path, cut):
    good = GOLD["file_bytes"].tobytes()
    if cut == "short_marker":
        data = good[:2]
    elif cut == "short_payload":
        data = good[:len(good) - 40]
    elif cut == "bad_start":
        data = struct.pack("<i", 8) + good[4:]
    else:
        data = good[:-4] + struct.pack("<i", 7)
    f = tmp_path / "bad.dat"
    f.write_bytes(data)
    with pytest.raises(ValueError):
        dumpio.read_particles(f)
