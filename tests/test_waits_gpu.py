"""Bounded device waits give up and report instead of hanging.

Every wait of the library on something another block or the copy engine completes -- the
radix sort's look-back on its predecessor tiles, the staging barriers of the bulk copies
-- polls under a time limit (cosmo_x_set_wait_limit).  These tests run waits that can
never be satisfied through the same code (cosmo_x_wait_test): a flag no block sets, and a
staging barrier armed for a bulk copy that is never issued.  No GPU faults or hangs: each
wait runs out after a few milliseconds, raises its bit in the device error word, and the
kernel returns; the library stays usable."""
import os
import subprocess
import sys
import time

import numpy as np
import pytest

from cosmosphere_b200 import capi, inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("kind,bit", [(0, 8), (1, 4)])
def test_unsatisfiable_wait_gives_up_with_its_error_bit(kind, bit):
    c = capi.Cosmo()
    old = c.wait_limit()
    c.set_wait_limit(2_000_000)        # 2 ms
    try:
        t0 = time.perf_counter()
        e = c.wait_test(kind)
        dt = time.perf_counter() - t0
    finally:
        c.set_wait_limit(old)
    assert e == bit
    assert dt < 5.0
    # the error word was cleared and the library still solves, bit for bit as the oracle
    p = inputs.lattice(10)
    n = p.n
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    c.density(n, p["pmass"])
    o = O.Oracle()
    assert o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], with_gradients=False) == 0
    np.testing.assert_array_equal(c.download(capi.HSML, n)[0], o.unsorted("h"))


def test_wait_timeout_is_reported_as_a_fatal_error():
    code = ("import sys; sys.path.insert(0, %r)\nfrom cosmosphere_b200 import capi\n"
            "c = capi.Cosmo(); c.set_wait_limit(1_000_000); c.wait_test(1, fatal=True)\n" % REPO)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode != 0
    assert "FATAL: cosmo_x_wait_test: device error 0x4 (staging wait timeout" in r.stderr
