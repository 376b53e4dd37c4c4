"""The C-ABI library without a GPU: it loads, exports every symbol the headers declare,
and its checks that run before any CUDA call behave as the reference's."""
import os
import re
import subprocess
import sys

import pytest

from cosmosphere_b200 import capi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(REPO, "include", "cosmosphere.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cosmo_\w+|densityiterate_gpu_c|force_gpu_c)\s*\(", txt)))


@pytest.mark.parametrize("quintic", [False, True])
def test_library_exports_every_declared_symbol(quintic):
    L = capi.load(quintic)
    names = _declared()
    assert "densityiterate_gpu_c" in names and "cosmo_download" in names
    for name in names:
        assert hasattr(L, name), name


def test_exports_list_matches_header():
    assert sorted(capi.EXPORTS) == _declared()


def test_slot_table_and_kernel_radius():
    c = capi.Cosmo()
    assert [c.slot_ncomp(s) for s in range(0, 10)] == [0, 3, 1, 3, 3, 2, 3, 4, 6, 0]
    assert c.kernel_radius() == 2.0
    assert capi.Cosmo(quintic=True).kernel_radius() == 3.0


def test_static_archive_builds(tmp_path):
    # the archive Phantom links (-lcosmoSPHere)
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "cosmosphere_b200"), "static"], check=True)
    assert os.path.exists(os.path.join(REPO, "cosmosphere_b200", "lib", "libcosmoSPHere.a"))


def _child(code):
    return subprocess.run([sys.executable, "-c", "import sys; sys.path.insert(0, %r)\n" % REPO + code],
                          capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("call,msg", [
    ("c.upload(capi.POS, np.zeros(30), 10)", "FATAL: cosmo_upload(slot=1) with n=10 but the device arrays are sized for 0"),
    ("c.download(capi.HSML, 10)", "FATAL: cosmo_download(slot=2) with n=10 but the device arrays are sized for 0"),
    ("c.density(10, 0.1)", "FATAL: densityiterate_gpu_c called with n=10 but the device arrays are sized for 0"),
    ("c.force(10, 0.1)", "FATAL: force_gpu_c called with n=10 but the device arrays are sized for 0"),
])
def test_fatal_before_any_device_work(call, msg):
    r = _child("import numpy as np\nfrom cosmosphere_b200 import capi\nc = capi.Cosmo()\n" + call)
    assert r.returncode != 0
    assert msg in r.stderr


# Field keys of the reference's stderr lines, in print order: COSMO_STATS
# (src/dens_c_api.cu:113-122), COSMO_FORCE (src/force_c_api.cu:74-79) and COSMO_MEM
# (src/dens_c_api.cu:95-97).
REF_KEYS = {
    0: ["n", "leaves", "iters", "vecin", "upload", "bbox", "keysort", "tree", "nodes", "jbuild", "nrkern",
        "gjbuild", "gradkern", "download", "gpusum", "solve", "unaccounted", "total"],
    1: ["n", "leaves", "upsweep", "jbuild", "upload", "prep", "kernel", "download", "gpusum", "wall",
        "unaccounted"],
    2: ["n", "device_used", "host_peak"],
}
REF_HEAD = {0: "COSMO_STATS", 1: "COSMO_FORCE", 2: "COSMO_MEM"}


@pytest.mark.parametrize("which", [0, 1, 2])
def test_stats_lines_have_the_reference_fields(which):
    """Each statistics line carries the reference's keys in the reference's order, with
    two decimals for times, integers for counts, and the '|' group separators."""
    c = capi.Cosmo()
    nvals = {0: 18, 1: 11, 2: 5}[which]
    vals = [1403000.0, 40000.0, 6.0] + [1.234 + k for k in range(nvals - 3)]
    line = c.stats_line(which, vals)
    assert line.startswith(REF_HEAD[which] + " ") and line.endswith("\n")
    keys = re.findall(r"(\w+)=", line)
    assert keys == REF_KEYS[which]
    assert "n=1403000 " in line
    if which == 0:
        assert line.count(" | ") == 2 and "leaves=40000 iters=6 | vecin=1.23 upload=2.23" in line
        assert line.rstrip().endswith("total=15.23")
    elif which == 1:
        assert line.count(" | ") == 2 and "leaves=40000 | upsweep=6.00 jbuild=1.23 upload=2.23" in line
    else:
        assert re.fullmatch(r"COSMO_MEM n=\d+ device_used=\d+\.\d\d GB of \d+\.\d\d GB \(\d+ bytes/particle\) "
                            r"host_peak=\d+\.\d\d GB\n", line)


def test_wait_limit_setting_round_trips():
    """The bounded-wait limit is a host setting (no device work to set it)."""
    c = capi.Cosmo()
    old = c.wait_limit()
    assert old > 0
    c.set_wait_limit(12345)
    assert c.wait_limit() == 12345
    c.set_wait_limit(0)                 # restores the default
    assert c.wait_limit() == 1_000_000_000
    c.set_wait_limit(old)
