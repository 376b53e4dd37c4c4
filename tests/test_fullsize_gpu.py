"""Parity at the benchmark's full sizes: the lattice-100 workload (1,403,000 particles) and
the Plummer workload (2,000,000 particles, quintic, log-normal h) against the CPU oracle,
bit for bit on every structure and field, run as a stepping caller would -- the solve
repeated, so the Newton loop runs as a graph -- and the graph-run loop equal to the host
loop on the same inputs."""
import numpy as np
import pytest

from cosmosphere_b200 import capi, inputs
from oracle import oracle as O
from test_parity_gpu import _thermo, _vel_acc, check_all

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(900, method="thread")]


def solve(p, quintic, hfact, repeats=1):
    n = p.n
    v, a = _vel_acc(p)
    c = capi.Cosmo(quintic)
    for _ in range(repeats):
        c.arrays_init(n)
        c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
        c.upload(capi.HSML, p["h"])
        c.upload(capi.VEL, v)
        c.upload(capi.ACCEL, a)
        c.density(n, p["pmass"], hfact=hfact)
        c.upload(capi.THERMO, _thermo(p, hfact), sorted_=True)
        c.force(n, p["pmass"], beta=2.0, alphau=0.1)
    return c, v, a


def oracle_pair(p, quintic, hfact, v, a):
    o = O.Oracle(quintic=quintic)
    assert o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], hfact=hfact, vel=v, acc=a) == 0
    assert o.force(_thermo(p, hfact), beta=2.0, alphau=0.1) == 0
    return o


@pytest.mark.parametrize("case", ["lattice100", "plummer2m"])
def test_full_size_matches_oracle(case):
    if case == "lattice100":
        p, quintic, hfact = inputs.lattice100_workload(100), False, 1.2
    else:
        p, quintic, hfact = inputs.plummer(2000000, rmax=20.0, hfact=1.0, lnsigma=0.3, vfrac=0.5, seed=42), True, 1.0
    c, v, a = solve(p, quintic, hfact, repeats=3)
    assert c.scalar("loopGraph") == 1
    o = oracle_pair(p, quintic, hfact, v, a)
    check_all(c, o)


def test_full_size_graph_loop_equals_host_loop():
    p = inputs.lattice100_workload(100)
    c, _, _ = solve(p, False, 1.2, repeats=3)
    assert c.scalar("loopGraph") == 1
    g = {k: c.array(k).copy() for k in ("h", "rho", "gradh", "divv", "xi", "ddivvdt", "fx", "fy", "fz", "f4",
                                         "vsigmax", "divvF")}
    try:
        assert c.set_option("newton_graph", 0) == 0
        c, _, _ = solve(p, False, 1.2)
        assert c.scalar("loopGraph") == 0
        for k, vg in g.items():
            np.testing.assert_array_equal(c.array(k), vg, err_msg=k)
    finally:
        c.set_option("newton_graph", 1)
