"""Parity of the CUDA library, called through its C-ABI, with the CPU oracle on the same
seeded inputs.  The plain FP64 form is required to be bit-exact on everything: keys,
sort order, leaf tree, octree, node geometry, j-leaf lists, h, rho, gradh, the gradient
fields and the forces (the specification's bound for the FP64 fields is 1e-10 relative;
bit equality is the stronger property the library is built to hold)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from cosmosphere_b200 import capi, inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

TREE = ["keys", "order", "csTree", "counts", "layout", "prefixes", "childOffsets", "internalToLeaf",
        "levelRange", "leafToInternal", "centers", "sizes"]
FIELDS = ["x", "y", "z", "h", "rho", "gradh", "divv", "xi", "ddivvdt"]
FORCE = ["fx", "fy", "fz", "f4", "vsigmax", "divvF"]


def _vel_acc(p, seed=5):
    n = p.n
    if "vx" in p:
        v = np.stack([p["vx"], p["vy"], p["vz"]])
    else:
        v = np.stack([inputs.gaussian(n, 0, 0.1, seed + k) for k in range(3)])
    a = np.stack([inputs.gaussian(n, 0, 1.0, seed + 10 + k) for k in range(3)])
    return v, a


def _thermo(p, hfact):
    n = p.n
    if "pro2" in p:
        return np.stack([p["pro2"], p["cs"], p["alpha"], p["u"]])
    rho = p["pmass"] * (hfact / p["h"]) ** 3
    return np.stack([(2.0 / 3.0) / rho, np.full(n, np.sqrt(10.0 / 9.0)), np.full(n, 1.0), np.full(n, 1.0)])


def run_pair(p, *, quintic=False, box=None, force=True, tolh=1e-4, disc=0, beta=2.0, alphau=0.1):
    n = p.n
    hfact = 1.0 if quintic else 1.2
    v, a = _vel_acc(p)
    c = capi.Cosmo(quintic)
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    c.upload(capi.VEL, v)
    c.upload(capi.ACCEL, a)
    c.density(n, p["pmass"], periodic_box=box, tolh=tolh, hfact=hfact)
    o = O.Oracle(quintic=quintic)
    st = o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], periodic_box=box, tolh=tolh, hfact=hfact,
                   vel=v, acc=a)
    assert st == 0
    if force:
        th = _thermo(p, hfact)
        c.upload(capi.THERMO, th, sorted_=True)
        c.force(n, p["pmass"], beta=beta, alphau=alphau, disc=disc)
        assert o.force(th, beta=beta, alphau=alphau, disc=disc) == 0
    return c, o


def assert_same(c, o, names):
    for k in names:
        g, r = c.array(k), o.array(k)
        assert g.shape == r.shape, (k, g.shape, r.shape)
        np.testing.assert_array_equal(g, r, err_msg=k)


def assert_lists_same(c, o):
    assert_same(c, o, ["jcount", "jOffset", "jlist"])


def check_all(c, o, force=True):
    assert c.scalar("nAlive") == o.scalar("nAlive")
    assert c.scalar("nLeaves") == o.scalar("nLeaves")
    assert c.scalar("numNodes") == o.scalar("numNodes")
    assert c.scalar("itersRun") == o.scalar("itersRun")
    np.testing.assert_array_equal(c.array("activePerIter"), o.array("activePerIter"))
    assert_same(c, o, TREE)
    nA = int(o.scalar("nAlive"))
    np.testing.assert_array_equal(c.array("particleLeaf")[:nA], o.array("particleLeaf")[:nA])
    assert_same(c, o, FIELDS)
    if force:
        assert_same(c, o, FORCE + ["hmax_node"])
    assert_lists_same(c, o)                       # gather after density; symmetric after force
    assert c.scalar("pairsDensity") == o.scalar("pairsDensity")
    assert c.scalar("pairsGrad") == o.scalar("pairsGrad")
    if force:
        assert c.scalar("pairsForce") == o.scalar("pairsForce")


def test_lattice_jiggle_open():
    p = inputs.lattice(16)
    inputs.jiggle_ref(p["h"], 42)
    c, o = run_pair(p)
    check_all(c, o)


def test_lattice100_workload_small():
    p = inputs.lattice100_workload(20)
    c, o = run_pair(p)
    check_all(c, o)


@pytest.mark.parametrize("case", ["plummer_lognormal", "lattice_open"])
def test_density_only_incremental_lists(case):
    """Density without gradients: the Newton lists are rebuilt incrementally when an h
    outgrows its leaf's list (only outgrown or loosened leaves walk, the rest copy), the
    fill pass copies what the count pass kept (lists up to 512 entries) or walks again
    (longer lists), and the exact lists of the last iteration are rebuilt at the end.
    Iteration counts, active counts, h, rho and those final lists equal the oracle's."""
    if case == "plummer_lognormal":
        p = inputs.plummer(20000, lnsigma=0.5, seed=7)
    else:
        p = inputs.lattice(18)
        inputs.jiggle_frac(p["h"], 0.2, 0.5, 1.6, 3)
    n = p.n
    c = capi.Cosmo()
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    assert c.density_status(n, p["pmass"], with_gradients=False) == 0
    o = O.Oracle()
    assert o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], with_gradients=False) == 0
    assert c.scalar("itersRun") == o.scalar("itersRun")
    np.testing.assert_array_equal(c.array("activePerIter"), o.array("activePerIter"))
    assert_same(c, o, ["h", "rho", "gradh"])
    assert_lists_same(c, o)
    assert c.scalar("pairsDensity") == o.scalar("pairsDensity")
    if case == "plummer_lognormal":
        assert int(c.array("jcount").max()) > 512      # some lists take the walking fill


@pytest.mark.parametrize("overflow", [False, True])
def test_symmetric_row_overflow_takes_the_group_path(overflow):
    """Particles whose symmetric row would hold more than 128 entries (a compact core in
    a wide halo of large h) take the group path in the gradient sweep and the force pass;
    when no row overflows those passes skip the group path altogether.  Either way every
    field equals the oracle's."""
    if overflow:
        p = inputs.plummer(6000, lnsigma=0.9, seed=12)
    else:
        p = inputs.lattice(14)
        inputs.jiggle_ref(p["h"], 42)
    c, o = run_pair(p)
    assert c.scalar("rowOverflow") == (1.0 if overflow else 0.0)
    check_all(c, o)


@pytest.mark.parametrize("n", [33, 64, 65, 130])
def test_small_sets_around_one_leaf(n):
    """A set of one leaf, exactly one full leaf, one particle over (the root splits into
    eight) and two leaves' worth: every structure and field equals the oracle's."""
    rng = np.random.default_rng(n)
    x, y, z = rng.random((3, n))
    p = inputs.Particles(x=x, y=y, z=z, h=np.full(n, 1.2 * (1.0 / n) ** (1.0 / 3.0)), pmass=1.0 / n)
    c, o = run_pair(p)
    check_all(c, o)


def test_periodic_jittered_lattice():
    x, y, z = (np.asarray(v) for v in np.meshgrid(*(np.arange(12) / 12.0,) * 3, indexing="ij"))
    n = x.size
    rng = np.random.default_rng(11)
    p = inputs.Particles(x=(x.ravel() + rng.uniform(0, 0.02, n)) % 1.0, y=(y.ravel() + rng.uniform(0, 0.02, n)) % 1.0,
                         z=(z.ravel() + rng.uniform(0, 0.02, n)) % 1.0, h=np.full(n, 1.2 / 12), pmass=1.0 / n)
    inputs.jiggle_frac(p["h"], 0.05, 0.65, 1.35, 9)
    c, o = run_pair(p, box=[0.0, 1.0, 0.0, 1.0, 0.0, 1.0])
    check_all(c, o)


def test_quintic_plummer_lognormal():
    p = inputs.plummer(12000, lnsigma=0.3, seed=42)
    c, o = run_pair(p, quintic=True)
    check_all(c, o)


def test_disc_viscosity_and_partial_heating():
    p = inputs.lattice100_workload(12)
    c, o = run_pair(p, disc=1, alphau=0.5)
    check_all(c, o)
    th = _thermo(p, 1.2)
    c.upload(capi.THERMO, th, sorted_=True)
    c.force(p.n, p["pmass"], beta=2.0, alphau=0.5, disc=0, pdv=0, shock=1)
    o.force(th, beta=2.0, alphau=0.5, disc=0, pdv=0, shock=1)
    assert_same(c, o, FORCE)


def test_dead_particles():
    p = inputs.lattice(12)
    dead = np.arange(3, p.n, 41)
    p["h"][dead] = -1.0
    p["h"][7] = 0.0
    c, o = run_pair(p)
    check_all(c, o)
    n = p.n
    h = c.download(capi.HSML, n)[0]
    np.testing.assert_array_equal(h[dead], -1.0)
    f = c.download(capi.FORCE_OUT, n)
    assert np.all(f[:, dead] == 0.0)
    g = c.download(capi.GRAD_OUT, n)
    assert np.all(g[1, dead] == 1.0) and np.all(g[0, dead] == 0.0)


def test_c_abi_transfers_round_trip():
    p = inputs.lattice100_workload(14)
    c, o = run_pair(p)
    n = p.n
    pos = c.download(capi.POS, n)
    np.testing.assert_array_equal(pos, np.stack([p["x"], p["y"], p["z"]]))
    np.testing.assert_array_equal(c.download(capi.HSML, n)[0], o.unsorted("h"))
    d = c.download(capi.DENS_OUT, n)
    np.testing.assert_array_equal(d[0], o.unsorted("rho"))
    np.testing.assert_array_equal(d[1], o.unsorted("gradh"))
    g = c.download(capi.GRAD_OUT, n)
    for k, name in enumerate(("divv", "xi", "ddivvdt")):
        np.testing.assert_array_equal(g[k], o.unsorted(name))
    f = c.download(capi.FORCE_OUT, n)
    for k, name in enumerate(FORCE):
        np.testing.assert_array_equal(f[k], o.unsorted(name))
    # upload_sorted then download returns what was sent, in the caller's order
    v2 = np.stack([inputs.gaussian(n, 0, 1, 77 + k) for k in range(3)])
    c.upload(capi.VEL, v2, sorted_=True)
    np.testing.assert_array_equal(c.download(capi.VEL, n), v2)
    th = c.download(capi.THERMO, n)
    np.testing.assert_array_equal(th, _thermo(p, 1.2))


def test_pinned_host_buffers_and_repeat_solve():
    p = inputs.lattice100_workload(14)
    n = p.n
    c = capi.Cosmo()
    buf = np.ascontiguousarray(np.stack([p["x"], p["y"], p["z"]]))
    hb = p["h"].copy()
    c.pin(buf)
    c.pin(hb)
    c.arrays_init(n)
    outs = []
    for _ in range(2):
        c.upload(capi.POS, buf)
        c.upload(capi.HSML, hb)
        c.density(n, p["pmass"])
        outs.append(c.download(capi.DENS_OUT, n))
    c.unpin(buf)
    c.unpin(hb)
    np.testing.assert_array_equal(outs[0], outs[1])
    # force twice on the same tree: the symmetric list is cached, results identical
    th = _thermo(p, 1.2)
    c.upload(capi.THERMO, th, sorted_=True)
    c.force(n, p["pmass"])
    f1 = c.download(capi.FORCE_OUT, n)
    c.force(n, p["pmass"])
    np.testing.assert_array_equal(f1, c.download(capi.FORCE_OUT, n))


def test_resize_between_solves():
    for npx in (10, 14, 10):
        p = inputs.lattice(npx)
        c, o = run_pair(p, force=False)
        assert_same(c, o, ["h", "rho", "gradh"])


def test_lattice50_reference_driver_case():
    """The reference driver's `lattice 50` (173,850 particles, open boundaries)."""
    p = inputs.lattice(50)
    c, o = run_pair(p, force=True)
    check_all(c, o)


def test_lattice50_unit_periodic_box():
    """The same lattice in the unit periodic box [0, 1)^3 (the lattice is not fitted to
    the period, so the rows at the wrap are closer than the spacing), density + force."""
    p = inputs.lattice(50)
    c, o = run_pair(p, box=[0.0, 1.0, 0.0, 1.0, 0.0, 1.0], force=True)
    check_all(c, o)


def _child(code, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, "-c", "import sys; sys.path.insert(0, %r)\n" % REPO + code],
                          capture_output=True, text=True, timeout=300, env=e)


PRE = ("import numpy as np\nfrom cosmosphere_b200 import capi, inputs\n"
       "p = inputs.lattice(10); n = p.n; c = capi.Cosmo(); c.arrays_init(n)\n"
       "c.upload(capi.POS, np.stack([p['x'], p['y'], p['z']])); c.upload(capi.HSML, p['h'])\n")


def test_fatal_unconverged_within_cap():
    r = _child(PRE + "c.density(n, p['pmass'])\n", env={"COSMO_MAX_ITER": "1"})
    assert r.returncode != 0
    assert "FATAL: solveDensH: unconverged=" in r.stderr


def test_fatal_force_before_density():
    r = _child(PRE + "c.force(n, p['pmass'])\n")
    assert r.returncode != 0
    assert "FATAL: force_gpu_c called with no GPU density solve for this particle set" in r.stderr


def test_fatal_upload_sorted_before_density():
    r = _child(PRE + "c.upload(capi.THERMO, np.zeros(4 * n), n, sorted_=True)\n")
    assert r.returncode != 0
    assert "with no ordering: a density solve must have run first" in r.stderr


def test_fatal_periodic_support():
    code = ("import numpy as np\nfrom cosmosphere_b200 import capi\n"
            "g = (np.arange(3) + 0.5) / 3; X, Y, Z = np.meshgrid(g, g, g, indexing='ij')\n"
            "c = capi.Cosmo(); c.arrays_init(27)\n"
            "c.upload(capi.POS, np.stack([X.ravel(), Y.ravel(), Z.ravel()])); c.upload(capi.HSML, np.full(27, 0.4))\n"
            "c.density(27, 1 / 27, periodic_box=[0, 1, 0, 1, 0, 1])\n")
    r = _child(code)
    assert r.returncode != 0
    assert "reaches half the periodic box" in r.stderr


def test_reference_driver_runs_unchanged_on_this_library():
    """The reference's own standalone driver (src/main.cu, compiled from the reference by
    oracle/Makefile against libcosmoSPHere) runs on this library; its printed h and rho
    ranges match the oracle's for the same lattice and jiggle."""
    drv = os.path.join(REPO, "oracle", "_ref", "ref_driver_b200")
    if not os.path.exists(drv):
        pytest.skip("reference driver not built (needs the reference checkout at build time)")
    r = subprocess.run([drv, "lattice", "20", "no_output", "jiggle"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if "Output" in ln and "range" in ln]
    assert len(lines) == 4          # h and rho, for the flat and the warp-per-leaf call
    p = inputs.lattice(20)
    inputs.jiggle_ref(p["h"], 42)
    o = O.Oracle()
    assert o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], with_gradients=False) == 0
    h, rho = o.array("h"), o.array("rho")
    want_h = " Output h   range: [%.6e, %.6e]" % (h.min(), h.max())
    want_r = " Output rho range: [%.6e, %.6e]" % (rho.min(), rho.max())
    assert lines[0] == want_h and lines[2] == want_h
    assert lines[1] == want_r and lines[3] == want_r


def test_reference_driver_reads_a_particle_file(tmp_path):
    """A particle file written by cosmosphere_b200.dumpio, read by the reference's own
    driver (its include/io.hpp reader) and solved on this library, gives the h.txt that
    this library's solve of the same particles, written by dumpio.write_h, gives."""
    drv = os.path.join(REPO, "oracle", "_ref", "ref_driver_b200")
    if not os.path.exists(drv):
        pytest.skip("reference driver not built (needs the reference checkout at build time)")
    from cosmosphere_b200 import dumpio
    p = inputs.lattice(12)
    inputs.jiggle_ref(p["h"], 7)
    f = tmp_path / "lat12.dat"
    dumpio.write_particles(f, p["x"], p["y"], p["z"], p["h"], p["pmass"])
    out_ref = tmp_path / "h_ref.txt"
    r = subprocess.run([drv, str(f), str(out_ref)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    q = dumpio.read_particles(f)
    n = q.n
    c = capi.Cosmo()
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([q["x"], q["y"], q["z"]]))
    c.upload(capi.HSML, q["h"])
    c.density(n, q["pmass"])
    out_ours = tmp_path / "h_ours.txt"
    dumpio.write_h(out_ours, c.download(capi.HSML, n)[0])
    assert out_ours.read_bytes() == out_ref.read_bytes()


@pytest.mark.parametrize("option", ["staging", "sym_prefilter"])
def test_kernel_variants_keep_parity(option):
    """The bulk-copy staging of the Newton kernels' j-stream and the FP32-prefiltered
    symmetric row builder are variants of the same passes: with either switched on, every
    structure and field still equals the oracle's bit for bit (jiggled lattice, and a
    log-normal quintic Plummer sphere whose groups spread in h)."""
    for quintic in (False, True):
        c = capi.Cosmo(quintic)
        assert c.set_option(option, 1) == 0
        try:
            if quintic:
                p = inputs.plummer(12000, lnsigma=0.5, seed=21)
            else:
                p = inputs.lattice100_workload(16)
            cc, o = run_pair(p, quintic=quintic)
            check_all(cc, o)
        finally:
            c.set_option(option, 0)


def test_one_particle_cut_items_keep_parity():
    """With the leaf cut lowered so that nearly every leaf is cut into one-particle items
    (each scanning the tree for the cells on its own support sphere, and filtering its
    candidates by that sphere), every structure and field still equals the oracle's bit
    for bit: a log-normal quintic Plummer sphere, and the jiggled periodic lattice."""
    for quintic in (True, False):
        c = capi.Cosmo(quintic)
        assert c.set_option("split_stream", 64) == 0 and c.set_option("split_work", 32) == 0
        try:
            if quintic:
                p = inputs.plummer(12000, lnsigma=0.5, seed=23)
                cc, o = run_pair(p, quintic=True)
            else:
                x, y, z = (np.asarray(v).ravel() for v in np.meshgrid(*(np.arange(12) / 12.0,) * 3, indexing="ij"))
                n = x.size
                rng = np.random.default_rng(5)
                p = inputs.Particles(x=(x + rng.uniform(0, 0.02, n)) % 1.0, y=(y + rng.uniform(0, 0.02, n)) % 1.0,
                                     z=(z + rng.uniform(0, 0.02, n)) % 1.0, h=np.full(n, 1.2 / 12), pmass=1.0 / n)
                inputs.jiggle_frac(p["h"], 0.05, 0.65, 1.35, 6)
                cc, o = run_pair(p, box=[0.0, 1.0, 0.0, 1.0, 0.0, 1.0])
            check_all(cc, o)
        finally:
            c.set_option("split_stream", 0)
            c.set_option("split_work", 0)


def _solve_arrays(p, quintic, box=None):
    n = p.n
    c = capi.Cosmo(quintic)
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    c.upload(capi.VEL, np.stack([inputs.gaussian(n, 0, 0.1, 31 + k) for k in range(3)]))
    c.upload(capi.ACCEL, np.zeros((3, n)))
    c.density(n, p["pmass"], periodic_box=box, hfact=1.0 if quintic else 1.2)
    out = {k: c.array(k).copy() for k in ("h", "rho", "gradh", "divv", "xi", "ddivvdt")}
    out["iters"] = c.scalar("itersRun")
    out["active"] = c.array("activePerIter").copy()
    out["graph"] = c.scalar("loopGraph")
    return out


@pytest.mark.parametrize("case", ["lattice", "plummer_lognormal", "periodic"])
def test_newton_loop_graph_equals_host_loop(case):
    """The Newton loop run as one graph launch (a while node, with the list rebuilds and
    the row build as conditional nodes) and the host loop give the same h, rho and
    gradients bit for bit, in the same iterations with the same active counts."""
    quintic, box = False, None
    if case == "lattice":
        p = inputs.lattice100_workload(20)
    elif case == "plummer_lognormal":
        p = inputs.plummer(30000, lnsigma=0.5, seed=17)
        quintic = True
    else:
        p = inputs.uniform_box(20000, seed=8)
        box = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
    c = capi.Cosmo(quintic)
    try:
        assert c.set_option("newton_graph", 1) == 0
        # the graph is built when a solve's parameters repeat (buffers settled)
        for _ in range(3):
            g = _solve_arrays(p, quintic, box)
        assert c.set_option("newton_graph", 0) == 0
        h = _solve_arrays(p, quintic, box)
    finally:
        c.set_option("newton_graph", 1)
    assert g["graph"] == 1 and h["graph"] == 0
    assert g["iters"] == h["iters"]
    # later solves whose buffers need not grow (the buffers only grow, so a stepping
    # caller's stop growing) launch the same graph again
    q = dict(p)
    q["h"] = p["h"] * 0.99
    _solve_arrays(inputs.Particles(**q), quintic, box)
    builds = c.scalar("loopGraphBuilds")
    q["h"] = p["h"] * 0.98
    _solve_arrays(inputs.Particles(**q), quintic, box)
    assert c.scalar("loopGraph") == 1 and c.scalar("loopGraphBuilds") == builds
    np.testing.assert_array_equal(g["active"], h["active"])
    for k in ("h", "rho", "gradh", "divv", "xi", "ddivvdt"):
        np.testing.assert_array_equal(g[k], h[k], err_msg=k)


def test_newton_loop_graph_list_overflow_falls_back():
    """A graph-run loop whose list rebuild outgrows the storage the first lists sized
    reports it, and the solve is redone on the host loop: the results still equal the
    oracle's bit for bit."""
    c = capi.Cosmo(True)
    assert c.set_option("graph_list_store", 50) == 0    # half the first lists' entries
    try:
        p = inputs.plummer(12000, lnsigma=0.5, seed=29)
        builds = c.scalar("loopGraphBuilds")
        for _ in range(3):     # the graph is built once the parameters repeat
            cc, o = run_pair(p, quintic=True)
            assert cc.scalar("loopGraph") == 0
            check_all(cc, o)
        assert c.scalar("loopGraphBuilds") > builds
    finally:
        c.set_option("graph_list_store", 0)


def _step_arrays(p, quintic=False, box=None):
    c, o = run_pair(p, quintic=quintic, box=box)
    out = {k: c.array(k).copy() for k in FIELDS + FORCE}
    for k in ("pairsDensity", "pairsGrad", "pairsForce", "rowsFromNewton", "extraCount"):
        out[k] = c.scalar(k)
    return c, o, out


@pytest.mark.parametrize("case", ["lattice_open", "periodic", "plummer_quintic", "dead"])
def test_rows_from_newton_rows(case):
    """The gradient and force passes over the Newton rows' j, with the pairs another
    particle's larger support adds merged in, equal the oracle's bit for bit, and equal
    the passes over the symmetric rows built from the symmetric lists; the lists and hmax
    per node asked for afterwards are the reference's.  On the open lattice the surface
    particles' larger h adds such pairs to their neighbours' rows."""
    quintic, box = False, None
    if case == "lattice_open":
        p = inputs.lattice100_workload(20)
    elif case == "periodic":
        x, y, z = (np.asarray(v).ravel() for v in np.meshgrid(*(np.arange(14) / 14.0,) * 3, indexing="ij"))
        n = x.size
        rng = np.random.default_rng(3)
        p = inputs.Particles(x=(x + rng.uniform(0, 0.02, n)) % 1.0, y=(y + rng.uniform(0, 0.02, n)) % 1.0,
                             z=(z + rng.uniform(0, 0.02, n)) % 1.0, h=np.full(n, 1.2 / 14), pmass=1.0 / n)
        inputs.jiggle_frac(p["h"], 0.05, 0.65, 1.35, 4)
        box = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
    elif case == "plummer_quintic":
        p = inputs.plummer(12000, lnsigma=0.3, seed=42)
        quintic = True
    else:
        p = inputs.lattice100_workload(20)
        p["h"][np.arange(5, p.n, 37)] = -1.0
    cc = capi.Cosmo(quintic)
    try:
        assert cc.set_option("sym_from_rows", 1) == 0
        c, o, a = _step_arrays(p, quintic, box)
        check_all(c, o)
        assert cc.set_option("sym_from_rows", 0) == 0
        _, _, b = _step_arrays(p, quintic, box)
    finally:
        cc.set_option("sym_from_rows", 1)
    if case in ("lattice_open", "periodic", "dead"):
        assert a["rowsFromNewton"] == 1
    if case == "lattice_open":
        assert a["extraCount"] > 0
    assert b["rowsFromNewton"] == 0
    for k in FIELDS + FORCE + ["pairsDensity", "pairsGrad", "pairsForce"]:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("case", ["lattice_open", "periodic"])
def test_rows_from_newton_rows_mixed(case):
    """The mixed form's symmetric rows taken from its Newton rows (FP32 r^2, with dr^2
    taken again from the positions wherever it lies near a bound) are the rows built from
    the symmetric lists entry for entry, so its outputs are the same bits either way."""
    box = None
    if case == "lattice_open":
        p = inputs.lattice100_workload(20)
    else:
        x, y, z = (np.asarray(v).ravel() for v in np.meshgrid(*(np.arange(14) / 14.0,) * 3, indexing="ij"))
        n = x.size
        rng = np.random.default_rng(3)
        p = inputs.Particles(x=(x + rng.uniform(0, 0.02, n)) % 1.0, y=(y + rng.uniform(0, 0.02, n)) % 1.0,
                             z=(z + rng.uniform(0, 0.02, n)) % 1.0, h=np.full(n, 1.2 / 14), pmass=1.0 / n)
        inputs.jiggle_frac(p["h"], 0.05, 0.65, 1.35, 4)
        box = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
    n = p.n
    v, a = _vel_acc(p)
    th = _thermo(p, 1.2)

    def run():
        c = capi.Cosmo(False)
        c.set_precision(True)
        try:
            c.arrays_init(n)
            c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
            c.upload(capi.HSML, p["h"])
            c.upload(capi.VEL, v)
            c.upload(capi.ACCEL, a)
            c.density(n, p["pmass"], periodic_box=box, hfact=1.2)
            c.upload(capi.THERMO, th, sorted_=True)
            c.force(n, p["pmass"], beta=2.0, alphau=0.1)
            out = {k: c.array(k).copy() for k in FIELDS + FORCE}
            out["rowsFromNewton"] = c.scalar("rowsFromNewton")
            out["pairsForce"] = c.scalar("pairsForce")
        finally:
            c.set_precision(False)
        return out

    cc = capi.Cosmo(False)
    try:
        assert cc.set_option("sym_from_rows", 1) == 0
        a1 = run()
        assert cc.set_option("sym_from_rows", 0) == 0
        b0 = run()
    finally:
        cc.set_option("sym_from_rows", 1)
    assert a1["rowsFromNewton"] == 1 and b0["rowsFromNewton"] == 0
    for k in FIELDS + FORCE + ["pairsForce"]:
        np.testing.assert_array_equal(a1[k], b0[k], err_msg=k)


def test_rows_from_newton_rows_extras_fallback():
    """When the pairs other particles' supports add to the rows taken from the Newton rows
    do not all fit (here the merge holds one), the force pass builds the symmetric rows from
    the symmetric lists instead: every structure and field still equals the oracle's."""
    p = inputs.lattice100_workload(20)
    cc = capi.Cosmo(False)
    try:
        assert cc.set_option("sym_from_rows", 1) == 0
        assert cc.set_option("sym_extra_cap", 1) == 0
        c, o = run_pair(p)
        assert c.scalar("extraCount") > 1
        assert c.scalar("rowsFromNewton") == 0
        check_all(c, o)
    finally:
        cc.set_option("sym_extra_cap", 0)
        cc.set_option("sym_from_rows", 1)
