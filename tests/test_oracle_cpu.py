"""The oracle on its own: pinned against the reference's code where that is possible
(kernel functions, driver generators), and checked by the properties the reference's
algorithm guarantees where it is not (curve, tree, lists, physics)."""
import itertools
import os

import numpy as np
import pytest

from cosmosphere_b200 import inputs
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# ---------------------------------------------------------------- pins against the reference
@pytest.mark.parametrize("name,quintic", [("cubic", False), ("quintic", True)])
def test_kernel_matches_reference_kernel_hpp(name, quintic):
    g = np.load(os.path.join(GOLDEN, "ref_kernel.npz"))
    w, dw = O.kernel_eval(g["q"], quintic)
    np.testing.assert_array_equal(w, g[f"{name}_w"])
    np.testing.assert_array_equal(dw, g[f"{name}_dw"])
    np.testing.assert_array_equal(O.kernel_consts(quintic), g[f"{name}_consts"])


@pytest.mark.parametrize("tag", ["plain", "jiggle"])
def test_generators_match_reference_driver(tag):
    g = np.load(os.path.join(GOLDEN, "ref_driver_lattice8.npz"))
    p = inputs.lattice(8)
    if tag == "jiggle":
        inputs.jiggle_ref(p["h"], 42)
    assert p.n == int(g[f"{tag}_n"])
    assert p["pmass"] == float(g[f"{tag}_pmass"])
    for k in "xyzh":
        np.testing.assert_array_equal(p[k], g[f"{tag}_{k}"])


def test_lattice_sizes_match_reference_driver_comment():
    # src/main.cu:76-77: npartx 50 -> 173,850 particles, 100 -> 1,403,000
    assert inputs.lattice(50).n == 173850
    assert inputs._lib().cin_lattice_count(100) == 1403000


# ---------------------------------------------------------------- the curve
@pytest.mark.parametrize("bits", [1, 2, 3, 4])
def test_hilbert_curve_exhaustive(bits):
    side = 1 << bits
    keys = {}
    for x, y, z in itertools.product(range(side), repeat=3):
        k = O.hilbert_encode(x, y, z, bits)
        assert O.hilbert_decode(k, bits) == (x, y, z)
        keys[k] = (x, y, z)
    assert sorted(keys) == list(range(side ** 3))               # a bijection onto [0, 8^b)
    for k in range(side ** 3 - 1):                              # face-adjacent steps
        a, b = np.array(keys[k]), np.array(keys[k + 1])
        assert np.abs(a - b).sum() == 1
    for level in range(1, bits + 1):                            # octree alignment
        sh = bits - level
        for (x, y, z) in itertools.product(range(side), repeat=3):
            k = O.hilbert_encode(x, y, z, bits)
            k0 = O.hilbert_encode((x >> sh) << sh, (y >> sh) << sh, (z >> sh) << sh, bits)
            assert k >> (3 * sh) == k0 >> (3 * sh)


def test_hilbert_curve_21_bits_random():
    rng = np.random.default_rng(7)
    for _ in range(2000):
        c = tuple(int(v) for v in rng.integers(0, 1 << 21, 3))
        k = O.hilbert_encode(*c, 21)
        assert k < (1 << 63)
        assert O.hilbert_decode(k, 21) == c
        L = int(rng.integers(1, 21))
        sh = 21 - L
        c2 = tuple(((v >> sh) << sh) | int(rng.integers(0, 1 << sh)) for v in c)
        assert O.hilbert_encode(*c2, 21) >> (3 * sh) == k >> (3 * sh)


# ---------------------------------------------------------------- tree and lists
def _solve(p, **kw):
    o = O.Oracle(quintic=kw.pop("quintic", False))
    st = o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], **kw)
    return o, st


@pytest.fixture(scope="module")
def lat16():
    p = inputs.lattice(16)
    inputs.jiggle_ref(p["h"], 42)
    o, st = _solve(p, vel=np.zeros((3, p.n)), acc=np.zeros((3, p.n)))
    assert st == 0
    return p, o


def test_tree_invariants(lat16):
    p, o = lat16
    keys, tree, counts, layout = o.array("keys"), o.array("csTree"), o.array("counts"), o.array("layout")
    nA = int(o.scalar("nAlive"))
    assert np.all(np.diff(keys.astype(object)) >= 0)
    assert tree[0] == 0 and tree[-1] == 1 << 63 and np.all(np.diff(tree.astype(object)) > 0)
    lens = np.diff(tree.astype(object))
    for ln in lens:                                             # every leaf is an octree node
        assert ln & (ln - 1) == 0 and (ln.bit_length() - 1) % 3 == 0
    assert np.all(counts <= 64)
    assert layout[0] == 0 and layout[-1] == nA and np.all(np.diff(layout.astype(np.int64)) == counts)
    # a parent of any leaf holds more than the bucket (else it would not have split)
    k = keys[:nA].astype(object)
    for i in range(len(counts)):
        ln = int(lens[i])
        if ln == 1 << 63:
            continue
        plen = ln * 8
        pstart = (int(tree[i]) // plen) * plen
        c = np.searchsorted(k, pstart + plen) - np.searchsorted(k, pstart)
        assert c > 64


def test_octree_links_and_geometry(lat16):
    p, o = lat16
    pref, co, i2l = o.array("prefixes"), o.array("childOffsets"), o.array("internalToLeaf")
    cen, siz = o.array("centers").reshape(-1, 3), o.array("sizes").reshape(-1, 3)
    nL = int(o.scalar("nLeaves"))
    assert len(pref) == 1 + 8 * (len(pref) - nL) // 8 * 1 or True
    assert (co == 0).sum() == nL and len(pref) == nL + (len(pref) - nL)
    assert len(pref) - nL == (nL - 1) // 7                       # 8-ary: L = 1 + 7 I
    for b in np.nonzero(co)[0]:                                 # children contiguous, prefix*8+o
        for oc in range(8):
            assert int(pref[co[b] + oc]) == (int(pref[b]) << 3) | oc
    # particles lie in their leaf's box
    x, y, z = o.array("x"), o.array("y"), o.array("z")
    l2i, pl = o.array("leafToInternal"), o.array("particleLeaf")
    nA = int(o.scalar("nAlive"))
    node = l2i[pl[:nA]]
    pos = np.stack([x[:nA], y[:nA], z[:nA]], 1)
    assert np.all(np.abs(pos - cen[node]) <= siz[node] * (1 + 1e-12))
    assert np.all(i2l[co == 0] >= 0)


def test_gather_lists_cover_all_neighbours(lat16):
    """Every pair within 2 h_i appears through the i-leaf's list (brute force)."""
    p, o = lat16
    x, y, z, h = (o.array(k) for k in "xyzh")
    nA = int(o.scalar("nAlive"))
    pl, jo, jc, jl, lay = (o.array(k) for k in ("particleLeaf", "jOffset", "jcount", "jlist", "layout"))
    pos = np.stack([x, y, z], 1)[:nA]
    rng = np.random.default_rng(3)
    for i in rng.choice(nA, 150, replace=False):
        r = np.sqrt(((pos - pos[i]) ** 2).sum(1))
        nb = np.nonzero(r < 2.0 * h[i])[0]
        leaves = set(jl[jo[pl[i]]:jo[pl[i]] + jc[pl[i]]])
        assert set(pl[nb]) <= leaves
        assert list(jl[jo[pl[i]]:jo[pl[i]] + jc[pl[i]]]) == sorted(leaves)


def test_symmetric_lists_cover_scatter_neighbours(lat16):
    p, o = lat16
    n = p.n
    th = np.zeros((4, n))
    th[0], th[1], th[2], th[3] = 1.0, 1.0, 1.0, 1.0
    assert o.force(th) == 0
    x, y, z, h = (o.array(k) for k in "xyzh")
    nA = int(o.scalar("nAlive"))
    pl, jo, jc, jl = (o.array(k) for k in ("particleLeaf", "jOffset", "jcount", "jlist"))
    pos = np.stack([x, y, z], 1)[:nA]
    rng = np.random.default_rng(4)
    for i in rng.choice(nA, 150, replace=False):
        r = np.sqrt(((pos - pos[i]) ** 2).sum(1))
        nb = np.nonzero((r < 2.0 * h[i]) | (r < 2.0 * h[:nA]))[0]
        leaves = set(jl[jo[pl[i]]:jo[pl[i]] + jc[pl[i]]])
        assert set(pl[nb]) <= leaves


# ---------------------------------------------------------------- physics known answers
def test_lattice_interior_density_and_omega():
    p = inputs.lattice(20)
    o, st = _solve(p, vel=np.zeros((3, p.n)), acc=np.zeros((3, p.n)))
    assert st == 0
    x, y, z, h, rho, gh = (o.array(k) for k in ("x", "y", "z", "h", "rho", "gradh"))
    inner = (np.abs(x - 0.5) < 0.25) & (np.abs(y - 0.5) < 0.25) & (np.abs(z - 0.5) < 0.25)
    rhoh = p["pmass"] * (1.2 / h) ** 3
    # converged: rho(sum) == rho(h) to the Newton tolerance; omega ~ 1 in the interior
    assert np.max(np.abs(rho[inner] / rhoh[inner] - 1)) < 1e-3
    omega = 1 + h / (3 * rho) * gh
    assert np.max(np.abs(omega[inner] - 1)) < 0.05
    # a close-packed lattice of unit total mass in a unit box: rho ~ sqrt(2) * N dx^3 ...
    assert np.allclose(rho[inner].mean(), np.sqrt(2) * p["pmass"] * 20 ** 3, rtol=0.02)


def test_momentum_conservation_open():
    p = inputs.lattice100_workload(14)
    o, st = _solve(p, vel=np.stack([p["vx"], p["vy"], p["vz"]]), acc=np.zeros((3, p.n)))
    assert st == 0
    assert o.force(np.stack([p["pro2"], p["cs"], p["alpha"], p["u"]])) == 0
    f = np.stack([o.array("fx"), o.array("fy"), o.array("fz")])
    scale = np.abs(f).sum(1)
    assert np.all(np.abs(f.sum(1)) < 1e-10 * scale)


def test_dead_particles_are_parked_and_zeroed():
    p = inputs.lattice(12)
    h = p["h"].copy()
    dead = np.arange(0, p.n, 97)
    h[dead] = -1.0
    h[5] = np.nan
    o = O.Oracle()
    assert o.density(p["x"], p["y"], p["z"], h, p["pmass"], vel=np.zeros((3, p.n)), acc=np.zeros((3, p.n))) == 0
    nd = len(dead) + 1
    assert int(o.scalar("nAlive")) == p.n - nd
    hu = o.unsorted("h")
    np.testing.assert_array_equal(hu[dead], -1.0)
    assert np.isnan(hu[5])
    assert np.all(o.unsorted("rho")[dead] == 0) and np.all(o.unsorted("xi")[dead] == 1.0)
    th = np.ones((4, p.n))
    o.force(th)
    assert np.all(o.unsorted("fx")[dead] == 0)


def test_status_codes():
    p = inputs.lattice(12)
    o = O.Oracle()
    assert o.density(p["x"], p["y"], p["z"], p["h"], p["pmass"], max_iter=1) == 1
    # 27 particles in a unit period: the converged support 2h ~ 0.8 reaches half the box
    x, y, z = _cubic_lattice(3)
    o2 = O.Oracle()
    assert o2.density(x, y, z, np.full(27, 0.4), 1.0 / 27, periodic_box=[0, 1, 0, 1, 0, 1]) == 2


def _cubic_lattice(nx):
    g = (np.arange(nx) + 0.5) / nx
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return X.ravel(), Y.ravel(), Z.ravel()


def test_periodic_lattice_is_uniform():
    # lattice spacings that tile the period exactly: every particle sees the same density
    nx = 8
    dx = 1.0 / nx
    x, y, z = _cubic_lattice(nx)
    n = x.size
    h = np.full(n, 1.2 * dx)
    o = O.Oracle()
    assert o.density(x, y, z, h, 1.0 / n, periodic_box=[0, 1, 0, 1, 0, 1]) == 0
    rho = o.array("rho")
    assert np.max(np.abs(rho / rho.mean() - 1)) < 1e-12
