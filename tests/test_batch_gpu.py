"""The batched form: several independent sets (lattices, periodic uniform boxes, Plummer
spheres) solved in one forest with one density launch per Newton iteration.  In the
plain FP64 form each set must come out bit for bit as the same set solved alone (the
single-set path is itself bit-exact with the oracle); in the mixed form within the
1e-5 bound; and the leaf capacity (a tuning parameter of this form) must not change
the plain results."""
import numpy as np
import pytest

from cosmosphere_b200 import capi, inputs
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def make_sets():
    sets = []
    p = inputs.lattice(14); inputs.jiggle_ref(p["h"], 42); sets.append(dict(p))
    sets.append(dict(inputs.uniform_box(9000, seed=3), box=[0.0, 1.0, 0.0, 1.0, 0.0, 1.0]))
    q = inputs.plummer(15000, hfact=1.2, lnsigma=0.0, ulo=0.8, uhi=1.2, seed=4); sets.append(dict(q))
    p = inputs.lattice(9); sets.append(dict(p))
    sets.append(dict(inputs.uniform_box(4000, seed=5), box=[0.0, 1.0, 0.0, 1.0, 0.0, 1.0]))
    q = inputs.plummer(6000, hfact=1.2, lnsigma=0.0, ulo=0.8, uhi=1.2, seed=6)
    q["h"][::50] = -1.0                       # some dead particles in one set
    sets.append(dict(q))
    return sets


def single(s):
    n = s["x"].size
    c = capi.Cosmo()
    c.set_precision(False)
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([s["x"], s["y"], s["z"]]))
    c.upload(capi.HSML, s["h"])
    assert c.density_status(n, s["pmass"], periodic_box=s.get("box"), with_gradients=False) == 0
    return c.download(capi.HSML, n)[0], c.download(capi.DENS_OUT, n)


@pytest.fixture(scope="module")
def sets():
    return make_sets()


@pytest.fixture(scope="module")
def singles(sets):
    return [single(s) for s in sets]


def run_batch(sets, mixed=False, bucket=None):
    capi.Cosmo().set_precision(mixed)
    b = capi.Batch(sets, bucket=bucket)
    b.upload()
    assert b.density() == 0
    out = b.download()
    capi.Cosmo().set_precision(False)
    return b, out


def test_batch_plain_equals_each_set_alone(sets, singles):
    b, (h, rho, gh) = run_batch(sets)
    for k, (hs, d) in enumerate(singles):
        np.testing.assert_array_equal(h[k], hs, err_msg=f"set {k} h")
        np.testing.assert_array_equal(rho[k], d[0], err_msg=f"set {k} rho")
        np.testing.assert_array_equal(gh[k], d[1], err_msg=f"set {k} gradh")
    assert b.scalar("itersRun") >= 2


def test_batch_set_matches_oracle(sets):
    b, (h, rho, gh) = run_batch(sets)
    s = sets[2]
    o = O.Oracle()
    assert o.density(s["x"], s["y"], s["z"], s["h"], s["pmass"], with_gradients=False) == 0
    np.testing.assert_array_equal(h[2], o.unsorted("h"))
    np.testing.assert_array_equal(rho[2], o.unsorted("rho"))


def test_batch_mixed_within_bound(sets, singles):
    b, (h, rho, gh) = run_batch(sets, mixed=True)
    for k, (hs, d) in enumerate(singles):
        live = hs > 0
        assert np.max(np.abs(h[k][live] / hs[live] - 1)) <= 1e-5, k
        assert np.max(np.abs(rho[k][live] / d[0][live] - 1)) <= 1e-5, k


@pytest.mark.parametrize("bucket", [16, 32, 128])
def test_bucket_size_does_not_change_plain_results(sets, singles, bucket):
    """The leaf capacity changes the tree, the lists and the work items, but not the
    accepted pairs or their (ascending j) order: the plain results are the same bits."""
    b, (h, rho, gh) = run_batch(sets, bucket=bucket)
    for k, (hs, d) in enumerate(singles):
        np.testing.assert_array_equal(h[k], hs, err_msg=f"set {k}")
        np.testing.assert_array_equal(rho[k], d[0], err_msg=f"set {k}")


def test_graph_loop_equals_host_loop(sets):
    """The Newton loop run as one CUDA graph (device-side while condition) gives the
    same bits as the same loop driven from the host."""
    capi.Cosmo().set_precision(False)
    b = capi.Batch(sets)
    b.upload()
    assert b.density(graph=True) == 0
    g = b.download()
    assert b.scalar("graph") == 1.0
    iters_g = b.scalar("itersRun")
    assert b.density(graph=False) == 0
    hst = b.download()
    assert b.scalar("itersRun") == iters_g
    for a, c in zip(g, hst):
        for x, y in zip(a, c):
            np.testing.assert_array_equal(x, y)


def test_final_rho_mixed_within_bound(sets):
    """With rho re-evaluated at the converged h, the mixed form's rho is within 1e-5 of
    the FP64 form's (without it, rho is one Newton step behind h, and a particle that
    converges one iteration earlier in one form carries a rho one step apart)."""
    res = {}
    for mixed in (False, True):
        capi.Cosmo().set_precision(mixed)
        b = capi.Batch(sets)
        b.upload()
        assert b.density(final_rho=True) == 0
        res[mixed] = b.download()
    capi.Cosmo().set_precision(False)
    for k in range(len(sets)):
        h0, r0 = res[False][0][k], res[False][1][k]
        h1, r1 = res[True][0][k], res[True][1][k]
        live = h0 > 0
        assert np.max(np.abs(h1[live] / h0[live] - 1)) <= 1e-5, k
        assert np.max(np.abs(r1[live] / r0[live] - 1)) <= 1e-5, k


def test_batch_with_tiny_sets():
    """Sets of one leaf and just over one leaf beside a larger one: each comes out as the
    same set solved alone."""
    tiny = []
    for n in (33, 65, 700):
        rng = np.random.default_rng(100 + n)
        x, y, z = rng.random((3, n))
        tiny.append(dict(inputs.Particles(x=x, y=y, z=z, h=np.full(n, 1.2 * (1.0 / n) ** (1.0 / 3.0)),
                                          pmass=1.0 / n)))
    alone = [single(s) for s in tiny]
    b, (h, rho, gh) = run_batch(tiny)
    for k, (hs, d) in enumerate(alone):
        np.testing.assert_array_equal(h[k], hs, err_msg=f"set {k} h")
        np.testing.assert_array_equal(rho[k], d[0], err_msg=f"set {k} rho")
