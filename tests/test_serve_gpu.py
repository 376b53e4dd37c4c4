"""The served form: continuous batching of density + force requests over worker slots,
device-resident sets with warm-started continuation, and admission against an HBM
budget.  Requests are independent, so each result must be the same -- bit for bit in the
plain form -- served alone or in a concurrent mix."""
import numpy as np
import pytest

from cosmosphere_b200 import capi, inputs

# a hung wait would block the whole GPU run: end the process instead
pytestmark = [pytest.mark.gpu, pytest.mark.timeout(300, method="thread")]


def thermo_for(p, hfact=1.2):
    n = p.n
    rho = p["pmass"] * (hfact / p["h"]) ** 3
    return np.stack([(2.0 / 3.0) / rho, np.full(n, np.sqrt(10.0 / 9.0)), np.ones(n), np.ones(n)])


def requests():
    out = []
    p = inputs.lattice100_workload(16); out.append((p, None))
    q = inputs.plummer(30000, hfact=1.2, lnsigma=0.0, ulo=0.8, uhi=1.2, seed=11); out.append((q, None))
    u = inputs.uniform_box(25000, seed=12); u["vx"], u["vy"], u["vz"] = (inputs.gaussian(u.n, 0, 0.05, 20 + k) for k in range(3))
    out.append((u, [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]))
    p = inputs.lattice100_workload(12); out.append((p, None))
    q = inputs.plummer(8000, hfact=1.2, lnsigma=0.0, ulo=0.8, uhi=1.2, seed=13); out.append((q, None))
    u = inputs.uniform_box(6000, seed=14); out.append((u, [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]))
    return out


@pytest.fixture(scope="module")
def reqs():
    return requests()


def serve(reqs, slots, budget=150.0, keep=False):
    S = capi.Server(slots=slots, budget_gb=budget)
    try:
        ids = [S.submit(p, thermo_for(p), box=b, keep=keep) for p, b in reqs]
        res = [S.wait(i) for i in ids]
        stats = {"max_inflight": S.server_stat("max_inflight"),
                 "intervals": [(S.stat(i, "start"), S.stat(i, "done")) for i in ids]}
    finally:
        S.stop()
    return res, stats


def test_same_alone_and_in_the_mix(reqs):
    alone = []
    for r in reqs:
        res, _ = serve([r], slots=1)
        alone.append(res[0])
    mix, stats = serve(reqs, slots=4)
    for k, ((s1, a), (s2, b)) in enumerate(zip(alone, mix)):
        assert s1 == 1 and s2 == 1
        for key in ("h", "dens", "grad", "force"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"request {k} {key}")
    # the mix really overlapped on the device
    assert stats["max_inflight"] >= 2
    iv = stats["intervals"]
    assert any(a0 < b1 and b0 < a1 for i, (a0, a1) in enumerate(iv) for (b0, b1) in iv[i + 1:])


def test_served_request_equals_c_abi_solve(reqs):
    p, box = reqs[0]
    out, _ = serve([reqs[0]], slots=1)
    st, res = out[0]
    assert st == 1
    n = p.n
    c = capi.Cosmo()
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    c.upload(capi.VEL, np.stack([p["vx"], p["vy"], p["vz"]]))
    c.upload(capi.ACCEL, np.zeros((3, n)))
    c.density(n, p["pmass"])
    c.upload(capi.THERMO, thermo_for(p), sorted_=True)
    c.force(n, p["pmass"], beta=2.0, alphau=0.0)
    np.testing.assert_array_equal(res["h"], c.download(capi.HSML, n)[0])
    np.testing.assert_array_equal(res["dens"], c.download(capi.DENS_OUT, n))
    np.testing.assert_array_equal(res["force"], c.download(capi.FORCE_OUT, n))


def test_warm_started_continuation(reqs):
    p, box = reqs[0]
    n = p.n
    th = thermo_for(p)
    S = capi.Server(slots=2)
    try:
        r0 = S.submit(p, th, keep=True)
        st0, first = S.wait(r0)
        cs = th[1]
        dt = 0.1 * float(np.min(first["h"] / cs))
        r1 = S.cont(r0, dt, keep=True)
        st1, second = S.wait(r1)
        it_warm = S.stat(r1, "iters")
        it_cold = S.stat(r0, "iters")
    finally:
        S.stop()
    assert st0 == 1 and st1 == 1
    # the same step done cold through the C-ABI: advanced positions, previous h as the guess
    q = dict(p)
    q["x"], q["y"], q["z"] = p["x"] + p["vx"] * dt, p["y"] + p["vy"] * dt, p["z"] + p["vz"] * dt
    c = capi.Cosmo()
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([q["x"], q["y"], q["z"]]))
    c.upload(capi.HSML, first["h"])
    c.upload(capi.VEL, np.stack([p["vx"], p["vy"], p["vz"]]))
    c.upload(capi.ACCEL, np.zeros((3, n)))
    c.density(n, p["pmass"])
    c.upload(capi.THERMO, th, sorted_=True)
    c.force(n, p["pmass"], beta=2.0, alphau=0.0)
    np.testing.assert_array_equal(second["h"], c.download(capi.HSML, n)[0])
    np.testing.assert_array_equal(second["force"], c.download(capi.FORCE_OUT, n))
    assert it_warm <= it_cold


def test_admission_against_the_budget():
    four = [(inputs.uniform_box(8000, seed=40 + k), [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]) for k in range(4)]
    base = capi.load().cosmo_serve_stat(b"device_bytes")
    L = capi.load()
    est = L.cosmo_serve_stat(b"bytes_fixed") + L.cosmo_serve_stat(b"bytes_per_particle") * 8000
    budget = (base + 1.5 * est) / 1e9          # room for one set at a time
    res, stats = serve(four, slots=4, budget=budget)
    assert all(s == 1 for s, _ in res)
    assert stats["max_inflight"] == 1
    # a request that cannot fit beside what is already held is rejected, not queued forever
    S = capi.Server(slots=2, budget_gb=budget)
    try:
        big = inputs.lattice100_workload(24)
        rid = S.submit(big, thermo_for(big), keep=False)
        st, _ = S.wait(rid)
        assert st == -1
        assert S.server_stat("rejected") == 1
    finally:
        S.stop()


def test_lru_eviction_of_idle_resident_sets():
    L = capi.load()
    three = [(inputs.uniform_box(6000, seed=30 + k), [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]) for k in range(3)]
    # what one resident set of this size really holds on the device
    S = capi.Server(slots=1)
    try:
        base = S.server_stat("device_bytes")
        for p, b in three[:2]:
            assert S.wait(S.submit(p, thermo_for(p), box=b, keep=True))[0] == 1
        held = (S.server_stat("device_bytes") - base) / 2
    finally:
        S.stop()
    base = L.cosmo_serve_stat(b"device_bytes")
    est = L.cosmo_serve_stat(b"bytes_fixed") + L.cosmo_serve_stat(b"bytes_per_particle") * 6000
    assert held >= 0.5 * est
    S = capi.Server(slots=1, budget_gb=(base + 2 * held + 0.5 * est) / 1e9)   # two fit, a third does not
    try:
        ids = []
        for p, b in three:
            ids.append(S.submit(p, thermo_for(p), box=b, keep=True))
            assert S.wait(ids[-1])[0] == 1
        assert S.server_stat("evicted") == 1
        assert S.server_stat("resident_sets") == 2
        with pytest.raises(RuntimeError):
            S.cont(ids[0], 1e-4)            # the least recently used set was evicted
        assert S.wait(S.cont(ids[2], 1e-4))[0] == 1
    finally:
        S.stop()


def drift_wrap(x, v, dt, box):
    """Host drift of the served continuation: x + v dt, wrapped into a periodic box."""
    y = x + v * dt
    if box is not None:
        lo, hi = box[0], box[1]
        y = np.where(y >= hi, y - (hi - lo), np.where(y < lo, y + (hi - lo), y))
    return y


def test_continuations_queued_before_admission(reqs):
    """Continuations may be submitted while their set's first request still waits in the
    queue; they run after it, in order, and equal the same steps done through the C-ABI
    (periodic box: drifted coordinates wrap)."""
    p, box = reqs[2]
    n = p.n
    th = thermo_for(p)
    S = capi.Server(slots=1)
    try:
        blocker = S.submit(reqs[0][0], thermo_for(reqs[0][0]), keep=False)
        r0 = S.submit(p, th, box=box, keep=True)
        dt = 0.05
        r1 = S.cont(r0, dt)
        r2 = S.cont(r0, dt)
        out = [S.wait(r) for r in (blocker, r0, r1, r2)]
        assert S.stat(r1, "start") >= S.stat(r0, "done") and S.stat(r2, "start") >= S.stat(r1, "done")
    finally:
        S.stop()
    assert all(st == 1 for st, _ in out)
    c = capi.Cosmo()
    pos = np.stack([p["x"], p["y"], p["z"]])
    vel = np.stack([p["vx"], p["vy"], p["vz"]])
    h = p["h"]
    for k in range(3):
        if k:
            pos = drift_wrap(pos, vel, dt, box)
        c.arrays_init(n)
        c.upload(capi.POS, pos)
        c.upload(capi.HSML, h)
        c.upload(capi.VEL, vel)
        c.upload(capi.ACCEL, np.zeros((3, n)))
        c.density(n, p["pmass"], periodic_box=box)
        c.upload(capi.THERMO, th, sorted_=True)
        c.force(n, p["pmass"], beta=2.0, alphau=0.0)
        h = c.download(capi.HSML, n)[0]
        got = out[k + 1][1]
        np.testing.assert_array_equal(got["h"], h, err_msg=f"step {k}")
        np.testing.assert_array_equal(got["force"], c.download(capi.FORCE_OUT, n), err_msg=f"step {k}")
    assert np.all((pos >= 0.0) & (pos < 1.0))


def test_mixed_same_alone_and_in_the_mix(reqs):
    """The mixed-precision served form (the form the served bench runs): each request's
    result in a concurrent mix equals its result served alone within the mixed form's
    stated tolerance (1e-5 relative in h and rho, 1e-5 of the field's rms elsewhere), and
    both are within it of the plain FP64 result."""
    c = capi.Cosmo()
    plain = []
    for r in reqs:
        res, _ = serve([r], slots=1)
        plain.append(res[0])
    c.set_precision(True)
    try:
        alone = []
        for r in reqs:
            res, _ = serve([r], slots=1)
            alone.append(res[0])
        mix, stats = serve(reqs, slots=4)
    finally:
        c.set_precision(False)
    assert stats["max_inflight"] >= 2

    def close(a, b, what):
        for key in ("h", "dens"):
            x, y = a[key].reshape(-1), b[key].reshape(-1)
            if key == "dens":
                x, y = a[key][0], b[key][0]
            live = np.abs(y) > 0
            assert np.max(np.abs(x[live] / y[live] - 1.0)) <= 1e-5, (what, key)
        for key in ("grad", "force"):
            for comp in range(a[key].shape[0]):
                x, y = a[key][comp], b[key][comp]
                rms = np.sqrt(np.mean(y * y))
                if rms > 0:
                    assert np.max(np.abs(x - y)) <= 1e-5 * (rms + np.max(np.abs(y))), (what, key, comp)

    for k, ((s0, p0), (s1, a), (s2, b)) in enumerate(zip(plain, alone, mix)):
        assert s0 == 1 and s1 == 1 and s2 == 1
        close(b, a, f"request {k}: mix vs alone")
        close(a, p0, f"request {k}: mixed vs plain")
