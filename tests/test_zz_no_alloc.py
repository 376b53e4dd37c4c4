"""The allocation-free entry point, cosmo_hilbert_order_noalloc, against the keys and
sort order the regular density solve builds for the same particles.

It serves callers that cannot allocate device memory at call time (a fixed device
budget set at start-up, or GPU work of their own in flight that cudaMalloc's device-wide
synchronisation would stall).  This file is collected last on purpose."""
import numpy as np
import pytest

from cosmosphere_b200 import capi, inputs

pytestmark = pytest.mark.gpu


def _reference_order(p, box=None):
    """Keys and order from the regular entry points (cosmo_upload + densityiterate_gpu_c)."""
    n = p.n
    c = capi.Cosmo()
    c.arrays_init(n)
    c.upload(capi.POS, np.stack([p["x"], p["y"], p["z"]]))
    c.upload(capi.HSML, p["h"])
    c.density(n, p["pmass"], periodic_box=box)
    return c, c.array("keys"), c.array("order")


def _device(a, torch, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _noalloc_twice(p, box=None):
    """Two calls in a row of the allocation-free entry point on the same device inputs;
    each must give the regular path's keys and order, and the second reserves nothing."""
    import torch
    n = p.n
    c, want_keys, want_order = _reference_order(p, box)
    dx, dy, dz, dh = (_device(p[k], torch, torch.float64) for k in "xyzh")
    keys = torch.empty(n, dtype=torch.int64, device="cuda")
    order = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        keys.fill_(-1)
        order.fill_(-1)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = c.hilbert_order_noalloc(n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), dh.data_ptr(),
                                     keys.data_ptr(), order.data_ptr(), periodic_box=box)
        torch.cuda.synchronize()
        assert rc == 0, (call, rc)
        if call == 1:                       # after the first call's set-up, nothing more is reserved
            assert torch.cuda.mem_get_info()[0] == free_before
        np.testing.assert_array_equal(keys.cpu().numpy().view(np.uint64), want_keys, err_msg=f"call {call}")
        np.testing.assert_array_equal(order.cpu().numpy(), want_order, err_msg=f"call {call}")
    return want_keys, want_order


@pytest.mark.parametrize("periodic", [False, True])
def test_noalloc_matches_regular_entry_point_twice(periodic):
    p = inputs.lattice100_workload(24)
    if periodic:
        p["x"], p["y"], p["z"] = (np.mod(p[k] + 0.013, 1.0) for k in "xyz")
    box = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0] if periodic else None
    _noalloc_twice(p, box)


def test_noalloc_at_its_largest_size_with_dead_particles():
    """n = 524,288, the most the fixed scratch serves, with dead particles (h <= 0): the
    scratch covers the sort there, dead particles get the all-ones key and sit at the end
    of the order in their input order, exactly as in the regular path."""
    n = 1 << 19
    rng = np.random.default_rng(19)
    x, y, z = rng.random((3, n))
    h = np.full(n, 1.2 * n ** (-1.0 / 3.0))
    dead = np.sort(rng.choice(n, 1500, replace=False))
    h[dead] = -1.0
    h[dead[:7]] = 0.0
    p = inputs.Particles(x=x, y=y, z=z, h=h, pmass=1.0 / n)
    keys, order = _noalloc_twice(p)
    assert np.all(keys[-dead.size:] == np.uint64(2**64 - 1))
    assert np.all(keys[:-dead.size] < np.uint64(2**63))
    np.testing.assert_array_equal(order[-dead.size:], dead)


def test_noalloc_rejects_sizes_beyond_its_scratch(capfd):
    c = capi.Cosmo()
    assert c.hilbert_order_noalloc((1 << 19) + 1, 0, 0, 0, 0, 0, 0) == -1
    assert c.hilbert_order_noalloc(0, 0, 0, 0, 0, 0, 0) == -1
    err = capfd.readouterr().err
    assert "outside [1, 524288]" in err
    # periodic without a box is rejected before any device work
    assert c.L.cosmo_hilbert_order_noalloc(16, 0, 0, 0, 0, 1, None, 0, 0) == -1
    assert "needs box6" in capfd.readouterr().err
