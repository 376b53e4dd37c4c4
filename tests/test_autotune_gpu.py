"""The batched form's launch parameters and their autotuner on the GPU: any setting the
tuner may pick leaves the plain FP64 results bit for bit unchanged (per set, mixed
settings across the sets of one batch), out-of-range values are refused with nothing
set, and a tuning run over a small ensemble yields a table whose settings keep the
results too."""
import numpy as np
import pytest

from cosmosphere_b200 import autotune as at
from cosmosphere_b200 import capi
from tests.test_batch_gpu import make_sets

pytestmark = pytest.mark.gpu


def solve(sets, tuning=None, table=None, final_rho=True):
    capi.Cosmo().set_precision(False)
    b = capi.Batch(sets)
    if tuning is not None:
        b.set_tuning(**tuning)
    if table is not None:
        table.apply(b)
    b.upload()
    assert b.density(final_rho=final_rho) == 0
    return b, b.download()


@pytest.fixture(scope="module")
def sets():
    return make_sets()


@pytest.fixture(scope="module")
def reference(sets):
    return solve(sets)[1]


def same(a, b):
    for k in range(3):
        for x, y in zip(a[k], b[k]):
            np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("setting", [
    dict(bucket=16), dict(bucket=128), dict(bucket=512), dict(list_margin=1.0), dict(list_margin=1.3),
    dict(split_stream=32, split_work=32),               # every leaf cut into one-particle items
    dict(bucket=[16, 128, 32, 64, 128, 16], list_margin=[1.0, 1.3, 1.05, 1.15, 1.0, 1.3],
         split_stream=[2048, 16384, 32, 4096, 8192, 32], split_work=[65536, 262144, 64, 131072, 65536, 32]),
])
def test_any_setting_keeps_the_plain_results(sets, reference, setting):
    b, out = solve(sets, tuning=setting)
    same(out, reference)


def test_out_of_range_values_are_refused(sets, reference):
    b = capi.Batch(sets)
    for bad in (dict(bucket=4), dict(bucket=4096), dict(list_margin=0.9), dict(list_margin=2.5),
                dict(split_stream=8), dict(split_work=0)):
        with pytest.raises(ValueError):
            b.set_tuning(**bad)
    # nothing was set: the batch still solves with the defaults
    b.upload()
    assert b.density(final_rho=True) == 0
    same(b.download(), reference)


def test_tuning_run_on_a_small_ensemble(sets, reference):
    cands = {"bucket": (32, 64), "list_margin": (1.05, 1.15), "split_stream": (4096,), "split_work": (131072,)}
    table = at.tune(sets, max_particles=2e4, repeats=1, candidates=cands)
    assert set(table.entries) == {at.size_class(s["x"].size) for s in sets}
    for c, t in table.entries.items():
        assert t.bucket in cands["bucket"] and t.list_margin in cands["list_margin"]
        assert table.times[c]["tuned_s"] <= table.times[c]["default_s"]
    b, out = solve(sets, table=table)
    same(out, reference)
