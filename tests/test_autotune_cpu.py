"""Host logic of the batched form's autotuner (CPU only): size classes, sampling, the
coordinate descent over a synthetic cost, and the per-set tables it produces."""
import numpy as np
import pytest

from cosmosphere_b200 import autotune as at


def test_size_classes():
    assert at.size_class(1) == 0
    assert at.size_class(16383) == 13 and at.size_class(16384) == 14
    assert at.size_class(500_000) == 18
    with pytest.raises(ValueError):
        at.size_class(0)


def test_sample_spreads_over_the_class():
    sizes = list(range(1000, 21000, 1000))          # 20 sets, 210k particles
    members = list(range(20))
    assert at.sample_sets(sizes, members, 1e9) == members
    s = at.sample_sets(sizes, members, 50_000)
    assert 1 <= len(s) <= 5 and s[0] == 0 and s[-1] == 19
    assert at.sample_sets(sizes, [7], 10) == [7]
    assert at.sample_sets(sizes, [], 10) == []


def test_coordinate_descent_finds_the_separable_minimum():
    target = at.Tuning(bucket=32, list_margin=1.3, split_stream=8192, split_work=65536)

    def cost(t):
        return (abs(np.log2(t.bucket / target.bucket)) + abs(t.list_margin - target.list_margin)
                + abs(np.log2(t.split_stream / target.split_stream)) + abs(np.log2(t.split_work / target.split_work)))

    best, c, tried = at.coordinate_descent(cost)
    assert best == target and c == 0.0
    # one sweep: the start plus each parameter's other candidates, no setting twice
    assert len(tried) == len({t for t, _ in tried})
    assert len(tried) <= 1 + sum(len(v) - 1 for v in at.CANDIDATES.values())


def test_descent_keeps_the_default_when_nothing_is_faster():
    best, c, tried = at.coordinate_descent(lambda t: 1.0)
    assert best == at.DEFAULT and c == 1.0


def test_tune_builds_a_table_per_class_with_a_fake_timer():
    rng = np.random.default_rng(1)
    sizes = [3000, 5000, 70000, 90000, 12000]
    sets = [{"x": rng.random(n)} for n in sizes]
    calls = []

    def timer(sample, t, repeats):
        calls.append((tuple(len(s["x"]) for s in sample), t))
        n = sum(len(s["x"]) for s in sample)
        # small sets like small leaves, large ones large leaves
        return abs(np.log2(t.bucket) - (4 if n < 20000 else 7)) + 0.01 * t.list_margin

    table = at.tune(sets, timer=timer)
    assert set(table.entries) == {at.size_class(n) for n in sizes}
    assert table.for_size(3000).bucket == 16 and table.for_size(90000).bucket == 128
    assert table.for_size(3000).list_margin == 1.0
    per = table.per_set(sizes)
    assert per["bucket"].tolist() == [16, 16, 128, 128, 16]
    assert per["list_margin"].dtype == np.float64 and per["bucket"].dtype == np.int32
    # a class never tuned gets the default
    assert table.for_size(10**7) == at.DEFAULT
    for c, rec in table.times.items():
        assert rec["tuned_s"] <= rec["default_s"]


def test_table_round_trip(tmp_path):
    t = at.Table({14: at.Tuning(32, 1.05, 2048, 65536), 17: at.DEFAULT}, {14: {"tuned_s": 0.1}})
    f = tmp_path / "tune.json"
    t.save(f)
    u = at.Table.load(f)
    assert u.entries == t.entries and u.times == t.times


def test_apply_passes_per_set_arrays():
    class FakeBatch:
        sizes = [20000, 300000]

        def set_tuning(self, **kw):
            self.kw = kw

        def set_staging(self, on):
            self.staging = on

    b = FakeBatch()
    at.Table({at.size_class(300000): at.Tuning(bucket=128)}).apply(b)
    assert b.kw["bucket"].tolist() == [64, 128]
    assert b.kw["split_work"].tolist() == [131072, 131072]
    assert b.staging is False
    at.Table({}, staging=1).apply(b)
    assert b.staging is True


def test_confirm_keeps_the_faster_of_tuned_and_default():
    tuned = at.Table({14: at.Tuning(bucket=128)})
    times = {True: 1.0, False: 2.0}
    t, a, b = at.confirm([], tuned, timer=lambda sets, table, r: times[bool(table.entries)])
    assert t.entries == tuned.entries and t.staging == 0 and (a, b) == (1.0, 2.0)
    times = {True: 3.0, False: 2.0}
    t, a, b = at.confirm([], tuned, timer=lambda sets, table, r: times[bool(table.entries)])
    assert t.entries == {} and (a, b) == (3.0, 2.0)


def test_confirm_picks_the_batch_feed():
    tuned = at.Table({14: at.Tuning(bucket=128)})
    cost = {(True, 0): 2.0, (True, 1): 1.5, (False, 0): 2.5, (False, 1): 2.4}
    t, a, b = at.confirm([], tuned, timer=lambda sets, table, r: cost[(bool(table.entries), table.staging)])
    assert t.entries == tuned.entries and t.staging == 1 and (a, b) == (1.5, 2.4)
    t2 = at.Table.from_json(t.to_json())
    assert t2.staging == 1 and t2.entries == t.entries
