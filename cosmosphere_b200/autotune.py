"""Autotuner of the batched form.

For each size class of particle set it finds the launch parameters that solve that
class fastest on this GPU: the leaf bucket (particles per leaf, which sets the i-groups
and j-tiles the density engine streams), the list margin (how far beyond the current
gather radius the j-leaf lists are walked, trading list length against rebuilds), and
the work cut (the gather stream above which a leaf's active particles are split over
several warps, and the candidate pairs each such warp takes).  The search is coordinate
descent over timed solves of a sample of the class's sets, each timed on the device
(`t_total`, CUDA events around the whole batched solve) and taken as the minimum of a
few repeats.

Beside the per-class parameters, the batch as a whole picks how the Newton kernel feeds
its j-stream -- loaded directly, or staged into shared memory by bulk copies
(`cp.async.bulk` on an mbarrier) -- by timing the whole batch both ways (one launch serves
every set, so this choice cannot differ by class).

None of the parameters changes a plain-FP64 result: every pair test is exact and each
particle's sums run over its accepted pairs in ascending j whatever the tree, the lists
or the cut, so a tuned solve returns the same h, rho and d(rho)/dh bit for bit.  In the
mixed form they change only how FP32 partial sums are grouped.

Host-only logic; the timed solves go through `capi.Batch`.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import asdict, dataclass, replace
from typing import Callable, Dict, Iterable, List, Sequence

import numpy as np

PARAMS = ("bucket", "list_margin", "split_stream", "split_work")

# Values the search may pick, per parameter; the defaults are the library's own.
CANDIDATES: Dict[str, tuple] = {
    "bucket": (16, 32, 64, 128, 256, 512),
    "list_margin": (1.0, 1.05, 1.15, 1.3),
    "split_stream": (2048, 4096, 8192, 16384),
    "split_work": (65536, 131072, 262144),
}


@dataclass(frozen=True)
class Tuning:
    bucket: int = 64
    list_margin: float = 1.15
    split_stream: int = 4096
    split_work: int = 131072


DEFAULT = Tuning()


def size_class(n: int) -> int:
    """Size class of a set of n particles: floor(log2 n) (n >= 1)."""
    if n < 1:
        raise ValueError("a set holds at least one particle")
    return int(math.floor(math.log2(n)))


def sample_sets(sizes: Sequence[int], members: Sequence[int], max_particles: float) -> List[int]:
    """Indices of a sample of a class's sets: spread evenly over the class sorted by size,
    as many as fit in max_particles (at least one)."""
    order = sorted(members, key=lambda k: (sizes[k], k))
    if not order:
        return []
    total = sum(sizes[k] for k in order)
    if total <= max_particles:
        return order
    mean = total / len(order)
    m = max(1, min(len(order), int(max_particles // max(mean, 1.0))))
    picks = np.linspace(0, len(order) - 1, m).round().astype(int)
    return sorted({order[int(p)] for p in picks}, key=lambda k: (sizes[k], k))


def coordinate_descent(cost: Callable[[Tuning], float], start: Tuning = DEFAULT,
                       candidates: Dict[str, tuple] = CANDIDATES, sweeps: int = 1):
    """Minimise cost over the candidate grid one parameter at a time (each sweep visits
    every parameter once, holding the others at their best so far).  Returns the best
    setting, its cost and every (setting, cost) evaluated (each setting at most once)."""
    seen: Dict[Tuning, float] = {}

    def ev(t: Tuning) -> float:
        if t not in seen:
            seen[t] = float(cost(t))
        return seen[t]

    best = start
    best_cost = ev(best)
    for _ in range(max(1, sweeps)):
        moved = False
        for p in PARAMS:
            for v in candidates[p]:
                t = replace(best, **{p: v})
                c = ev(t)
                if c < best_cost:
                    best, best_cost, moved = t, c, True
        if not moved:
            break
    return best, best_cost, list(seen.items())


class Table:
    """Tuned parameters per size class, with the default for classes never tuned."""

    def __init__(self, entries: Dict[int, Tuning] | None = None, times: Dict[int, dict] | None = None,
                 staging: int = 0):
        self.entries: Dict[int, Tuning] = dict(entries or {})
        self.times: Dict[int, dict] = dict(times or {})
        self.staging = int(staging)   # the batch's j-stream feed: 1 staged, 0 direct

    def for_size(self, n: int) -> Tuning:
        return self.entries.get(size_class(n), DEFAULT)

    def per_set(self, sizes: Iterable[int]) -> Dict[str, np.ndarray]:
        """The per-set arrays cosmo_batch_set_tuning takes, for sets of these sizes."""
        ts = [self.for_size(int(n)) for n in sizes]
        return {"bucket": np.array([t.bucket for t in ts], dtype=np.int32),
                "list_margin": np.array([t.list_margin for t in ts], dtype=np.float64),
                "split_stream": np.array([t.split_stream for t in ts], dtype=np.int32),
                "split_work": np.array([t.split_work for t in ts], dtype=np.int32)}

    def apply(self, batch) -> None:
        """Set every set of a capi.Batch to its class's parameters, and the batch's feed."""
        batch.set_tuning(**self.per_set(batch.sizes))
        batch.set_staging(bool(self.staging))

    def with_staging(self, staging: int) -> "Table":
        return Table(self.entries, self.times, staging)

    def to_json(self) -> dict:
        return {"classes": {str(k): asdict(v) for k, v in sorted(self.entries.items())},
                "times": {str(k): v for k, v in sorted(self.times.items())}, "staging": self.staging}

    @classmethod
    def from_json(cls, d: dict) -> "Table":
        ent = {int(k): Tuning(**v) for k, v in d.get("classes", {}).items()}
        return cls(ent, {int(k): v for k, v in d.get("times", {}).items()}, int(d.get("staging", 0)))

    def save(self, path: str | os.PathLike) -> None:
        with open(path, "w") as f:
            json.dump(self.to_json(), f, indent=1, sort_keys=True)

    @classmethod
    def load(cls, path: str | os.PathLike) -> "Table":
        with open(path) as f:
            return cls.from_json(json.load(f))


def solve_time(sets, tuning: Tuning, repeats: int = 2, final_rho: bool = True) -> float:
    """Device time (s) of the batched solve of these sets with one setting for all of
    them: the minimum over repeats, after one untimed solve."""
    from . import capi
    b = capi.Batch(sets)
    b.set_tuning(**asdict(tuning))
    b.upload()
    if b.density(final_rho=final_rho) != 0:
        return math.inf
    best = math.inf
    for _ in range(max(1, repeats)):
        b.upload()
        if b.density(final_rho=final_rho) != 0:
            return math.inf
        best = min(best, b.scalar("t_total"))
    return best


def batch_time(sets, table: "Table", repeats: int = 2, final_rho: bool = True) -> float:
    """Device time (s) of the batched solve of all these sets with a table's per-class
    parameters: the minimum over repeats, after one untimed solve."""
    from . import capi
    b = capi.Batch(sets)
    table.apply(b)
    b.upload()
    if b.density(final_rho=final_rho) != 0:
        return math.inf
    best = math.inf
    for _ in range(max(1, repeats)):
        b.upload()
        if b.density(final_rho=final_rho) != 0:
            return math.inf
        best = min(best, b.scalar("t_total"))
    return best


def confirm(sets, table: "Table", repeats: int = 2, timer: Callable = batch_time):
    """The tuned table or the defaults, each with the direct and the staged j-stream feed,
    whichever solves the whole batch fastest: the classes are tuned on samples solved
    alone, and a setting can lose a few percent once every set shares the GPU.  Returns
    (table, tuned seconds, default seconds), the seconds of each with its better feed."""
    times = {}
    for name, base in (("tuned", table), ("default", Table())):
        for st in (0, 1):
            times[(name, st)] = timer(sets, base.with_staging(st), repeats)
    t_tuned = min(times[("tuned", 0)], times[("tuned", 1)])
    t_default = min(times[("default", 0)], times[("default", 1)])
    name, st = min(times, key=lambda k: (times[k], k[0] != "tuned", k[1]))
    best = (table if name == "tuned" else Table()).with_staging(st)
    return best, t_tuned, t_default


def tune(sets, max_particles: float = 2.0e6, repeats: int = 2, sweeps: int = 1,
         candidates: Dict[str, tuple] = CANDIDATES, timer: Callable = solve_time,
         classes: Iterable[int] | None = None) -> Table:
    """Tune every size class present in sets (or only those listed in classes).  timer
    (sets, tuning, repeats) -> seconds is the timed solve; the precision is whatever
    cosmo_set_precision holds."""
    sizes = [int(np.asarray(s["x"]).size) for s in sets]
    by_class: Dict[int, List[int]] = {}
    for k, n in enumerate(sizes):
        by_class.setdefault(size_class(n), []).append(k)
    wanted = set(by_class) if classes is None else set(classes) & set(by_class)
    table = Table()
    for c in sorted(wanted):
        idx = sample_sets(sizes, by_class[c], max_particles)
        sample = [sets[k] for k in idx]
        best, cost, tried = coordinate_descent(lambda t: timer(sample, t, repeats), DEFAULT, candidates, sweeps)
        table.entries[c] = best
        table.times[c] = {"sets": len(idx), "particles": int(sum(sizes[k] for k in idx)),
                          "default_s": next(v for t, v in tried if t == DEFAULT), "tuned_s": cost,
                          "evaluated": len(tried)}
    return table
