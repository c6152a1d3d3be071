"""Leaf-size autotuner for the device force path.

The leaf size (LinearBVH::maxLeafSize, LinearBVH.h:135-137) is the one free parameter that moves
work between pair interactions and node terms: small leaves mean fewer pairs and more multipole
terms. Which balance is fastest depends on N, theta, the distribution and, for batches, on the mix
of instance sizes, so it is measured, not modelled: the tuner runs force passes of the actual body
set at each candidate leaf size (CUDA-event phase times: sort, build and traversal) and keeps the
fastest. Force passes do not advance the simulation, so tuning leaves the state unchanged.

Results are cached per workload signature (solver id, N and instance-count buckets, theta) in a
JSON file, so a later run with a similar workload reuses the choice without measuring.

Block sizes and the traversal's 32-target tile are not tuned: the kernels size their grids from
the occupancy of the device (persistent grids, one warp per 32-target group).
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

DEFAULT_CANDIDATES = (4, 6, 8, 12, 16, 24, 32)


@dataclass
class TuneResult:
    leaf: int
    timings_ms: dict = field(default_factory=dict)  # leaf size -> device ms per force pass
    key: str = ""
    cached: bool = False


def workload_key(solver_id: str, n: int, instances: int, theta: float) -> str:
    """Bucketed workload signature: N and the instance count by powers of two, theta to 0.05."""
    nb = int(math.log2(max(n, 1)))
    ib = int(math.log2(max(instances, 1)))
    tb = round(float(theta) * 20) / 20
    return f"{solver_id}|n2^{nb}|i2^{ib}|theta{tb:.2f}"


class TuningCache:
    """Leaf sizes by workload key, kept in a JSON file (written on every store)."""

    def __init__(self, path: str | None = None):
        self.path = path or os.environ.get("NBODY_B200_TUNING") or os.path.join(
            os.path.expanduser("~"), ".cache", "nbody_b200", "tuning.json")
        self.entries = {}
        if os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    self.entries = json.load(f)
            except (OSError, ValueError):
                self.entries = {}

    def lookup(self, key: str):
        e = self.entries.get(key)
        return None if e is None else int(e["leaf"])

    def store(self, key: str, result: TuneResult):
        self.entries[key] = {"leaf": int(result.leaf),
                             "timings_ms": {str(k): float(v) for k, v in result.timings_ms.items()}}
        os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.entries, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def time_force_passes(solver, passes: int = 3) -> float:
    """Device milliseconds per force pass (all phases), after one untimed pass."""
    solver.update_accelerations_async()
    solver.synchronize()
    solver.enable_timing(True)
    for _ in range(passes):
        solver.update_accelerations_async()
    t = solver.phase_times()
    solver.enable_timing(False)
    return sum(v for k, v in t.items() if k.endswith("_ms")) / max(t["passes"], 1)


def select_leaf(timings_ms: dict, tolerance: float = 0.0) -> int:
    """The fastest candidate; with a tolerance, the largest leaf within (1 + tolerance) of it
    (larger leaves evaluate more pairs directly, so they are at least as accurate)."""
    best = min(timings_ms.values())
    ok = [leaf for leaf, t in timings_ms.items() if t <= best * (1.0 + tolerance)]
    return max(ok) if tolerance > 0 else min(timings_ms, key=timings_ms.get)


def tune_leaf_size(solver, candidates=DEFAULT_CANDIDATES, passes: int = 3, tolerance: float = 0.0) -> TuneResult:
    """Measure every candidate on the solver's current bodies and leave the best one set."""
    timings = {}
    for leaf in candidates:
        solver.max_leaf_size = int(leaf)
        timings[int(leaf)] = time_force_passes(solver, passes)
    leaf = select_leaf(timings, tolerance)
    solver.max_leaf_size = leaf
    return TuneResult(leaf=leaf, timings_ms=timings)


def autotune(solver, cache: TuningCache | None = None, candidates=DEFAULT_CANDIDATES, passes: int = 3,
             tolerance: float = 0.0) -> TuneResult:
    """Set the solver's leaf size for its current bodies: from the cache when the workload
    signature is known, otherwise by measurement (and the result is cached)."""
    key = workload_key(solver.id(), solver.body_count(), solver.instance_count(), solver.theta)
    if cache is not None:
        leaf = cache.lookup(key)
        if leaf is not None:
            solver.max_leaf_size = leaf
            return TuneResult(leaf=leaf, key=key, cached=True)
    result = tune_leaf_size(solver, candidates, passes, tolerance)
    result.key = key
    if cache is not None:
        cache.store(key, result)
    return result
