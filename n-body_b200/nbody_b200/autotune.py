"""Autotuner for the device force path: leaf size, traversal block size and traversal tile.

Three knobs change the speed of a force pass and none changes its decisions or interaction
counts for a given leaf size:

- the leaf size (LinearBVH::maxLeafSize, LinearBVH.h:135-137) moves work between pair
  interactions and multipole terms: small leaves mean fewer pairs and more node terms;
- the traversal block size (128 or 256 threads per block of the persistent traversal grid);
- the traversal tile: how many partially accepted nodes each warp stages in shared memory before
  it evaluates them (32 or 64): larger tiles balance the lanes better, smaller ones flush sooner.

Which setting is fastest depends on N, theta, the distribution and, for batches, on the mix of
instance sizes, so it is measured, not modelled: the tuner runs force passes of the actual body
set (CUDA-event phase times: sort, build and traversal) and keeps the fastest. It searches the
leaf size first at the default launch shape, then the launch shapes at that leaf size. Force
passes do not advance the simulation, so tuning leaves the state unchanged.

Results are cached per workload signature (solver id, N and instance-count buckets, theta) in a
JSON file, so a later run with a similar workload reuses the choice without measuring.
"""
from __future__ import annotations

import json
import math
import os
from dataclasses import dataclass, field

DEFAULT_CANDIDATES = (4, 6, 8, 12, 16, 24, 32)
DEFAULT_SHAPES = ((256, 64), (256, 32), (128, 64), (128, 32))


@dataclass
class TuneResult:
    leaf: int
    timings_ms: dict = field(default_factory=dict)  # leaf size -> device ms per force pass
    key: str = ""
    cached: bool = False
    shape: tuple = (256, 64)                           # (threads per block, tile)
    shape_timings_ms: dict = field(default_factory=dict)  # "threads x tile" -> device ms per force pass


def workload_key(solver_id: str, n: int, instances: int, theta: float) -> str:
    """Bucketed workload signature: N and the instance count by powers of two, theta to 0.05."""
    nb = int(math.log2(max(n, 1)))
    ib = int(math.log2(max(instances, 1)))
    tb = round(float(theta) * 20) / 20
    return f"{solver_id}|n2^{nb}|i2^{ib}|theta{tb:.2f}"


class TuningCache:
    """Settings by workload key, kept in a JSON file (written on every store)."""

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
        """(leaf, shape) for the key, or None; entries written before shapes were tuned have the
        default shape."""
        e = self.entries.get(key)
        if e is None:
            return None
        return int(e["leaf"]), tuple(int(x) for x in e.get("shape", (256, 64)))

    def store(self, key: str, result: TuneResult):
        self.entries[key] = {"leaf": int(result.leaf), "shape": [int(x) for x in result.shape],
                             "timings_ms": {str(k): float(v) for k, v in result.timings_ms.items()},
                             "shape_timings_ms": {str(k): float(v) for k, v in result.shape_timings_ms.items()}}
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
    """Measure every candidate leaf size on the solver's current bodies and leave the best one set."""
    timings = {}
    for leaf in candidates:
        solver.max_leaf_size = int(leaf)
        timings[int(leaf)] = time_force_passes(solver, passes)
    leaf = select_leaf(timings, tolerance)
    solver.max_leaf_size = leaf
    return TuneResult(leaf=leaf, timings_ms=timings, shape=tuple(solver.traversal_shape))


def tune_shape(solver, shapes=DEFAULT_SHAPES, passes: int = 3):
    """Measure every traversal launch shape at the solver's current leaf size and leave the best
    one set. Returns (best shape, {"threads x tile": ms})."""
    timings = {}
    for shape in shapes:
        solver.traversal_shape = shape
        timings[tuple(shape)] = time_force_passes(solver, passes)
    best = min(timings, key=timings.get)
    solver.traversal_shape = best
    return best, {f"{t}x{e}": ms for (t, e), ms in timings.items()}


def autotune(solver, cache: TuningCache | None = None, candidates=DEFAULT_CANDIDATES, passes: int = 3,
             tolerance: float = 0.0, shapes=DEFAULT_SHAPES) -> TuneResult:
    """Set the solver's leaf size and traversal launch shape for its current bodies: from the cache
    when the workload signature is known, otherwise by measurement (and the result is cached)."""
    key = workload_key(solver.id(), solver.body_count(), solver.instance_count(), solver.theta)
    if cache is not None:
        hit = cache.lookup(key)
        if hit is not None:
            leaf, shape = hit
            solver.max_leaf_size = leaf
            solver.traversal_shape = shape
            return TuneResult(leaf=leaf, key=key, cached=True, shape=shape)
    solver.traversal_shape = (0, 0)  # the default shape while the leaf size is measured
    result = tune_leaf_size(solver, candidates, passes, tolerance)
    if shapes:
        result.shape, result.shape_timings_ms = tune_shape(solver, shapes, passes)
    result.key = key
    if cache is not None:
        cache.store(key, result)
    return result
