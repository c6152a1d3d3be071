"""Autotuner (nbody_b200/autotune.py): leaf size and traversal launch shape selection, workload keys
and the cache, driven by a fake solver on the CPU (the device path is exercised in
test_gpu_autotune)."""
import json

import pytest


class FakeSolver:
    """Solver-like object whose force-pass time depends on the leaf size."""

    def __init__(self, cost, n=100000, instances=1, theta=0.5, shape_cost=None):
        self.cost, self.n, self.inst, self._theta = cost, n, instances, theta
        self.shape_cost = shape_cost or (lambda shape: 0.0)
        self.shape = (256, 64)
        self.max_leaf_size = 16
        self.sets = []
        self._passes = 0
        self._timing = False
        self._ms = 0.0

    def id(self):
        return "linear-bvh-4p"

    def body_count(self):
        return self.n

    def instance_count(self):
        return self.inst

    @property
    def theta(self):
        return self._theta

    @property
    def traversal_shape(self):
        return self.shape

    @traversal_shape.setter
    def traversal_shape(self, shape):
        self.shape = (256, 64) if tuple(shape) == (0, 0) else tuple(shape)

    def __setattr__(self, k, v):
        if k == "max_leaf_size" and "sets" in self.__dict__:
            self.__dict__["sets"].append(v)
        object.__setattr__(self, k, v)

    def update_accelerations_async(self):
        if self._timing:
            self._passes += 1
            self._ms += self.cost(self.max_leaf_size) + self.shape_cost(self.shape)

    def synchronize(self):
        pass

    def enable_timing(self, on):
        self._timing = on
        self._passes = 0
        self._ms = 0.0

    def phase_times(self):
        return {"traverse_ms": self._ms, "sort_ms": 0.0, "passes": self._passes}


def test_picks_fastest_and_leaves_it_set(nb):
    from nbody_b200 import autotune as at

    s = FakeSolver(lambda leaf: abs(leaf - 8) + 10.0)
    r = at.tune_leaf_size(s, candidates=(4, 8, 16, 32), passes=2)
    assert r.leaf == 8 and s.max_leaf_size == 8
    assert r.timings_ms == {4: 14.0, 8: 10.0, 16: 18.0, 32: 34.0}
    assert s.sets[:4] == [4, 8, 16, 32]


def test_tolerance_prefers_larger_leaf(nb):
    from nbody_b200 import autotune as at

    assert at.select_leaf({4: 10.0, 8: 10.2, 16: 11.0}, tolerance=0.05) == 8
    assert at.select_leaf({4: 10.0, 8: 10.2, 16: 11.0}) == 4


def test_workload_key_buckets(nb):
    from nbody_b200 import autotune as at

    assert at.workload_key("linear-bvh-4p", 1 << 20, 1, 0.5) == "linear-bvh-4p|n2^20|i2^0|theta0.50"
    assert at.workload_key("linear-bvh-4p", (1 << 20) + 5, 1, 0.49) == at.workload_key("linear-bvh-4p", 1 << 20, 1, 0.5)
    assert at.workload_key("x", 9279659, 256, 0.55) == "x|n2^23|i2^8|theta0.55"


def test_cache_round_trip_and_reuse(nb, tmp_path):
    from nbody_b200 import autotune as at

    path = str(tmp_path / "t.json")
    cache = at.TuningCache(path)
    s = FakeSolver(lambda leaf: 100.0 / leaf + leaf)  # best at 8 or 12
    r = at.autotune(s, cache, candidates=(4, 8, 12, 16), passes=1)
    assert not r.cached and r.leaf in (8, 12)
    saved = json.load(open(path))
    assert saved[r.key]["leaf"] == r.leaf
    s2 = FakeSolver(lambda leaf: pytest.fail("a cached workload must not be measured again"))
    r2 = at.autotune(s2, at.TuningCache(path), candidates=(4, 8, 12, 16))
    assert r2.cached and r2.leaf == r.leaf and s2.max_leaf_size == r.leaf


def test_shape_tuned_after_leaf(nb, tmp_path):
    from nbody_b200 import autotune as at

    s = FakeSolver(lambda leaf: abs(leaf - 12) + 10.0, shape_cost=lambda sh: {(128, 32): -1.0}.get(sh, 0.0))
    cache = at.TuningCache(str(tmp_path / "t.json"))
    r = at.autotune(s, cache, candidates=(8, 12, 16), passes=1)
    assert r.leaf == 12 and r.shape == (128, 32) and s.traversal_shape == (128, 32)
    assert set(r.shape_timings_ms) == {"256x64", "256x32", "128x64", "128x32"}
    s2 = FakeSolver(lambda leaf: pytest.fail("cached"))
    r2 = at.autotune(s2, at.TuningCache(str(tmp_path / "t.json")), candidates=(8, 12, 16))
    assert r2.cached and r2.shape == (128, 32) and s2.traversal_shape == (128, 32) and s2.max_leaf_size == 12


def test_cache_entry_without_shape_reads_default(nb, tmp_path):
    from nbody_b200 import autotune as at

    path = tmp_path / "old.json"
    path.write_text(json.dumps({"k": {"leaf": 8, "timings_ms": {"8": 1.0}}}))
    assert at.TuningCache(str(path)).lookup("k") == (8, (256, 64))
