"""Leaf-size autotuning on the device: the measurement leaves the state untouched and the chosen
leaf size gives the same results as a context configured with it directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_plain_keeps_state(nb, tmp_path):
    from nbody_b200 import autotune as at

    pm, vel = nb.scenarios.plummer(50000, seed=3)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, 1e-4), theta=0.5) as s:
        r = s.autotune(cache=at.TuningCache(str(tmp_path / "t.json")), candidates=(8, 16), passes=1)
        assert r.leaf in (8, 16) and s.max_leaf_size == r.leaf
        assert set(r.timings_ms) == {8, 16} and all(t > 0 for t in r.timings_ms.values())
        p, v = s.bodies()
        assert np.array_equal(p, pm) and np.array_equal(v, vel)
        acc = s.update_accelerations()
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, 1e-4), theta=0.5,
                                      max_leaf_size=r.leaf) as ref:
        assert np.array_equal(acc, ref.update_accelerations())


def test_autotune_batch(nb):
    sizes = [3000, 20000, 700, 12000]
    bodies = [nb.scenarios.plummer(n, seed=10 + k)[0] for k, n in enumerate(sizes)]
    with nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, 1e-4)) as s:
        s.set_instances(sizes, np.concatenate(bodies))
        r = s.autotune(candidates=(6, 12, 24), passes=1)
        assert r.leaf in (6, 12, 24) and r.key.endswith("theta0.30") and "|i2^2|" in r.key
        acc = s.update_accelerations()
    with nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, 1e-4), max_leaf_size=r.leaf) as ref:
        ref.set_instances(sizes, np.concatenate(bodies))
        assert np.array_equal(acc, ref.update_accelerations())
