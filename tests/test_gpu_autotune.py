"""Autotuning on the device: the measurement leaves the state untouched, and the chosen leaf size
and traversal launch shape give the same results as a context configured with them directly.
Every launch shape takes the same decisions: interaction counts are equal across shapes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_plain_keeps_state(nb, tmp_path):
    from nbody_b200 import autotune as at

    pm, vel = nb.scenarios.plummer(50000, seed=3)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, 1e-4), theta=0.5) as s:
        r = s.autotune(cache=at.TuningCache(str(tmp_path / "t.json")), candidates=(8, 16), passes=1)
        assert r.leaf in (8, 16) and s.max_leaf_size == r.leaf
        assert s.traversal_shape == r.shape and len(r.shape_timings_ms) == 4
        assert set(r.timings_ms) == {8, 16} and all(t > 0 for t in r.timings_ms.values())
        p, v = s.bodies()
        assert np.array_equal(p, pm) and np.array_equal(v, vel)
        acc = s.update_accelerations()
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, 1e-4), theta=0.5,
                                      max_leaf_size=r.leaf) as ref:
        ref.traversal_shape = r.shape
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
        ref.traversal_shape = r.shape
        assert np.array_equal(acc, ref.update_accelerations())


@pytest.mark.parametrize("order", [1, 2])
def test_launch_shapes_take_the_same_decisions(nb, oracle, order):
    from conftest import rel_err

    pm, _ = nb.scenarios.plummer(30000, seed=17)
    ref, rc = oracle.bh_accelerations(pm, eps=1e-4, theta=0.5, leaf=16, order=order)
    with nb.Solver(bodies=pm, order=order, rule=nb.Gravity(1.0, 1e-4), theta=0.5, max_leaf_size=16) as s:
        for shape in [(256, 64), (256, 32), (128, 64), (128, 32)]:
            s.traversal_shape = shape
            acc = s.update_accelerations()
            c = s.counts()
            assert (c["particle_particle"], c["node_particle"]) == (int(rc[0]), int(rc[1])), shape
            e = rel_err(acc, ref)
            assert np.sqrt(np.mean(e ** 2)) < 2e-6 and e.max() < 1e-4, shape
        with pytest.raises(nb.NBodyError):
            s.traversal_shape = (192, 64)
