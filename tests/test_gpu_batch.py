"""Batched independent instances (nb_set_instances) and CUDA-graph stepping, on a GPU.

Each instance of a batch is an independent simulation with its own box, codes, tree and theta;
the batched pipeline runs one launch per phase over all of them. Every instance sees exactly the
operations of a standalone run in the same order, so results must match a standalone context
bit for bit: sorted codes, tree records, accelerations, interaction counts and trajectories.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 1e-4


def make_instances(nb, sizes, seed=0):
    rng = np.random.default_rng(seed)
    bodies, vels, thetas = [], [], []
    for k, n in enumerate(sizes):
        if k % 2:
            pm, vel = nb.scenarios.plummer(n, seed=1000 + k)
        else:
            pm, vel = nb.scenarios.uniform_ball(n, seed=2000 + k)
            vel[:, :3] = rng.normal(scale=0.1, size=(n, 3)).astype(np.float32)
        pm[:, :3] += np.float32(10.0 * k)  # instances far apart: any cross-talk would show
        bodies.append(pm)
        vels.append(vel)
        thetas.append(np.float32(rng.uniform(0.4, 0.7)))
    return bodies, vels, np.array(thetas, np.float32)


def standalone(nb, pm, vel, theta, order, steps=0):
    with nb.Solver(bodies=pm, rule=nb.Gravity(1.0, EPS), velocities=vel, order=order, theta=float(theta),
                   max_leaf_size=16, time_step=1e-3) as s:
        if steps:
            s.step(steps)
            return s.bodies()
        acc = s.update_accelerations()
        return acc, s.tree(), s.counts()


SIZES = [1, 17, 33, 1000, 4096, 5000, 16, 250, 12345, 2]


@pytest.mark.parametrize("order", [1, 2])
def test_batch_matches_standalone_bit_exact(nb, order):
    bodies, vels, thetas = make_instances(nb, SIZES, seed=order)
    with nb.Solver(order=order, rule=nb.Gravity(1.0, EPS), max_leaf_size=16, time_step=1e-3) as s:
        s.set_instances(SIZES, np.concatenate(bodies), np.concatenate(vels), thetas)
        acc = s.update_accelerations()
        t = s.tree()
        roots = s.instance_roots()
        counts = s.counts()
    starts = np.concatenate([[0], np.cumsum(SIZES)])
    rec = nb.decode_records(t["records"], order)
    tot_pp = tot_np = 0
    for k, n in enumerate(SIZES):
        a_ref, t_ref, c_ref = standalone(nb, bodies[k], vels[k], thetas[k], order)
        lo, hi = starts[k], starts[k + 1]
        assert np.array_equal(acc[lo:hi], a_ref), f"instance {k}"
        assert np.array_equal(t["codes"][lo:hi], t_ref["codes"])
        assert np.array_equal(t["ids"][lo:hi] - lo, t_ref["ids"])
        # the instance's subtree is its standalone tree, shifted in preorder and in body positions
        r0, nn = roots[k], t_ref["num_nodes"]
        sub = t["records"][r0:r0 + nn]
        ref = t_ref["records"]
        assert np.array_equal(sub[:, :4], ref[:, :4])      # MAC centre and threshold
        assert np.array_equal(sub[:, 8:], ref[:, 8:])      # centre of mass, mass, moments
        link = rec["link"][r0:r0 + nn]
        rlink = nb.decode_records(ref, order)["link"]
        leaf = rlink[:, 1] >= 0
        assert np.array_equal(link[leaf] - lo, rlink[leaf])
        assert np.array_equal(link[~leaf, 0] - r0, rlink[~leaf, 0])
        tot_pp += c_ref["particle_particle"]
        tot_np += c_ref["node_particle"]
    assert counts["particle_particle"] == tot_pp
    assert counts["node_particle"] == tot_np


def test_batch_steps_match_standalone(nb):
    sizes = [3000, 40, 777, 2048]
    bodies, vels, thetas = make_instances(nb, sizes, seed=5)
    with nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, EPS), max_leaf_size=16, time_step=1e-3) as s:
        s.set_instances(sizes, np.concatenate(bodies), np.concatenate(vels), thetas)
        s.enable_graphs(True)
        s.step(5)
        pm, vel = s.bodies()
    starts = np.concatenate([[0], np.cumsum(sizes)])
    for k in range(len(sizes)):
        p_ref, v_ref = standalone(nb, bodies[k], vels[k], thetas[k], 2, steps=5)
        assert np.array_equal(pm[starts[k]:starts[k + 1]], p_ref)
        assert np.array_equal(vel[starts[k]:starts[k + 1]], v_ref)


@pytest.mark.parametrize("steps", [1, 2, 3, 6])
def test_graph_steps_equal_plain_steps(nb, steps):
    pm, vel = nb.scenarios.plummer(20000, seed=71)
    out = []
    for graphs in (False, True):
        with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, EPS), theta=0.5,
                                          max_leaf_size=16, time_step=1e-3) as s:
            s.enable_graphs(graphs)
            s.step(steps)
            s.step(steps)  # a second call replays the captured graph
            out.append(s.bodies())
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_many_instances_two_instance_passes(nb):
    """More than 256 instances: the instance sort takes two 8-bit passes."""
    rng = np.random.default_rng(9)
    sizes = [int(x) for x in rng.integers(1, 60, size=300)]
    bodies, vels, thetas = make_instances(nb, sizes, seed=9)
    with nb.LinearBVHSolver(rule=nb.Gravity(1.0, EPS), max_leaf_size=8) as s:
        s.set_instances(sizes, np.concatenate(bodies), np.concatenate(vels), thetas)
        acc = s.update_accelerations()
    starts = np.concatenate([[0], np.cumsum(sizes)])
    for k in (0, 1, 150, 255, 256, 257, 299):
        with nb.LinearBVHSolver(bodies=bodies[k], rule=nb.Gravity(1.0, EPS), theta=float(thetas[k]),
                                max_leaf_size=8) as r:
            assert np.array_equal(acc[starts[k]:starts[k + 1]], r.update_accelerations())
