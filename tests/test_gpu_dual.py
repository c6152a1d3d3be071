"""Parity of the dual-tree solver (MultipoleImplicitLinearBVHFMMSolver<3>) with the oracle, through
the C ABI (needs an sm_100 GPU).

Bit-exact: the octupole tree (boxes, body counts, diagonal lengths, centres of mass, masses,
quadrupole and octupole moments, links) and the interaction counts (particle-particle,
node-particle, particle-node, node-node), so the device takes exactly the reference's
loadBalancedBreak split, balanced start lists, lock-step / passive-tree decisions and activeTree
walks.
Within tolerance: accelerations. They sum the same interactions as the oracle in another order
(block reductions of partial local fields and near-field sums); the bound is stated per test,
relative to |a| per body.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

# Same interactions, same node data; FP32 sums in a different order.
ACC_RMS_TOL = 5e-6
ACC_MAX_TOL = 5e-4


def dual_solver(nb, pm, leaf=64, theta=0.4, eps=1e-4, G=1.0, vel=None):
    return nb.OctupoleImplicitLinearBVHFMMSolver(bodies=pm, rule=nb.Gravity(G, eps), velocities=vel, theta=theta,
                                                 max_leaf_size=leaf)


def two_spheres(nb, n, seed):
    """Two Hernquist spheres on a collision course (the dual-tree benchmark scene, scaled down)."""
    a, va = nb.scenarios.hernquist(n // 2, seed=seed)
    b, vb = nb.scenarios.hernquist(n - n // 2, seed=seed + 1)
    a[:, 0] -= np.float32(1.5)
    b[:, 0] += np.float32(1.5)
    va[:, 0] += np.float32(0.2)
    vb[:, 0] -= np.float32(0.2)
    return np.concatenate([a, b]), np.concatenate([va, vb])


def check_dual_tree(nb, oracle, s, pm, leaf):
    t = s.tree()
    box = oracle.bbox(pm)
    codes = oracle.morton_codes(pm, box)
    perm = oracle.sort_codes(codes)
    assert np.array_equal(t["codes"], codes[perm])
    assert np.array_equal(t["ids"], perm)
    tree = oracle.build_tree(codes[perm], leaf)
    bb, cm, mo = oracle.summarize(tree, pm[perm], 3)
    b, e, l, r = tree
    assert t["num_nodes"] == len(b)
    rec = nb.decode_dual_records(t["records"])
    assert np.array_equal(rec["bmin"], bb[:, 0:3])
    assert np.array_equal(rec["bmax"], bb[:, 3:6])
    assert np.array_equal(rec["size"], e - b)
    d = (bb[:, 3:6] - bb[:, 0:3]).astype(np.float32)
    diag = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32)
    assert np.array_equal(rec["diag"], diag)
    assert np.array_equal(rec["com"], cm[:, :3])
    assert np.array_equal(rec["mass"], cm[:, 3])
    assert np.array_equal(rec["quadrupole"], mo[:, 0:6])
    assert np.array_equal(rec["octupole"], mo[:, 6:16])
    leaf_mask = l < 0
    link = rec["link"]
    assert np.array_equal(link[leaf_mask, 0], b[leaf_mask])
    assert np.array_equal(link[leaf_mask, 1], e[leaf_mask])
    assert np.array_equal(link[~leaf_mask, 0], r[~leaf_mask])
    assert np.array_equal(link[~leaf_mask, 1], -1 - b[~leaf_mask])


def check_against_oracle(nb, oracle, pm, leaf, theta, eps=1e-4, G=1.0, tree=True):
    with dual_solver(nb, pm, leaf=leaf, theta=theta, eps=eps, G=G) as s:
        assert s.id() == "implicit-linear-bvh-fmm-8p"
        acc = s.update_accelerations()
        counts = s.counts()
        if tree:
            check_dual_tree(nb, oracle, s, pm, leaf)
    ref, rc = oracle.dual_accelerations(pm, G=G, eps=float(np.float32(eps)), theta=theta, leaf=leaf, order=3)
    got = [counts["particle_particle"], counts["node_particle"], counts["particle_node"], counts["node_node"]]
    assert got == [int(x) for x in rc], (got, rc)
    err = rel_err(acc, ref)
    assert np.sqrt(np.mean(err ** 2)) <= ACC_RMS_TOL, np.sqrt(np.mean(err ** 2))
    assert err.max() <= ACC_MAX_TOL, err.max()
    return acc, counts


@pytest.mark.parametrize("n,leaf,theta", [(20000, 64, 0.4), (30000, 16, 0.5), (12000, 32, 0.7)])
def test_dual_uniform_ball(nb, oracle, n, leaf, theta):
    pm, _ = nb.scenarios.uniform_ball(n, seed=n)
    _, c = check_against_oracle(nb, oracle, pm, leaf, theta)
    assert c["node_node"] > 0 and c["particle_node"] > 0 and c["node_particle"] > 0


def test_dual_plummer(nb, oracle):
    pm, _ = nb.scenarios.plummer(40000, seed=3)
    check_against_oracle(nb, oracle, pm, 64, 0.4)


def test_dual_two_hernquist_spheres(nb, oracle):
    pm, _ = two_spheres(nb, 50000, seed=11)
    check_against_oracle(nb, oracle, pm, 64, 0.4)


@pytest.mark.parametrize("n", [1, 2, 3, 33, 65, 257, 1000, 4097])
def test_dual_ragged_sizes(nb, oracle, n):
    pm, _ = nb.scenarios.plummer(n, seed=100 + n)
    check_against_oracle(nb, oracle, pm, 16, 0.5)


def test_dual_theta_zero_is_direct(nb, oracle):
    """theta = 0: nothing is approximated, every pair is evaluated directly."""
    pm, _ = nb.scenarios.uniform_ball(3000, seed=8)
    acc, c = check_against_oracle(nb, oracle, pm, 16, 0.0)
    assert c["particle_particle"] == 3000 * 3000
    assert c["node_particle"] == c["particle_node"] == c["node_node"] == 0


def test_dual_duplicates_and_coincident(nb, oracle):
    rng = np.random.default_rng(4)
    pm, _ = nb.scenarios.uniform_ball(6000, seed=4)
    pm[3000:4000] = pm[0]                    # a cluster of coincident bodies (one Morton code)
    pm[4000:4500, :3] = pm[4500:5000, :3]    # duplicated positions
    pm[:, 3] = rng.uniform(0.5, 1.5, len(pm)).astype(np.float32) / len(pm)
    check_against_oracle(nb, oracle, pm, 16, 0.5)


def test_dual_planar(nb, oracle):
    pm, _ = nb.scenarios.uniform_ball(8000, seed=5)
    pm[:, 2] = 0.0
    check_against_oracle(nb, oracle, pm, 32, 0.5)


def test_dual_G_and_softening(nb, oracle):
    pm, _ = nb.scenarios.plummer(10000, seed=6)
    check_against_oracle(nb, oracle, pm, 64, 0.4, eps=1e-3, G=2.5)


def test_dual_zero_softening_target_near_origin(nb, oracle):
    """epsilon = 0 and a target 1e-14 from the origin: the padding of partly filled pair tiles adds
    exactly zero (a massless source at the origin would give 0 * inf there)."""
    pm, _ = nb.scenarios.uniform_ball(12000, seed=32)
    pm = pm[np.linalg.norm(pm[:, :3].astype(np.float64), axis=1) > 0.05]
    pm = np.ascontiguousarray(np.concatenate([pm, np.array([[1e-14, 0.0, 0.0, pm[0, 3]]], dtype=np.float32)]))
    acc, _ = check_against_oracle(nb, oracle, pm, 64, 0.4, eps=0.0)
    assert np.all(np.isfinite(acc))


def test_dual_accuracy_vs_fp64(nb, oracle):
    """The dual-tree field against FP64 direct summation: RMS relative error well under 1e-3."""
    pm, _ = two_spheres(nb, 60000, seed=21)
    with dual_solver(nb, pm, leaf=64, theta=0.4) as s:
        acc = s.update_accelerations()
    idx = np.random.default_rng(0).choice(len(pm), 4096, replace=False)
    ref = oracle.direct_f64(pm, idx, eps=float(np.float32(1e-4)))
    err = rel_err(acc[idx], ref)
    assert np.sqrt(np.mean(err ** 2)) < 1e-4


def test_dual_repeatable(nb):
    pm, _ = nb.scenarios.plummer(30000, seed=7)
    with dual_solver(nb, pm) as s:
        a = s.update_accelerations()
        b = s.update_accelerations()
    assert np.array_equal(a, b)


def test_dual_step_is_kick_drift(nb, oracle):
    """nb_step with the dual solver: the accelerations of the current state, then the reference's
    kick-drift (bit-exact given those accelerations)."""
    pm, vel = two_spheres(nb, 20000, seed=31)
    with nb.OctupoleImplicitLinearBVHFMMSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, 1e-4), theta=0.4,
                                               max_leaf_size=64, time_step=5e-4) as s:
        acc = s.update_accelerations()
        s.step(1)
        p1, v1 = s.bodies()
    p_ref, v_ref = oracle.kick_drift(pm, vel, acc, np.float32(5e-4))
    assert np.array_equal(p1, p_ref)
    assert np.array_equal(v1, v_ref)


def test_dual_graph_steps_equal_plain(nb):
    pm, vel = two_spheres(nb, 20000, seed=41)
    out = []
    for graphs in (False, True):
        with nb.OctupoleImplicitLinearBVHFMMSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, 1e-4),
                                                   theta=0.4, max_leaf_size=64, time_step=5e-4) as s:
            s.enable_graphs(graphs)
            s.step(2)
            s.step(2)
            out.append(s.bodies())
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_dual_rejects_batches_and_other_orders(nb):
    pm, _ = nb.scenarios.plummer(100, seed=1)
    with pytest.raises(nb.NBodyError):
        nb.MultipoleImplicitLinearBVHFMMSolver(bodies=pm, order=2)
    with dual_solver(nb, pm) as s:
        with pytest.raises(nb.NBodyError):
            s.set_instances([50, 50], pm)


def test_dual_pool_growth_theta_zero(nb):
    """theta = 0 at N = 60000 asks for far more near-field roots than the initial pool holds: the
    context grows the pool and reruns the pass; the result is every pair, as the direct sum."""
    pm, _ = nb.scenarios.uniform_ball(60000, seed=12)
    with dual_solver(nb, pm, leaf=16, theta=0.0) as s:
        acc = s.update_accelerations()
        c = s.counts()
    assert c["particle_particle"] == 60000 * 60000
    assert c["node_particle"] == c["particle_node"] == c["node_node"] == 0
    with nb.NaiveSolver(bodies=pm, rule=nb.Gravity(1.0, 1e-4)) as d:
        ref = d.update_accelerations()
    err = rel_err(acc, ref)
    assert np.sqrt(np.mean(err ** 2)) < 1e-5
