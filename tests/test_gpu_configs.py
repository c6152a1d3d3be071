"""The batched, served and dual-tree rows checked against the oracle at their own configurations,
on a GPU (the other GPU tests compare these paths with the standalone GPU solver; these feed the
same instances straight to the oracle).

- Batched: 256 Plummer instances, N log-uniform in [1024, 200000], theta uniform in [0.4, 0.7] per
  instance, softening 0.01, quadrupole, the leaf size the autotuner picks for the batch. Each
  checked instance matches ActiveTreeSolver::updateAccelerations (ActiveTreeSolver.h:33-72) run
  by the oracle on that instance alone with its own theta.
- Served: requests of different sizes and thetas admitted while others run; each result after k
  steps matches the oracle stepping the request alone (accelerations, then kick-drift,
  Solver.h:103-139).
- Dual tree: two Hernquist spheres of 2^21 bodies each, theta 0.4, field order 4
  (ImplicitDualTraversalSolver.h:42-69): FP64 error on a seeded 65,536-body subsample, repeatable
  results, and exact interaction counts against the oracle on the same scene at 2 x 65,536 bodies.

Tolerances: accelerations sum the same interactions as the oracle in another order (rsqrt instead
of sqrt and division, FP32 sums in another order), so the relative error per target is bounded by
RMS 2e-6 and max 1e-4, as in the single-instance parity tests; counts are exact.
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

ACC_RMS_TOL = 2e-6
ACC_MAX_TOL = 1e-4
ORACLE_ALL_TARGETS = 40000  # instances up to this size are checked on every target, counts included


def _check_acc(got, ref):
    e = rel_err(got, ref)
    assert np.sqrt(np.mean(e ** 2)) < ACC_RMS_TOL, np.sqrt(np.mean(e ** 2))
    assert e.max() < ACC_MAX_TOL, e.max()


def test_batched_configuration_matches_oracle(nb, oracle):
    sizes, thetas, bodies, vels = nb.scenarios.batched_plummer(256, seed=44)
    eps = nb.scenarios.softening_to_epsilon(0.01)
    with nb.QuadrupoleLinearBVHSolver(rule=nb.Gravity(1.0, eps), max_leaf_size=16, time_step=5e-4) as s:
        s.set_instances(sizes, np.concatenate(bodies), np.concatenate(vels), thetas)
        leaf = s.autotune(candidates=(8, 12, 16), passes=1).leaf
        acc = s.update_accelerations()
        inst_counts = s.instance_counts()
        total = s.counts()
    assert int(inst_counts[:, 0].sum()) == total["particle_particle"]
    assert int(inst_counts[:, 1].sum()) == total["node_particle"]
    starts = np.concatenate([[0], np.cumsum(sizes)])
    order = np.argsort(sizes)
    picks = sorted({int(order[0]), int(order[1]), int(order[64]), int(order[128]), int(order[200]), int(order[-1]), 0,
                    255})
    rng = np.random.default_rng(4400)
    checked_all = 0
    for k in picks:
        pm = bodies[k]
        got = acc[starts[k]:starts[k + 1]]
        th = float(thetas[k])
        if len(pm) <= ORACLE_ALL_TARGETS:
            ref, rc = oracle.bh_accelerations(pm, eps=eps, theta=th, leaf=leaf, order=2)
            assert int(inst_counts[k, 0]) == int(rc[0]), (k, inst_counts[k], rc)
            assert int(inst_counts[k, 1]) == int(rc[1]), (k, inst_counts[k], rc)
            _check_acc(got, ref)
            checked_all += 1
        else:  # the largest instances: a seeded subsample of targets
            idx = np.sort(rng.choice(len(pm), 4096, replace=False))
            ref, _ = oracle.bh_targets(pm, pm[idx], eps=eps, theta=th, leaf=leaf, order=2)
            _check_acc(got[idx], ref)
    assert checked_all >= 4
    assert sizes[order[-1]] > 150000  # the largest instance was among the checked ones


def test_served_requests_match_oracle_stepping(nb, oracle):
    """Requests of both scenario kinds, sizes and thetas, arriving while others run; each one's
    final bodies against the oracle stepping it alone."""
    dt = 5e-4
    eps = nb.scenarios.softening_to_epsilon(0.01)
    reqs = []  # (bodies, velocities, theta, steps, arrival tick)
    for k, (n, theta, steps, arrive) in enumerate([(2048, 0.4, 6, 0), (6000, 0.7, 4, 0), (3100, 0.55, 5, 1),
                                                    (9000, 0.45, 3, 2), (2500, 0.65, 7, 4)]):
        gen = nb.scenarios.plummer if k % 2 == 0 else nb.scenarios.uniform_ball
        pm, vel = gen(n, seed=900 + k)
        reqs.append((pm, vel, theta, steps, arrive))
    with nb.Server(rule=nb.Gravity(1.0, eps), order=2, max_leaf_size=16, time_step=dt) as sv:
        ids, tick = {}, 0
        while len(ids) < len(reqs) or any(sv.status(r)[0] != nb.Server.DONE for r in ids.values()):
            for k, (pm, vel, theta, steps, arrive) in enumerate(reqs):
                if arrive == tick and k not in ids:
                    ids[k] = sv.submit(pm, vel, theta=theta, steps=steps)
            sv.tick()
            tick += 1
            assert tick < 100
        results = {k: sv.take_result(ids[k], len(reqs[k][0])) for k in ids}
    for k, (pm, vel, theta, steps, _) in enumerate(reqs):
        p, v = pm.copy(), vel.copy()
        for _ in range(steps):
            a, _ = oracle.bh_accelerations(p, eps=eps, theta=theta, leaf=16, order=2)
            p, v = oracle.kick_drift(p, v, a, np.float32(dt))
        gp, gv = results[k]
        assert np.array_equal(gp[:, 3], pm[:, 3])
        assert np.abs(gp[:, :3] - p[:, :3]).max() < 1e-5 * np.abs(p[:, :3]).max(), k
        assert np.abs(gv[:, :3] - v[:, :3]).max() < 1e-4 * np.abs(v[:, :3]).max(), k


DUAL_THETA = 0.4
DUAL_LEAF = 64


def test_dual_tree_configuration(nb, oracle):
    torch = pytest.importorskip("torch")
    eps = nb.scenarios.softening_to_epsilon(0.005)
    # exact counts on the same scene at 2 x 65,536 bodies, where the oracle takes every target
    small, _ = nb.scenarios.colliding_hernquist(1 << 16, seed=146)
    with nb.OctupoleImplicitLinearBVHFMMSolver(bodies=small, rule=nb.Gravity(1.0, eps), theta=DUAL_THETA,
                                               max_leaf_size=DUAL_LEAF) as s:
        acc_small = s.update_accelerations()
        c = s.counts()
    ref, rc = oracle.dual_accelerations(small, eps=eps, theta=DUAL_THETA, leaf=DUAL_LEAF, order=3)
    got = [c["particle_particle"], c["node_particle"], c["particle_node"], c["node_node"]]
    assert got == [int(x) for x in rc], (got, rc)
    e = rel_err(acc_small, ref)
    assert np.sqrt(np.mean(e ** 2)) < 5e-6 and e.max() < 5e-4
    # the full scene: 2 x 2^21 bodies
    pm, vel = nb.scenarios.colliding_hernquist(1 << 21, seed=46)
    n = len(pm)
    with nb.OctupoleImplicitLinearBVHFMMSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, eps),
                                               theta=DUAL_THETA, max_leaf_size=DUAL_LEAF) as s:
        s.set_fp64_summaries(65536)  # the configuration's FP64 root-level moments
        a1 = s.update_accelerations()
        c1 = s.counts()
        a2 = s.update_accelerations()
        c2 = s.counts()
        rng = np.random.default_rng(65536)
        idx = np.sort(rng.choice(n, 65536, replace=False))
        dpm = torch.from_numpy(pm).cuda()
        dtg = torch.from_numpy(pm[idx].copy()).cuda()
        out = torch.zeros((len(idx), 3), dtype=torch.float64, device="cuda")
        s.direct_device(n, dpm.data_ptr(), len(idx), dtg.data_ptr(), out.data_ptr(), 64)
        s.synchronize()
        exact = out.cpu().numpy()
    assert np.array_equal(a1, a2) and c1 == c2  # repeatable, bit for bit
    rel = np.linalg.norm(a1[idx, :3].astype(np.float64) - exact, axis=1) / np.linalg.norm(exact, axis=1)
    assert np.sqrt(np.mean(rel ** 2)) <= 1e-4, np.sqrt(np.mean(rel ** 2))
    assert c1["particle_particle"] > 0 and c1["node_node"] > 0
