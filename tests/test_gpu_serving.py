"""Continuous-batching server (nb_server_*), on a GPU.

Requests arrive while others run, are admitted by a resident-memory budget, and advance together
in one batched force pass per tick. The check that matters for serving: each request's result is
the same alone and in the mix. The stated tolerance is zero: a request's arithmetic does not
depend on its batch-mates, so the final bodies must equal a standalone run bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 1e-4
DT = 1e-3


def alone(nb, pm, vel, theta, steps):
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, EPS), theta=theta,
                                      max_leaf_size=16, time_step=DT) as s:
        s.step(steps)
        return s.bodies()


def test_results_equal_alone_and_in_the_mix(nb):
    reqs = [(3000, 0.5, 4, 0), (777, 0.6, 7, 1), (5000, 0.45, 3, 1), (1, 0.5, 2, 2), (2500, 0.7, 5, 4)]
    data = []
    for k, (n, theta, steps, arrive) in enumerate(reqs):
        pm, vel = nb.scenarios.plummer(n, seed=300 + k)
        data.append((pm, vel, theta, steps, arrive))
    with nb.Server(rule=nb.Gravity(1.0, EPS), order=2, max_leaf_size=16, time_step=DT) as sv:
        ids = {}
        tick = 0
        while len(ids) < len(data) or any(sv.status(r)[0] != nb.Server.DONE for r in ids.values()):
            for k, (pm, vel, theta, steps, arrive) in enumerate(data):
                if arrive == tick and k not in ids:
                    ids[k] = sv.submit(pm, vel, theta=theta, steps=steps)
            sv.tick()
            tick += 1
            assert tick < 100
        stats = sv.stats()
        results = {k: sv.take_result(ids[k], len(data[k][0])) for k in ids}
    assert stats["completed"] == len(data) and stats["relayouts"] >= 3
    for k, (pm, vel, theta, steps, _) in enumerate(data):
        p_ref, v_ref = alone(nb, pm, vel, theta, steps)
        assert np.array_equal(results[k][0], p_ref), f"request {k}"
        assert np.array_equal(results[k][1], v_ref), f"request {k}"


def test_budget_admission_waits_for_memory(nb):
    pm1, v1 = nb.scenarios.plummer(4000, seed=1)
    pm2, v2 = nb.scenarios.plummer(3000, seed=2)
    budget = 4500 * 544  # room for one request at a time
    with nb.Server(rule=nb.Gravity(1.0, EPS), hbm_budget_bytes=budget, time_step=DT) as sv:
        a = sv.submit(pm1, v1, theta=0.5, steps=3)
        b = sv.submit(pm2, v2, theta=0.5, steps=2)
        sv.tick()
        assert sv.status(a)[0] == nb.Server.RUNNING and sv.status(b)[0] == nb.Server.QUEUED
        while sv.status(b)[0] != nb.Server.DONE:
            sv.tick()
        assert sv.status(a)[0] == nb.Server.DONE
        ra = sv.take_result(a, 4000)
        rb = sv.take_result(b, 3000)
        with pytest.raises(nb.NBodyError):
            sv.submit(np.zeros((10000, 4), np.float32), steps=1)  # larger than the whole budget
    assert np.array_equal(ra[0], alone(nb, pm1, v1, 0.5, 3)[0])
    assert np.array_equal(rb[0], alone(nb, pm2, v2, 0.5, 2)[0])


def test_zero_step_request_returns_its_input(nb):
    pm, vel = nb.scenarios.uniform_ball(100, seed=3)
    with nb.Server(rule=nb.Gravity(1.0, EPS)) as sv:
        r = sv.submit(pm, vel, steps=0)
        sv.tick()
        out = sv.take_result(r, 100)
    assert np.array_equal(out[0], pm) and np.array_equal(out[1], vel)


def test_rejects_non_finite_input(nb):
    pm, vel = nb.scenarios.plummer(100, seed=4)
    with nb.Server(rule=nb.Gravity(1.0, EPS), time_step=DT) as sv:
        bad = pm.copy()
        bad[7, 1] = np.nan
        with pytest.raises(nb.NBodyError):
            sv.submit(bad, vel, steps=1)
        badv = vel.copy()
        badv[3, 0] = np.inf
        with pytest.raises(nb.NBodyError):
            sv.submit(pm, badv, steps=1)
        assert sv.stats()["submitted"] == 0


def test_cancel_queued_and_running(nb):
    sizes = [3000, 2000, 1500]
    data = [nb.scenarios.plummer(n, seed=50 + k) for k, n in enumerate(sizes)]
    with nb.Server(rule=nb.Gravity(1.0, EPS), time_step=DT, hbm_budget_bytes=(3000 + 2000) * 544) as sv:
        a = sv.submit(*data[0], theta=0.5, steps=4)
        b = sv.submit(*data[1], theta=0.5, steps=4)
        c = sv.submit(*data[2], theta=0.5, steps=3)  # waits for memory
        sv.tick()
        assert sv.status(c)[0] == nb.Server.QUEUED
        sv.cancel(c)  # queued: gone at once
        with pytest.raises(nb.NBodyError):
            sv.status(c)
        sv.cancel(b)  # running: dropped from the layout at the next tick
        while sv.status(a)[0] != nb.Server.DONE:
            sv.tick()
        with pytest.raises(nb.NBodyError):
            sv.status(b)
        st = sv.stats()
        ra = sv.take_result(a, sizes[0])
    assert st["cancelled"] == 2 and st["completed"] == 1
    assert np.array_equal(ra[0], alone(nb, *data[0], 0.5, 4)[0])


@pytest.mark.parametrize("point", [0, 1])
def test_allocation_failure_keeps_server_consistent(nb, point):
    """An allocation failure during a re-layout (injected on the host) fails that tick; the server
    stays consistent, and once memory is available again every request still ends bit-identical
    to a standalone run."""
    small = [nb.scenarios.plummer(n, seed=70 + k) for k, n in enumerate([800, 600])]
    big = nb.scenarios.plummer(9000, seed=79)  # needs larger staging and context buffers
    with nb.Server(rule=nb.Gravity(1.0, EPS), time_step=DT) as sv:
        ids = [sv.submit(*small[0], theta=0.5, steps=5), sv.submit(*small[1], theta=0.6, steps=5)]
        sv.tick()
        sv.tick()
        sv.inject_alloc_failures(point, 1)
        ids.append(sv.submit(*big, theta=0.5, steps=3))
        with pytest.raises(nb.NBodyError):
            sv.tick()
        st = sv.stats()
        assert st["failed_ticks"] == 1
        if point == 0:
            assert sv.status(ids[2])[0] == nb.Server.QUEUED  # put back, nothing laid out
        else:
            assert sv.status(ids[2])[0] == nb.Server.RUNNING  # staged; loaded at the next tick
        guard = 0
        while any(sv.status(r)[0] != nb.Server.DONE for r in ids):
            sv.tick()
            guard += 1
            assert guard < 50
        results = [sv.take_result(r, n) for r, n in zip(ids, [800, 600, 9000])]
    refs = [alone(nb, *small[0], 0.5, 5), alone(nb, *small[1], 0.6, 5), alone(nb, *big, 0.5, 3)]
    for (p, v), (pr, vr) in zip(results, refs):
        assert np.array_equal(p, pr) and np.array_equal(v, vr)
