"""The radix sort's bounded look-back wait, run out on purpose (nb_selftest_bounded_wait).

A pass whose predecessor tile never publishes its counts waits on a flag that nothing sets; the
wait is bounded by a timer, so the kernel sets its error bit and returns, the host reads
NB_ERR_DEVICE_TIMEOUT, and the device keeps working. Every index of that pass stays inside its
buffers, so nothing faults: only the wait's limit is exercised.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_lookback_wait_runs_out_and_reports(nb):
    t0 = time.perf_counter()
    rc = nb.lib().nb_selftest_bounded_wait(0, 50)
    elapsed = time.perf_counter() - t0
    assert rc == nb.NB_ERR_DEVICE_TIMEOUT, rc
    assert elapsed < 10.0  # the kernel returned at its limit (plus set-up), it did not hang
    # the device is still usable: a normal force pass afterwards gives the usual counts
    pm, _ = nb.scenarios.plummer(5000, seed=3)
    with nb.LinearBVHSolver(bodies=pm, rule=nb.Gravity(1.0, 1e-4), theta=0.5, max_leaf_size=16) as s:
        acc = s.update_accelerations()
        assert np.all(np.isfinite(acc)) and s.counts()["particle_particle"] > 0


def test_selftest_rejects_bad_limits(nb):
    assert nb.lib().nb_selftest_bounded_wait(0, 0) == nb.NB_ERR_INVALID_ARGUMENT
    assert nb.lib().nb_selftest_bounded_wait(0, 5000) == nb.NB_ERR_INVALID_ARGUMENT
