"""Full-size checks of the force path (needs an sm_100 GPU): N = 2^20 Plummer sphere, quadrupole,
leaf 16, theta 0.5, softening 0.005 - the configuration the throughput metric is quoted on.

At this size the oracle evaluates a seeded subsample of targets against the full tree, and the
rest is checked through size-independent properties (sorted codes, a permutation, leaves that
tile the body range in order, force accuracy against the FP64 direct sum)."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

N = 1 << 20


@pytest.fixture(scope="module")
def plummer_1m(nb):
    pm, vel = nb.scenarios.plummer(N, seed=43)
    return pm, vel


def test_full_size_tree_properties_and_parity(nb, oracle, plummer_1m):
    pm, _ = plummer_1m
    eps = nb.scenarios.softening_to_epsilon(0.005)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, rule=nb.Gravity(1.0, eps), theta=0.5, max_leaf_size=16) as s:
        acc = s.update_accelerations()
        t = s.tree()
    codes, ids = t["codes"], t["ids"]
    assert np.all(codes[1:] >= codes[:-1])
    assert np.array_equal(np.sort(ids), np.arange(N, dtype=np.uint32))
    ref_codes = oracle.morton_codes(pm)
    assert np.array_equal(codes, ref_codes[ids])
    # ties keep input order
    same = codes[1:] == codes[:-1]
    assert np.all(ids[1:][same] > ids[:-1][same])
    rec = nb.decode_records(t["records"], 2)
    link = rec["link"]
    leaves = link[link[:, 1] >= 0]
    assert leaves[0, 0] == 0 and leaves[-1, 1] == N
    assert np.array_equal(leaves[1:, 0], leaves[:-1, 1])
    # oracle on a seeded target subsample against the full tree
    rng = np.random.default_rng(7)
    idx = np.sort(rng.choice(N, 2048, replace=False))
    ref, _ = oracle.bh_targets(pm, pm[idx], eps=eps, theta=0.5, leaf=16, order=2)
    err = rel_err(acc[idx], ref)
    assert np.sqrt(np.mean(err ** 2)) < 2e-6 and err.max() < 1e-4


def test_force_accuracy_vs_fp64(nb, plummer_1m):
    """The metric's accuracy bar: relative RMS force error <= 1e-3 against an FP64 direct sum."""
    torch = pytest.importorskip("torch")
    pm, _ = plummer_1m
    eps = nb.scenarios.softening_to_epsilon(0.005)
    rng = np.random.default_rng(11)
    idx = np.sort(rng.choice(N, 8192, replace=False))
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, rule=nb.Gravity(1.0, eps), theta=0.5, max_leaf_size=16) as s:
        acc = s.update_accelerations()
        dpm = torch.from_numpy(pm).cuda()
        dt = torch.from_numpy(pm[idx].copy()).cuda()
        out = torch.zeros((len(idx), 3), dtype=torch.float64, device="cuda")
        s.direct_device(N, dpm.data_ptr(), len(idx), dt.data_ptr(), out.data_ptr(), 64)
        s.synchronize()
    err = rel_err(acc[idx], out.cpu().numpy())
    rms = float(np.sqrt(np.mean(err ** 2)))
    assert rms <= 1e-3, rms
