"""Parity of the CUDA force path with the oracle, through the C ABI (needs an sm_100 GPU).

Bit-exact: global bounding box, Morton codes, sort permutation (ties by input index), tree
topology, node centres of mass, masses, quadrupole moments, bounding-box centres, the MAC
thresholds, and the interaction counts (so every target takes exactly the reference's
approximate/open decisions).
Within tolerance: accelerations. They differ from the oracle only by the interaction kernels'
rsqrt and summation order; the bound is stated per test (relative to |a| per target).
"""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu

# Acceleration tolerance vs the oracle (same interactions, same node data, FP32 rsqrt + sum order).
ACC_RMS_TOL = 2e-6
ACC_MAX_TOL = 1e-4


def make_solver(nb, pm, order=1, leaf=16, theta=0.5, eps=1e-4, G=1.0, vel=None, solver=None):
    cls = solver or (nb.LinearBVHSolver if order == 1 else nb.QuadrupoleLinearBVHSolver)
    return cls(bodies=pm, rule=nb.Gravity(G, eps), velocities=vel, theta=theta, max_leaf_size=leaf)


def oracle_tree(oracle, pm, leaf, order):
    box = oracle.bbox(pm)
    codes = oracle.morton_codes(pm, box)
    perm = oracle.sort_codes(codes)
    sc = codes[perm]
    tree = oracle.build_tree(sc, leaf)
    bb, cm, mo = oracle.summarize(tree, pm[perm], order)
    return box, codes, perm, sc, tree, bb, cm, mo


def check_tree(nb, oracle, s, pm, leaf, order, theta):
    t = s.tree()
    box, codes, perm, sc, tree, bb, cm, mo = oracle_tree(oracle, pm, leaf, order)
    assert np.array_equal(t["bbox"], box)
    assert np.array_equal(t["codes"], sc)
    assert np.array_equal(t["ids"], perm)
    b, e, l, r = tree
    assert t["num_nodes"] == len(b)
    rec = nb.decode_records(t["records"], order)
    link = rec["link"]
    leaf_mask = l < 0
    assert np.array_equal(link[:, 1] >= 0, leaf_mask)
    assert np.array_equal(link[leaf_mask, 0], b[leaf_mask])
    assert np.array_equal(link[leaf_mask, 1], e[leaf_mask])
    # internal nodes link their right child (the left child is the next node in preorder)
    assert np.array_equal(link[~leaf_mask, 0], r[~leaf_mask])
    assert np.all(l[~leaf_mask] == np.arange(len(b))[~leaf_mask] + 1)
    # summaries, bit-exact
    assert np.array_equal(rec["com"], cm[:, :3])
    assert np.array_equal(rec["mass"], cm[:, 3])
    center = ((bb[:, 3:6] + bb[:, 0:3]) / np.float32(2.0)).astype(np.float32)
    assert np.array_equal(rec["center"], center)
    if order == 2:
        assert np.array_equal(rec["quadrupole"], mo[:, :6])
    # MAC thresholds: the smallest d2 with diag2 / d2 < theta^2
    d = (bb[:, 3:6] - bb[:, 0:3]).astype(np.float32)
    diag2 = ((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]).astype(np.float32)
    tt = np.float32(theta) * np.float32(theta)
    thr = rec["mac_threshold"]
    ok = np.isfinite(thr)
    with np.errstate(divide="ignore", invalid="ignore"):
        assert np.all((diag2[ok] / thr[ok]) < tt)
        below = np.nextafter(thr[ok], np.float32(0))
        assert not np.any((below > 0) & ((diag2[ok] / below) < tt))
    return t


def check_accelerations(oracle, s, pm, acc, order, leaf, theta, eps, G=1.0, rms_tol=ACC_RMS_TOL,
                        max_tol=ACC_MAX_TOL):
    ref, counts = oracle.bh_accelerations(pm, G=G, eps=eps, theta=theta, leaf=leaf, order=order)
    c = s.counts()
    assert c["particle_particle"] == counts[0]
    assert c["node_particle"] == counts[1]
    err = rel_err(acc, ref)
    assert np.sqrt(np.mean(err ** 2)) < rms_tol, f"rms {np.sqrt(np.mean(err ** 2))}"
    assert err.max() < max_tol, f"max {err.max()}"
    assert np.all(acc[:, 3] == 0)


@pytest.mark.parametrize("order", [1, 2])
@pytest.mark.parametrize("n,leaf,theta", [(2000, 16, 0.5), (4097, 8, 0.3), (3000, 64, 0.7), (1500, 1, 0.5)])
def test_uniform_ball(nb, oracle, order, n, leaf, theta):
    pm, _ = nb.scenarios.uniform_ball(n, seed=7 + n)
    with make_solver(nb, pm, order=order, leaf=leaf, theta=theta) as s:
        acc = s.update_accelerations()
        check_tree(nb, oracle, s, pm, leaf, order, theta)
        check_accelerations(oracle, s, pm, acc, order, leaf, theta, 1e-4)


@pytest.mark.parametrize("order", [1, 2])
def test_plummer_sphere(nb, oracle, order):
    pm, _ = nb.scenarios.plummer(20000, seed=11)
    eps = nb.scenarios.softening_to_epsilon(0.005)
    with make_solver(nb, pm, order=order, leaf=16, theta=0.5, eps=eps) as s:
        acc = s.update_accelerations()
        check_tree(nb, oracle, s, pm, 16, order, 0.5)
        check_accelerations(oracle, s, pm, acc, order, 16, 0.5, eps)


@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 31, 33, 2047, 2048, 2049])
def test_small_and_ragged_sizes(nb, oracle, n):
    pm, _ = nb.scenarios.uniform_ball(n, seed=100 + n)
    for order in (1, 2):
        with make_solver(nb, pm, order=order, leaf=16, theta=0.5) as s:
            acc = s.update_accelerations()
            check_tree(nb, oracle, s, pm, 16, order, 0.5)
            check_accelerations(oracle, s, pm, acc, order, 16, 0.5, 1e-4)


def test_duplicate_positions(nb, oracle):
    """Equal Morton codes: leaves larger than maxLeafSize (LinearBVH.h:115-120), zero self terms."""
    rng = np.random.default_rng(5)
    base, _ = nb.scenarios.uniform_ball(300, seed=3)
    pm = np.concatenate([base, np.repeat(base[:7], 40, axis=0)])
    pm = pm[rng.permutation(len(pm))].copy()
    for order in (1, 2):
        with make_solver(nb, pm, order=order, leaf=4, theta=0.5) as s:
            acc = s.update_accelerations()
            check_tree(nb, oracle, s, pm, 4, order, 0.5)
            check_accelerations(oracle, s, pm, acc, order, 4, 0.5, 1e-4)


def test_all_bodies_coincident(nb, oracle):
    pm = np.tile(np.array([[0.25, -1.5, 3.0, 0.5]], np.float32), (1000, 1))
    with make_solver(nb, pm, order=2, leaf=16) as s:
        acc = s.update_accelerations()
        t = s.tree()
        assert t["num_nodes"] == 1
        assert np.all(t["codes"] == 0)
        assert np.array_equal(t["ids"], np.arange(1000))
        assert np.all(acc == 0)


def test_planar_and_degenerate_axes(nb, oracle):
    pm, _ = nb.scenarios.uniform_ball(5000, seed=9)
    pm[:, 2] = 0.0
    for order in (1, 2):
        with make_solver(nb, pm, order=order, leaf=16, theta=0.5) as s:
            acc = s.update_accelerations()
            check_tree(nb, oracle, s, pm, 16, order, 0.5)
            check_accelerations(oracle, s, pm, acc, order, 16, 0.5, 1e-4)


def test_theta_zero_is_direct_sum(nb, oracle):
    """theta = 0 never approximates: the tree solver reduces to the pairwise sum."""
    pm, _ = nb.scenarios.uniform_ball(3000, seed=21)
    with make_solver(nb, pm, order=2, leaf=16, theta=0.0) as s:
        acc = s.update_accelerations()
        c = s.counts()
        assert c["node_particle"] == 0 and c["particle_particle"] == 3000 * 3000
        ref = oracle.direct_f32(pm, eps=1e-4)
        err = rel_err(acc, ref)
        assert err.max() < 1e-4


def test_zero_softening(nb, oracle):
    """epsilon = 0: equal positions must contribute exactly nothing (Gravity.h:203)."""
    pm, _ = nb.scenarios.uniform_ball(4000, seed=23)
    for order in (1, 2):
        with make_solver(nb, pm, order=order, leaf=16, theta=0.5, eps=0.0) as s:
            acc = s.update_accelerations()
            assert np.all(np.isfinite(acc))
            check_accelerations(oracle, s, pm, acc, order, 16, 0.5, 0.0, max_tol=1e-3)


def near_origin_scene(nb, n, seed):
    """A ball with no body within 0.05 of the origin plus one body 1e-14 from it."""
    pm, _ = nb.scenarios.uniform_ball(n, seed=seed)
    pm = pm[np.linalg.norm(pm[:, :3].astype(np.float64), axis=1) > 0.05]
    extra = np.array([[1e-14, 0.0, 0.0, pm[0, 3]]], dtype=np.float32)
    return np.ascontiguousarray(np.concatenate([pm, extra]))


def test_zero_softening_target_near_origin(nb, oracle):
    """epsilon = 0 and a target 1e-14 from the origin: padding and masked terms stay exactly zero
    (no 0 * inf from a distance below 1e-13)."""
    pm = near_origin_scene(nb, 4000, 31)
    for order in (1, 2):
        with make_solver(nb, pm, order=order, leaf=16, theta=0.5, eps=0.0) as s:
            acc = s.update_accelerations()
            assert np.all(np.isfinite(acc))
            check_accelerations(oracle, s, pm, acc, order, 16, 0.5, 0.0, max_tol=1e-3)


def test_gravitational_constant(nb, oracle):
    pm, _ = nb.scenarios.uniform_ball(2500, seed=29)
    with make_solver(nb, pm, order=2, leaf=16, theta=0.5, G=2.5) as s:
        acc = s.update_accelerations()
        check_accelerations(oracle, s, pm, acc, 2, 16, 0.5, 1e-4, G=2.5)


def test_empty_body_set(nb):
    pm = np.zeros((0, 4), np.float32)
    with make_solver(nb, pm, order=2) as s:
        acc = s.update_accelerations()
        assert acc.shape == (0, 4)
        s.step(3)
        s.synchronize()


def test_naive_solver_matches_oracle(nb, oracle):
    pm, _ = nb.scenarios.plummer(6000, seed=31)
    with make_solver(nb, pm, solver=nb.NaiveSolver, eps=1e-4) as s:
        assert s.id() == "naive"
        acc = s.update_accelerations()
        ref = oracle.direct_f32(pm, eps=1e-4)
        err = rel_err(acc, ref)
        assert np.sqrt(np.mean(err ** 2)) < 2e-6 and err.max() < 1e-4


@pytest.mark.parametrize("order", [1, 2])
def test_steps_match_oracle_integrator(nb, oracle, order):
    """Solver::step = accelerations, v += a dt, x += v dt (Solver.h:103-139), three steps."""
    pm, vel = nb.scenarios.plummer(5000, seed=37)
    eps = 1e-4
    dt = 1e-3
    with make_solver(nb, pm, order=order, leaf=16, theta=0.5, eps=eps, vel=vel) as s:
        s.time_step = dt
        s.step(3)
        gpm, gvel = s.bodies()
    p, v = pm.copy(), vel.copy()
    for _ in range(3):
        a, _ = oracle.bh_accelerations(p, eps=eps, theta=0.5, leaf=16, order=order)
        p, v = oracle.kick_drift(p, v, a, dt)
    assert np.array_equal(gpm[:, 3], pm[:, 3])
    scale = np.abs(p[:, :3]).max()
    assert np.abs(gpm[:, :3] - p[:, :3]).max() < 1e-5 * scale
    assert np.abs(gvel[:, :3] - v[:, :3]).max() < 1e-5 * np.abs(v[:, :3]).max()


def test_kick_drift_bit_exact(nb, oracle):
    """With theta = 0 and one body per leaf the first kick-drift sees identical inputs."""
    pm, vel = nb.scenarios.uniform_ball(64, seed=41)
    vel[:, :3] = np.random.default_rng(1).normal(size=(64, 3)).astype(np.float32)
    with make_solver(nb, pm, solver=nb.NaiveSolver, eps=1e-4, vel=vel) as s:
        s.time_step = 0.01
        acc = s.update_accelerations()
        s2 = make_solver(nb, pm, solver=nb.NaiveSolver, eps=1e-4, vel=vel)
        s2.time_step = 0.01
        s2.step(1)
        gpm, gvel = s2.bodies()
        s2.close()
    p, v = oracle.kick_drift(pm, vel, acc, 0.01)
    assert np.array_equal(gvel[:, :3], v[:, :3])
    assert np.array_equal(gpm[:, :3], p[:, :3])


def test_set_config_between_steps(nb, oracle):
    pm, _ = nb.scenarios.uniform_ball(3000, seed=43)
    with make_solver(nb, pm, order=1, leaf=16, theta=0.5) as s:
        s.update_accelerations()
        s.theta = 0.8
        s.max_leaf_size = 32
        acc = s.update_accelerations()
        check_tree(nb, oracle, s, pm, 32, 1, 0.8)
        check_accelerations(oracle, s, pm, acc, 1, 32, 0.8, 1e-4)
        assert s.id() == "linear-bvh"


def test_device_direct_sum_f64(nb, oracle):
    torch = pytest.importorskip("torch")
    pm, _ = nb.scenarios.plummer(8192, seed=47)
    idx = np.arange(0, 8192, 7)
    dpm = torch.from_numpy(pm).cuda()
    dt = torch.from_numpy(pm[idx].copy()).cuda()
    out = torch.zeros((len(idx), 3), dtype=torch.float64, device="cuda")
    with make_solver(nb, pm[:1], eps=1e-4) as s:
        s.direct_device(len(pm), dpm.data_ptr(), len(idx), dt.data_ptr(), out.data_ptr(), 64)
        s.synchronize()
    # the device kernel widens the float epsilon of the rule; give the oracle the same value
    ref = oracle.direct_f64(pm, idx=idx, eps=float(np.float32(1e-4)))
    got = out.cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_repeatable(nb):
    pm, _ = nb.scenarios.plummer(30000, seed=53)
    with make_solver(nb, pm, order=2, leaf=16, theta=0.5) as s:
        a1 = s.update_accelerations()
        s.set_bodies(pm)
        a2 = s.update_accelerations()
    assert np.array_equal(a1, a2)


def test_energy_diagnostics_fp64(nb):
    """nb_energy: FP64 kinetic and softened potential energy of the current bodies, against numpy."""
    pm, vel = nb.scenarios.plummer(1500, seed=14)
    pm[10] = pm[11]  # a coincident pair is excluded, as the force excludes it
    eps, G = 1e-3, 1.7
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(G, eps)) as s:
        k, u = s.energy()
    p = pm[:, :3].astype(np.float64)
    m = pm[:, 3].astype(np.float64)
    d = p[None, :, :] - p[:, None, :]
    r2 = (d * d).sum(-1)
    same = r2 == 0.0
    inv = np.where(same, 0.0, 1.0 / np.sqrt(r2 + np.float64(np.float32(eps))))
    u_ref = -0.5 * np.float64(np.float32(G)) * (m[:, None] * m[None, :] * inv).sum()
    k_ref = 0.5 * (m * (vel[:, :3].astype(np.float64) ** 2).sum(1)).sum()
    assert abs(k - k_ref) <= 1e-12 * abs(k_ref)
    assert abs(u - u_ref) <= 1e-12 * abs(u_ref)


def test_energy_conserved_over_steps(nb):
    """Leapfrog-style kick-drift with the quadrupole tree: total energy drifts little over 50 steps."""
    pm, vel = nb.scenarios.plummer(20000, seed=15)
    eps = nb.scenarios.softening_to_epsilon(0.01)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, eps), theta=0.5,
                                      max_leaf_size=16, time_step=1e-3) as s:
        e0 = sum(s.energy())
        s.step(50)
        e1 = sum(s.energy())
    assert abs(e1 - e0) <= 1e-3 * abs(e0)


def test_config_c1_ten_steps(nb, oracle):
    """The 10,000-body uniform-ball configuration (monopole, leaf 16, theta 0.5, softening 0.01,
    dt 1e-3, 10 steps): trajectory against the oracle stepping with its own accelerations, and the
    interaction counts of the first pass exact."""
    pm, vel = nb.scenarios.uniform_ball(10000, seed=42)
    eps = nb.scenarios.softening_to_epsilon(0.01)
    with nb.LinearBVHSolver(bodies=pm, velocities=vel, rule=nb.Gravity(1.0, eps), theta=0.5, max_leaf_size=16,
                            time_step=1e-3) as s:
        s.update_accelerations()
        c = s.counts()
        s.step(10)
        gpm, gvel = s.bodies()
    a, rc = oracle.bh_accelerations(pm, eps=eps, theta=0.5, leaf=16, order=1)
    assert c["particle_particle"] == rc[0] and c["node_particle"] == rc[1]
    p, v = pm.copy(), vel.copy()
    for _ in range(10):
        a, _ = oracle.bh_accelerations(p, eps=eps, theta=0.5, leaf=16, order=1)
        p, v = oracle.kick_drift(p, v, a, np.float32(1e-3))
    assert np.abs(gpm[:, :3] - p[:, :3]).max() < 1e-5 * np.abs(p[:, :3]).max()
    assert np.abs(gvel[:, :3] - v[:, :3]).max() < 1e-4 * np.abs(v[:, :3]).max()


@pytest.mark.parametrize("cls_name,n,theta,leaf", [
    ("QuadrupoleLinearBVHSolver", 20000, 0.5, 16),
    ("LinearBVHSolver", 9000, 0.5, 16),
    ("OctupoleImplicitLinearBVHFMMSolver", 30000, 0.4, 64),
])
def test_fp64_top_level_summaries(nb, cls_name, n, theta, leaf):
    """The precision option (nb_set_fp64_summaries): bounding boxes and so every decision and
    interaction count stay the reference's; the FP64-combined moments move the accelerations by
    rounding only, and turning the option off restores the FP32 results bit for bit."""
    pm, _ = nb.scenarios.plummer(n, seed=31)
    eps = 1e-4
    with getattr(nb, cls_name)(bodies=pm, rule=nb.Gravity(1.0, eps), theta=theta, max_leaf_size=leaf) as s:
        a32 = s.update_accelerations()[:, :3].astype(np.float64)
        c32 = s.counts()
        s.set_fp64_summaries(1)
        a64 = s.update_accelerations()[:, :3].astype(np.float64)
        c64 = s.counts()
        s.set_fp64_summaries(0)
        again = s.update_accelerations()[:, :3].astype(np.float64)
    assert c64 == c32
    assert np.array_equal(again, a32)
    rel = np.linalg.norm(a64 - a32, axis=1) / np.linalg.norm(a32, axis=1)
    assert np.sqrt(np.mean(rel ** 2)) < 1e-5
    assert not np.array_equal(a64, a32)  # the option does change the top-level moments
