"""Target sharding of the device context (nb_set_shard), checked on one GPU.

Two (or three) contexts on the same device play the ranks. They run one after another, never
waiting on each other: each steps its own slice, then the test copies every rank's chunk into the
other contexts' buffers, which is what the in-place all-gather does across GPUs. The gathered state
must equal an unsharded context's state bit for bit after every step.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 1e-4


def make(nb, cls, pm, vel, rank=None, world=None, theta=0.5, leaf=16):
    s = cls(rule=nb.Gravity(1.0, EPS), theta=theta, max_leaf_size=leaf, time_step=1e-3)
    if world is not None:
        s.set_shard(rank, world)
    s.set_bodies(pm, vel)
    return s


@pytest.mark.parametrize("cls_name,n,world,theta,leaf", [
    ("QuadrupoleLinearBVHSolver", 50000, 2, 0.5, 16),
    ("LinearBVHSolver", 12345, 3, 0.5, 16),
    ("QuadrupoleLinearBVHSolver", 40, 2, 0.5, 16),
    ("NaiveSolver", 3000, 2, 0.5, 16),
    # dual tree: tasks of passive nodes outside a rank's slice are dropped, the rest run unchanged
    ("OctupoleImplicitLinearBVHFMMSolver", 60000, 3, 0.4, 64),
    ("OctupoleImplicitLinearBVHFMMSolver", 20000, 4, 0.4, 16),
    ("MultipoleImplicitLinearBVHFMMSolver", 9000, 2, 0.5, 32),
    ("OctupoleImplicitLinearBVHFMMSolver", 70, 4, 0.4, 16),  # chunks of 32: rank 3 holds no target
])
def test_emulated_ranks_equal_unsharded(nb, cls_name, n, world, theta, leaf):
    import torch

    cls = getattr(nb, cls_name)
    pm, vel = nb.scenarios.plummer(n, seed=5)
    ref = make(nb, cls, pm, vel, theta=theta, leaf=leaf)
    ranks = [make(nb, cls, pm, vel, r, world, theta, leaf) for r in range(world)]
    chunk, _, _ = nb.shard_range(n, 0, world)
    try:
        for _ in range(4):
            ref.step(1)
            for s in ranks:
                s.step(1)
                s.synchronize()
            views = [s.shard_tensors(world * chunk) for s in ranks]
            for dst in range(world):
                for src in range(world):
                    if src != dst:
                        lo, hi = src * chunk, (src + 1) * chunk
                        for k in range(2):
                            views[dst][k][lo:hi].copy_(views[src][k][lo:hi])
            torch.cuda.synchronize()
            for s in ranks:
                s.shard_gathered()
            p_ref, v_ref = ref.bodies()
            for s in ranks:
                p, v = s.bodies()
                assert np.array_equal(p, p_ref)
                assert np.array_equal(v, v_ref)
    finally:
        ref.close()
        for s in ranks:
            s.close()


def test_shard_guards(nb):
    pm, vel = nb.scenarios.plummer(1000, seed=1)
    with nb.QuadrupoleLinearBVHSolver(bodies=pm, velocities=vel) as s:
        with pytest.raises(nb.NBodyError):
            s.set_shard(1, 3)  # 3 chunks of 352 bodies exceed the buffers sized for 1000 (1024)
    with nb.QuadrupoleLinearBVHSolver() as s:
        s.set_shard(0, 2)
        s.set_bodies(pm, vel)
        with pytest.raises(nb.NBodyError):
            s.step(2)  # one step per call when sharded
        with pytest.raises(nb.NBodyError):
            s.set_instances([500, 500], pm)
        with pytest.raises(nb.NBodyError):
            s.set_shard(2, 2)
    with nb.OctupoleImplicitLinearBVHFMMSolver() as s:
        s.set_shard(0, 2)  # the dual-tree solver shards over targets as well
        with pytest.raises(nb.NBodyError):
            s.set_instances([500, 500], pm)


def test_dual_shard_counts_add_up(nb):
    """The ranks' interaction counts: every pair term of the unsharded pass belongs to exactly one
    target, so the ranks' pair counts add up to it; far-field tasks above the slices run on every
    rank whose slice they cover, so node-node counts add up to at least the unsharded count."""
    pm, vel = nb.scenarios.plummer(40000, seed=9)
    world = 3
    with make(nb, nb.OctupoleImplicitLinearBVHFMMSolver, pm, vel, theta=0.4, leaf=64) as ref:
        ref.update_accelerations()
        c_ref = ref.counts()
    pp = nn = 0
    for r in range(world):
        with make(nb, nb.OctupoleImplicitLinearBVHFMMSolver, pm, vel, r, world, theta=0.4, leaf=64) as s:
            s.update_accelerations()
            c = s.counts()
            pp += c["particle_particle"]
            nn += c["node_node"]
    assert pp == c_ref["particle_particle"]
    assert nn >= c_ref["node_node"]
