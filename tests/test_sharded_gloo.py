"""Target sharding of one instance over ranks (ShardedStepper), as world-size-2 gloo processes on
the CPU.

The device solver cannot run here, so the ranks drive a host model with the device context's
sharding semantics: each step sorts the whole state into Morton order (stable), evaluates the
oracle's Barnes-Hut accelerations for the rank's slice only, applies the kick-drift to that slice,
and exposes the state buffers (capacity world * chunk) for the in-place all-gather. The gathered
run must equal the single-rank run bit for bit, and the slice arithmetic comes from the library's
nb_shard_range (a host function that needs no device).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import REPO  # noqa: F401  (sets the import paths)

EPS = 1e-4
THETA = 0.5
LEAF = 16
DT = np.float32(1e-3)


class HostShardModel:
    """Host model of a sharded context: state in slot order, slices by nb_shard_range."""

    def __init__(self, pm, vel, rank, world):
        import nbody_b200 as nb
        import oracle as O

        self.nb, self.O = nb, O
        self.n = len(pm)
        self.rank, self.world = rank, world
        chunk, _, _ = nb.shard_range(self.n, rank, world)
        cap = max(self.n, chunk * world)
        self.pm = np.zeros((cap, 4), np.float32)
        self.vel = np.zeros((cap, 4), np.float32)
        self.pm[: self.n] = pm
        self.vel[: self.n] = vel
        self.ids = np.arange(self.n, dtype=np.int64)

    def body_count(self):
        return self.n

    def step(self, k):
        assert k == 1
        O, n = self.O, self.n
        pm, vel = self.pm[:n], self.vel[:n]
        codes = O.morton_codes(pm, O.bbox(pm))
        perm = O.sort_codes(codes)
        self.pm[:n] = pm[perm]
        self.vel[:n] = vel[perm]
        self.ids = self.ids[perm]
        _, first, count = self.nb.shard_range(n, self.rank, self.world)
        if count:
            sl = slice(first, first + count)
            acc, _ = O.bh_targets(self.pm[:n], self.pm[sl], eps=EPS, theta=THETA, leaf=LEAF, order=2)
            p, v = O.kick_drift(self.pm[sl], self.vel[sl], acc, DT)
            self.pm[sl] = p
            self.vel[sl] = v

    def shard_tensors(self, rows):
        return torch.from_numpy(self.pm[:rows]), torch.from_numpy(self.vel[:rows])

    def shard_gathered(self):
        pass

    def state(self):
        out_p = np.zeros((self.n, 4), np.float32)
        out_v = np.zeros((self.n, 4), np.float32)
        out_p[self.ids] = self.pm[: self.n]
        out_v[self.ids] = self.vel[: self.n]
        return out_p, out_v


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, n, steps, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import sys

    sys.path[:0] = [os.path.join(REPO, "n-body_b200"), os.path.join(REPO, "oracle")]
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import nbody_b200 as nb

    pm, vel = nb.scenarios.plummer(n, seed=77)
    model = HostShardModel(pm, vel, rank, world)
    nb.ShardedStepper(model).step(steps)
    p, v = model.state()
    np.save(os.path.join(out_dir, f"p{rank}.npy"), p)
    np.save(os.path.join(out_dir, f"v{rank}.npy"), v)
    dist.destroy_process_group()


@pytest.mark.parametrize("n,world", [(3000, 2), (1001, 2), (40, 2)])
def test_two_rank_gather_equals_single_rank(tmp_path, nb, oracle, n, world):
    steps = 3
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n, steps, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    pm, vel = nb.scenarios.plummer(n, seed=77)
    single = HostShardModel(pm, vel, 0, 1)
    for _ in range(steps):
        single.step(1)
    p_ref, v_ref = single.state()
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"p{r}.npy"), p_ref)
        assert np.array_equal(np.load(tmp_path / f"v{r}.npy"), v_ref)


def test_shard_range_covers_all_bodies(nb):
    for n in (0, 1, 31, 32, 33, 1000, 4097, 1 << 20):
        for world in (1, 2, 3, 4, 7, 8):
            covered = []
            for r in range(world):
                chunk, first, count = nb.shard_range(n, r, world)
                assert chunk % 32 == 0 and chunk * world >= n
                assert count >= 0 and (count == 0 or first == r * chunk)
                covered.extend(range(first, first + count))
            assert covered == list(range(n))
    with pytest.raises(nb.NBodyError):
        nb.shard_range(10, 2, 2)
    with pytest.raises(nb.NBodyError):
        nb.shard_range(10, 0, 0)
