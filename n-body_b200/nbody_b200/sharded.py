"""One instance advanced by several processes, one GPU each, sharded over targets.

Every rank holds the whole body set. Each step it sorts and builds the tree over all bodies,
evaluates accelerations and the kick-drift for its own slice of the Morton-ordered bodies only
(nb_set_shard), then all ranks all-gather the updated positions and velocities in place: rank r's
slice sits at offset r * chunk of the same buffer, so the all-gather (NCCL's in-place form, where
the send buffer is the receiver's own chunk) leaves the whole state on every rank. This is the
path's one exchange: 32 bytes per body per step.

The stepper drives any solver-like object with step(1), body_count(), shard_tensors(rows) and
shard_gathered(): the device solver in production, a host model in the CPU tests.
"""
from __future__ import annotations


class ShardedStepper:
    def __init__(self, solver, group=None):
        import torch.distributed as dist

        from . import shard_range

        self.solver = solver
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self._range = shard_range

    def slice(self):
        """(chunk, first, count) of this rank's Morton-ordered bodies."""
        return self._range(self.solver.body_count(), self.rank, self.world)

    def gather(self):
        """All-gather the ranks' slices of positions and velocities into every rank's state."""
        import torch.distributed as dist

        chunk, _, _ = self.slice()
        lo, hi = self.rank * chunk, (self.rank + 1) * chunk
        for t in self.solver.shard_tensors(self.world * chunk):
            dist.all_gather_into_tensor(t, t[lo:hi], group=self.group)
        self.solver.shard_gathered()

    def step(self, steps: int = 1):
        for _ in range(steps):
            self.solver.step(1)
            self.gather()
