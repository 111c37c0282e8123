"""Data-parallel training of the parameter MLP: one process per GPU, each rank trains on its own windows, and one
all-reduce per step averages the 812-double weight gradient and the loss sum before every rank takes the same Adam
step. The denoise path itself has no cross-GPU exchange (each GPU runs its own frame stream); this is the one place
where ranks talk, and it moves 6.5 KB per step, so plain NCCL all-reduce over NVLink is the right tool.

The logic here only touches torch tensors and ``torch.distributed``, so it runs the same under NCCL (device tensors
that view the trainer's accumulators) and under gloo (CPU tensors, which is how it is tested without a GPU).
"""
from __future__ import annotations

import numpy as np


class DataParallel:
    """Rank bookkeeping and the per-step reductions. world == 1 (or no process group) makes every call a no-op."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self._dist = dist if dist.is_available() and dist.is_initialized() else None
        self.group = group
        self.rank = self._dist.get_rank(group) if self._dist else 0
        self.world = self._dist.get_world_size(group) if self._dist else 1

    def seed_rng(self, base_seed: int) -> np.random.Generator:
        """The generator that draws this rank's window seeds. Ranks draw from disjoint residue classes (see
        window_seed), so no two ranks train on the same window in a step."""
        return np.random.default_rng([int(base_seed), self.rank])

    def window_seed(self, rng: np.random.Generator, n_seeds: int) -> int:
        """A seed in [0, n_seeds) congruent to this rank modulo world. Needs n_seeds >= world: with fewer seeds than
        ranks some rank would have no seed of its own."""
        if n_seeds < self.world:
            raise ValueError(f"window_seed: {n_seeds} seeds cannot give each of {self.world} ranks its own")
        per = (n_seeds - self.rank + self.world - 1) // self.world  # seeds congruent to rank in [0, n_seeds)
        return int(rng.integers(0, per)) * self.world + self.rank

    def average_(self, *tensors) -> None:
        """In-place mean over ranks of each tensor (SUM all-reduce, then divide by world)."""
        if self._dist is None or self.world == 1:
            return
        for t in tensors:
            self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM, group=self.group)
            t.div_(self.world)

    def broadcast_(self, tensor, src: int = 0) -> None:
        if self._dist is not None and self.world > 1:
            self._dist.broadcast(tensor, src=src, group=self.group)

    def max_divergence(self, tensor) -> float:
        """max |tensor - tensor on rank 0| over all ranks and elements (0.0 when the ranks agree)."""
        if self._dist is None or self.world == 1:
            return 0.0
        ref = tensor.clone()
        self._dist.broadcast(ref, src=0, group=self.group)
        d = (tensor - ref).abs().max().reshape(1).to(tensor.dtype)
        self._dist.all_reduce(d, op=self._dist.ReduceOp.MAX, group=self.group)
        return float(d.item())


def finish_step(trainer, dp: DataParallel | None, n_frames: int, lr: float, clip: float, **adam):
    """End of one training step: average the gradient and loss accumulators over ranks (in place, on the trainer's
    stream), read the mean per-frame loss, then take the Adam step. Returns (loss, grad_norm)."""
    if dp is not None and dp.world > 1:
        grad, loss = trainer.accumulators()
        dp.average_(grad, loss)
    loss = trainer.loss_sum() / n_frames
    gn = trainer.step(lr, clip=clip, **adam)
    return loss, gn
