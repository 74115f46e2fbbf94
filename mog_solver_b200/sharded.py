"""One simulation whose particles are split over the ranks of a process
group: the multi-GPU form of the force-and-step path (no counterpart in the
reference, which runs on a single GL context).

Each rank holds a shard of the particles.  One step is

1. deposit the local particles into all k fixed-point grids (integers);
2. ``all_reduce(SUM)`` of the grids over the group -- integer addition, so
   every rank ends with the same, bit-exact total whatever the split;
3. the identical spectral solve on every rank;
4. gather and update of the rank's own particles.

The fixed-point scale is chosen once from the global total mass, so every
rank quantises the same way; the trajectory is then bit-identical to a
single-process run over all particles, for any number of ranks.

``LibraryStages`` runs the stages through the C ABI (``mog_deposit``,
``mog_solve``, ``mog_update``) on the rank's GPU, and the all-reduce over
NCCL; any object with the same three methods can stand in (the CPU tests
use the integer oracle over gloo).
"""
from __future__ import annotations

from dataclasses import replace
from typing import Any, Callable, Mapping

import numpy as np

from .config import MogConfig


def _torch():
    import torch

    return torch


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of rank's particles: contiguous, sizes differ by at most one."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


class LibraryStages:
    """The three stages of a step through the C ABI on one GPU."""

    def __init__(self, cfg: MogConfig, scale_bits: int, device=None,
                 offsets: np.ndarray | None = None, rotations: np.ndarray | None = None):
        from .simulation import Simulation

        c = replace(cfg, scale_bits=scale_bits if cfg.mass_mode == "u64" else cfg.scale_bits)
        self.sim = Simulation(c, device=device, offsets=offsets, rotations=rotations)

    def deposit(self, pos):
        return self.sim.mass_grid(pos)

    def solve(self, mass):
        return self.sim.solve_grid(mass)

    def update(self, pos, vel, force, dt: float) -> None:
        self.sim.pos, self.sim.vel = pos, vel
        self.sim.update_from_grid(force, dt)

    def close(self) -> None:
        self.sim.close()


class ShardedSimulation:
    """A simulation sharded over ``group`` (default: the world group).

    pos, vel: this rank's particles, (n_local, 4) float32 tensors on the
    stages' device.  ``stages``: a callable (cfg, scale_bits) -> object with
    deposit / solve / update; by default LibraryStages on ``device``.
    """

    def __init__(self, cfg: Mapping[str, Any] | MogConfig, pos, vel=None, *, group=None,
                 stages: Callable[[MogConfig, int], Any] | None = None, device=None):
        import torch.distributed as dist

        torch = _torch()
        self.cfg = cfg if isinstance(cfg, MogConfig) else MogConfig.from_dict(cfg)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.pos = pos
        self.vel = torch.zeros_like(pos) if vel is None else vel
        self.timescale = 1.0
        self.scale_bits = self._global_scale_bits()
        if stages is None:
            self.stages = LibraryStages(self.cfg, self.scale_bits, device=device)
        else:
            self.stages = stages(self.cfg, self.scale_bits)
        self.steps_taken = 0

    def _global_scale_bits(self) -> int:
        """The configured scale, else the one for the total mass of all shards."""
        import torch.distributed as dist

        from .simulation import auto_scale_bits

        if self.cfg.scale_bits is not None or self.cfg.mass_mode != "u64":
            return self.cfg.scale_bits if self.cfg.scale_bits is not None else 0
        torch = _torch()
        total = self.pos[:, 3].to(torch.float64).sum().reshape(1)
        dist.all_reduce(total, op=dist.ReduceOp.SUM, group=self.group)
        n = torch.tensor([self.pos.shape[0]], dtype=torch.int64, device=total.device)
        dist.all_reduce(n, op=dist.ReduceOp.SUM, group=self.group)
        return auto_scale_bits(float(total.item()) if int(n.item()) else 1.0)

    def step(self, n_steps: int = 1) -> None:
        import torch.distributed as dist

        dt = float(self.cfg.dt * self.timescale)
        for _ in range(n_steps):
            mass = self.stages.deposit(self.pos)
            dist.all_reduce(mass, op=dist.ReduceOp.SUM, group=self.group)  # integer: exact
            force = self.stages.solve(mass)
            self.stages.update(self.pos, self.vel, force, dt)
            self.steps_taken += 1

    def gather(self):
        """All ranks' particles in rank order, on every rank: (pos, vel)."""
        import torch.distributed as dist

        torch = _torch()
        sizes = [torch.zeros(1, dtype=torch.int64, device=self.pos.device) for _ in range(self.world)]
        dist.all_gather(sizes, torch.tensor([self.pos.shape[0]], dtype=torch.int64,
                                            device=self.pos.device), group=self.group)
        m = max(int(s.item()) for s in sizes)
        out = []
        for t in (self.pos, self.vel):
            pad = torch.zeros((m, 4), dtype=t.dtype, device=t.device)
            pad[: t.shape[0]] = t
            parts = [torch.empty_like(pad) for _ in range(self.world)]
            dist.all_gather(parts, pad, group=self.group)
            out.append(torch.cat([p[: int(s.item())] for p, s in zip(parts, sizes)]))
        return out[0], out[1]

    def close(self) -> None:
        close = getattr(self.stages, "close", None)
        if close is not None:
            close()
