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

``PeerShardedSimulation`` is the same step without a library collective:
the deposit adds each rank's cells straight into the owning rank's buffer
over NVLink and an exchange kernel gathers the owners' slices
(``mog_shard_*``, csrc/shard.cu); the ranks swap CUDA IPC handles of those
buffers once, over the process group.  ``LocalPeerGroup`` holds all ranks
in one process (one handle each, on one GPU or several), which is how the
peer exchange runs on a single GPU.
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


def _peer_config(cfg: MogConfig, scale_bits: int) -> MogConfig:
    return replace(cfg, scale_bits=scale_bits if cfg.mass_mode == "u64" else cfg.scale_bits)


def exchange_handles(accum: bytes, flags: bytes, group=None) -> tuple[bytes, bytes]:
    """Every rank's 64-byte CUDA IPC handles of its accumulation buffer and
    flags, each list concatenated in rank order (what mog_shard_connect
    takes).  Collective over ``group``."""
    import torch.distributed as dist

    if len(accum) != 64 or len(flags) != 64:
        raise ValueError("IPC handles are 64 bytes")
    blobs = [None] * dist.get_world_size(group)
    dist.all_gather_object(blobs, (bytes(accum), bytes(flags)), group=group)
    return b"".join(b[0] for b in blobs), b"".join(b[1] for b in blobs)


def _stream(device):
    import ctypes

    torch = _torch()
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class PeerShardedSimulation(ShardedSimulation):
    """A simulation sharded over ``group`` whose grid sum runs over peer
    memory (``mog_shard_step``): one process per GPU, every GPU able to
    reach the others' memory (NVLink).  Same constructor arguments as
    ShardedSimulation, without ``stages``.
    """

    def __init__(self, cfg: Mapping[str, Any] | MogConfig, pos, vel=None, *, group=None,
                 device=None):
        import ctypes

        import torch.distributed as dist

        from . import _lib as libmod
        from .simulation import Simulation

        torch = _torch()
        self.cfg = cfg if isinstance(cfg, MogConfig) else MogConfig.from_dict(cfg)
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.pos = pos
        self.vel = torch.zeros_like(pos) if vel is None else vel
        self.timescale = 1.0
        self.steps_taken = 0
        self.scale_bits = self._global_scale_bits()
        self.stages = None
        self._lib = libmod.lib()
        self.sim = Simulation(_peer_config(self.cfg, self.scale_bits), device=device)
        self.sim.set_particles(self.pos, self.vel)
        self.pos, self.vel = self.sim.pos, self.sim.vel
        h = self.sim.handle
        libmod.check(self._lib.mog_shard_init(h, self.rank, self.world), "mog_shard_init")
        a, f = (ctypes.c_uint8 * 64)(), (ctypes.c_uint8 * 64)()
        libmod.check(self._lib.mog_shard_export(h, a, f), "mog_shard_export")
        accum, flags = exchange_handles(bytes(a), bytes(f), group)
        libmod.check(self._lib.mog_shard_connect(h, accum, flags), "mog_shard_connect")
        dist.barrier(group=group)

    def step(self, n_steps: int = 1) -> None:
        from . import _lib as libmod

        dt = float(self.cfg.dt * self.timescale)
        h = self.sim.handle
        for _ in range(n_steps):
            libmod.check(self._lib.mog_shard_step(h, self.pos.data_ptr(), self.vel.data_ptr(),
                                                  int(self.pos.shape[0]), dt,
                                                  _stream(self.pos.device)), "mog_shard_step")
            self.steps_taken += 1

    def status(self) -> int:
        return self.sim.status()

    def close(self) -> None:
        """Every rank's last step must be done before any rank frees its
        buffers: synchronise, meet the others, then destroy."""
        import torch.distributed as dist

        torch = _torch()
        if self.pos.is_cuda:
            torch.cuda.synchronize(self.pos.device)
        dist.barrier(group=self.group)
        self.sim.close()


class LocalPeerGroup:
    """All ``world`` ranks of one peer-sharded simulation in this process:
    shard r's particles on handle r (on ``devices[r]``, default the current
    device).  A step runs every rank's deposit, then every exchange, then
    every solve and update, each rank on its device's current stream; on one
    GPU the ranks' kernels therefore run one after another and no exchange
    waits on a deposit that has not been issued."""

    def __init__(self, cfg: Mapping[str, Any] | MogConfig, pos_shards, vel_shards=None,
                 devices=None):
        import ctypes

        from . import _lib as libmod
        from .simulation import Simulation, auto_scale_bits

        torch = _torch()
        self.cfg = cfg if isinstance(cfg, MogConfig) else MogConfig.from_dict(cfg)
        self.world = len(pos_shards)
        if vel_shards is None:
            vel_shards = [None] * self.world
        devices = devices or [None] * self.world
        if self.cfg.scale_bits is None and self.cfg.mass_mode == "u64":
            total = sum(float(np.asarray(p, np.float64)[:, 3].sum()) if len(p) else 0.0
                        for p in (x.cpu().numpy() if hasattr(x, "cpu") else x for x in pos_shards))
            bits = auto_scale_bits(total if any(len(p) for p in pos_shards) else 1.0)
        else:
            bits = self.cfg.scale_bits if self.cfg.scale_bits is not None else 0
        self.scale_bits = bits
        self.sims = []
        for r in range(self.world):
            sim = Simulation(_peer_config(self.cfg, bits), device=devices[r])
            p = pos_shards[r]
            v = vel_shards[r]
            if len(p):
                sim.set_particles(p, v)
            else:
                z = torch.zeros((0, 4), dtype=torch.float32, device=sim.device)
                sim.pos, sim.vel = z, z.clone()
            self.sims.append(sim)
        lib = libmod.lib()
        handles = [s.handle for s in self.sims]
        for r, h in enumerate(handles):
            libmod.check(lib.mog_shard_init(h, r, self.world), "mog_shard_init")
        peers = (ctypes.c_void_p * self.world)(*[h.value for h in handles])
        for h in handles:
            libmod.check(lib.mog_shard_connect_local(h, peers), "mog_shard_connect_local")
        self.steps_taken = 0
        self.timescale = 1.0

    def step(self, n_steps: int = 1) -> None:
        from . import _lib as libmod
        from .simulation import torch_device

        lib = libmod.lib()
        dt = float(self.cfg.dt * self.timescale)
        for _ in range(n_steps):
            for s in self.sims:
                with torch_device(s.device):
                    libmod.check(lib.mog_shard_deposit(s.handle, s.pos.data_ptr(), s.n_particles,
                                                       _stream(s.device)), "mog_shard_deposit")
            for s in self.sims:
                with torch_device(s.device):
                    libmod.check(lib.mog_shard_exchange(s.handle, _stream(s.device)),
                                 "mog_shard_exchange")
            for s in self.sims:
                with torch_device(s.device):
                    libmod.check(lib.mog_shard_finish(s.handle, s.pos.data_ptr(), s.vel.data_ptr(),
                                                      s.n_particles, dt, _stream(s.device)),
                                 "mog_shard_finish")
            self.steps_taken += 1

    def gather(self):
        """All ranks' particles in rank order: (pos, vel) on the first rank's device."""
        torch = _torch()
        dev = self.sims[0].device
        return (torch.cat([s.pos.to(dev) for s in self.sims]),
                torch.cat([s.vel.to(dev) for s in self.sims]))

    def status(self) -> list[int]:
        return [s.status() for s in self.sims]

    def close(self) -> None:
        torch = _torch()
        for s in self.sims:
            torch.cuda.synchronize(s.device)
        for s in self.sims:
            s.close()
