"""The sharded step (mog_solver_b200.sharded) over gloo on the CPU: ranks
deposit their own particles, all-reduce the integer grids, solve and update
their own particles.  The stages here are the oracle's (integer deposit, FP64
solve rounded to FP32, update.glsl in C), so the only thing under test is the
sharding: the trajectory must be bit-identical to one process over all
particles, for any number of ranks and uneven shards."""
import os
import socket

import numpy as np
import pytest

import oracle
from oracle import pipeline as pl

torch = pytest.importorskip("torch")

CFG = {"n_grids": 3, "grid_size": 8, "world_size": 100.0, "num_particles": 1001, "G": 100.0,
       "dt": 1e-3, "damping": 0.999, "seed": 4}
STEPS = 3


class OracleStages:
    """deposit / solve / update on the CPU with the oracle."""

    def __init__(self, cfg, scale_bits):
        from mog_solver_b200.transforms import compute_transforms

        self.cfg, self.bits = cfg, scale_bits
        self.off, self.rot = compute_transforms(cfg.n_grids, cfg.grid_size, cfg.world_size,
                                                seed=cfg.seed)

    def deposit(self, pos):
        c = self.cfg
        m = oracle.deposit(pos.numpy(), self.rot, self.off, c.grid_size, c.world_size,
                           oracle.MASS_U64, self.bits)
        return torch.from_numpy(m.view(np.int64).copy())

    def solve(self, mass):
        c = self.cfg
        rho = mass.numpy().view(np.uint64).astype(np.float64) * 2.0 ** -self.bits
        F = pl.forces_grid_fp64(rho, c.G, c.world_size).astype(np.float32)
        out = np.zeros(F.shape[:-1] + (4,), np.float32)
        out[..., :3] = F
        return torch.from_numpy(out)

    def update(self, pos, vel, force, dt):
        c = self.cfg
        p, v = oracle.update(pos.numpy(), vel.numpy(), force.numpy(), self.rot, self.off,
                             c.grid_size, c.world_size, dt, c.damping)
        pos.copy_(torch.from_numpy(p))
        vel.copy_(torch.from_numpy(v))


def _particles(n):
    rng = np.random.default_rng(11)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.mod(rng.normal(50, 12, (n, 3)), 100.0)
    pos[:, 3] = rng.uniform(0.5, 1.5, n) / n
    vel = np.zeros_like(pos)
    vel[:, :3] = rng.normal(0, 0.1, (n, 3))
    return pos, vel


def _worker(rank, world, port, n, q):
    import torch.distributed as dist

    from mog_solver_b200.sharded import ShardedSimulation, shard_bounds

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        pos, vel = _particles(n)
        lo, hi = shard_bounds(n, rank, world)
        sim = ShardedSimulation(CFG, torch.from_numpy(pos[lo:hi].copy()),
                                torch.from_numpy(vel[lo:hi].copy()), stages=OracleStages)
        sim.step(STEPS)
        P, V = sim.gather()
        if rank == 0:
            q.put((P.numpy(), V.numpy(), sim.scale_bits))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run(world, n):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = q.get()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


def test_shard_bounds_cover_everything():
    from mog_solver_b200.sharded import shard_bounds

    for n in (0, 1, 5, 1001):
        for world in (1, 2, 3, 8):
            b = [shard_bounds(n, r, world) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
            assert max(h - l for l, h in b) - min(h - l for l, h in b) <= 1


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_trajectory_equals_single_process(world):
    n = CFG["num_particles"]
    P1, V1, bits1 = _run(1, n)
    Pw, Vw, bitsw = _run(world, n)
    assert bits1 == bitsw
    assert np.array_equal(P1.view(np.uint32), Pw.view(np.uint32))
    assert np.array_equal(V1.view(np.uint32), Vw.view(np.uint32))
    # and it moved
    pos, _ = _particles(n)
    assert not np.array_equal(P1, pos)


def test_a_rank_without_particles():
    """More ranks than particles: empty shards still take part in every
    all-reduce, and the result is the single-process one."""
    P1, V1, _ = _run(1, 2)
    P3, V3, _ = _run(3, 2)
    assert np.array_equal(P1.view(np.uint32), P3.view(np.uint32))
