"""The sharded step over peer memory (mog_shard_*, csrc/shard.cu) on one GPU:
all ranks are handles in this process (LocalPeerGroup), every rank's
deposit is issued before any exchange, so no kernel waits on one that has
not been launched.  The trajectory must be bit-identical to one handle
stepping all particles, for any number of ranks and any split (the grid
sum is integer).  A rank that never deposits makes the others' exchange
give up within its bound and raise MOG_FLAG_TIMEOUT."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _cfg(k, g, mass_mode, n):
    return {"n_grids": k, "grid_size": g, "world_size": 100.0, "num_particles": n, "G": 100.0,
            "dt": 1e-3, "damping": 0.999, "seed": 5, "mass_mode": mass_mode,
            "scale_bits": 40 if mass_mode == "u64" else None}


def _particles(n, mass_mode, seed=3):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.mod(rng.normal(50.0, 12.0, (n, 3)), 100.0)
    pos[:, 3] = 1.0 if mass_mode == "u32x1000" else rng.uniform(0.5, 1.5, n) / 1024
    vel = np.zeros_like(pos)
    vel[:, :3] = rng.normal(0.0, 1.0, (n, 3))
    return pos, vel


@pytest.mark.parametrize("world", [1, 2, 3, 4])
@pytest.mark.parametrize("k,g", [(6, 16), (5, 8), (3, 32), (2, 4)])
@pytest.mark.parametrize("mass_mode", ["u64", "u32x1000"])
def test_peer_sharded_trajectory_equals_one_handle(world, k, g, mass_mode):
    from mog_solver_b200 import Simulation
    from mog_solver_b200.sharded import LocalPeerGroup, shard_bounds

    n, steps = 20011, 7  # steps cycle the three slots twice
    pos, vel = _particles(n, mass_mode)
    ref = Simulation(_cfg(k, g, mass_mode, n))
    ref.set_particles(pos, vel)
    ref.step(steps)
    bounds = [shard_bounds(n, r, world) for r in range(world)]
    grp = LocalPeerGroup(_cfg(k, g, mass_mode, n), [pos[lo:hi] for lo, hi in bounds],
                         [vel[lo:hi] for lo, hi in bounds])
    try:
        grp.step(steps)
        P, V = grp.gather()
        torch.cuda.synchronize()
        assert grp.status() == [0] * world
        assert torch.equal(P, ref.pos) and torch.equal(V, ref.vel)
    finally:
        grp.close()
        ref.close()


def test_more_ranks_than_particles_and_grids():
    from mog_solver_b200 import Simulation
    from mog_solver_b200.sharded import LocalPeerGroup, shard_bounds

    n, k, world = 2, 3, 5
    pos, vel = _particles(n, "u64", seed=9)
    ref = Simulation(_cfg(k, 8, "u64", n))
    ref.set_particles(pos, vel)
    ref.step(4)
    bounds = [shard_bounds(n, r, world) for r in range(world)]
    grp = LocalPeerGroup(_cfg(k, 8, "u64", n), [pos[lo:hi] for lo, hi in bounds],
                         [vel[lo:hi] for lo, hi in bounds])
    try:
        grp.step(4)
        P, V = grp.gather()
        torch.cuda.synchronize()
        assert torch.equal(P, ref.pos) and torch.equal(V, ref.vel)
    finally:
        grp.close()
        ref.close()


def test_a_rank_that_never_deposits_times_out():
    """Rank 1 never deposits: rank 0's exchange waits on a flag that nothing
    sets, gives up within its bound, raises MOG_FLAG_TIMEOUT, and the
    context stays usable."""
    from mog_solver_b200 import FLAG_TIMEOUT, _lib
    from mog_solver_b200.sharded import LocalPeerGroup

    n = 1000
    pos, vel = _particles(n, "u64")
    grp = LocalPeerGroup(_cfg(4, 8, "u64", n), [pos[:500], pos[500:]], [vel[:500], vel[500:]])
    try:
        lib = _lib.lib()
        s0 = grp.sims[0]
        t0 = time.time()
        _lib.check(lib.mog_shard_deposit(s0.handle, s0.pos.data_ptr(), s0.n_particles, None),
                   "deposit")
        _lib.check(lib.mog_shard_exchange(s0.handle, None), "exchange")
        assert s0.status() == FLAG_TIMEOUT
        assert time.time() - t0 < 60.0
        s0.step()  # an ordinary step on the same context still runs
        torch.cuda.synchronize()
        assert torch.isfinite(s0.pos).all()
    finally:
        grp.close()


def test_peer_sharded_full_size():
    """The benchmark's size (N = 2^20 colliding disks, k = 240, g = 16) over
    4 ranks: bit-identical to one handle."""
    from mog_solver_b200 import Simulation, ics
    from mog_solver_b200.sharded import LocalPeerGroup, shard_bounds

    n, world, steps = 1 << 20, 4, 4
    cfg = dict(_cfg(240, 16, "u64", n), scale_bits=None)
    ref = Simulation(cfg)
    pos, vel = ics.two_disks(n, 100.0, seed=1, g_eff=ref.effective_g())
    ref.set_particles(pos, vel)
    cfg["scale_bits"] = ref.scale_bits
    ref.step(steps)
    bounds = [shard_bounds(n, r, world) for r in range(world)]
    grp = LocalPeerGroup(cfg, [pos[lo:hi] for lo, hi in bounds], [vel[lo:hi] for lo, hi in bounds])
    try:
        grp.step(steps)
        P, V = grp.gather()
        torch.cuda.synchronize()
        assert grp.status() == [0] * world
        assert torch.equal(P, ref.pos) and torch.equal(V, ref.vel)
    finally:
        grp.close()
        ref.close()
