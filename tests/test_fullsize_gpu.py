"""Size-independent properties at the benchmark's full size, where the oracle
would take too long: N = 2^20 colliding disks, k = 240 grids of 16^3.

* Every grid receives every particle's fixed-point mass exactly once, so
  each of the 240 grids sums to the same integer, sum_p trunc(m_p 2^bits).
* The spectral force conserves momentum: with the same cell for deposit and
  gather, sum_p q_p F_p = sum_i R_i sum_c rho_c F_c, and sum_c rho_c F_c
  vanishes term by term in exact arithmetic (k and -k cancel; the Nyquist
  derivative is dropped by the real part).  FP32 leaves it at rounding level.
* A step is deterministic: two handles advance the same particles to the
  same bits."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N, K, G, L = 1 << 20, 240, 16, 100.0


def _sim():
    from mog_solver_b200 import Simulation, ics

    sim = Simulation({"n_grids": K, "grid_size": G, "world_size": L, "num_particles": N,
                      "G": 100.0, "dt": 1e-5, "damping": 0.999, "seed": 2000})
    pos, vel = ics.two_disks(N, L, seed=1, g_eff=sim.effective_g())
    sim.set_particles(pos, vel)
    return sim, pos, vel


def test_full_size_deposit_gives_every_grid_the_total_mass():
    sim, pos, _ = _sim()
    try:
        grids = sim.mass_grid().cpu().numpy().view(np.uint64).reshape(K, -1)
        q = (pos[:, 3].astype(np.float32) * np.float32(2.0 ** sim.scale_bits)).astype(np.float64)
        total = int(np.floor(q).astype(np.uint64).sum(dtype=np.uint64))
        sums = grids.sum(axis=1, dtype=np.uint64)
        assert (sums == np.uint64(total)).all()
        assert sim.status() == 0
    finally:
        sim.close()


def test_full_size_forces_conserve_momentum():
    sim, pos, _ = _sim()
    try:
        F = sim.forces().cpu().numpy()[:, :3].astype(np.float64)
        q = np.floor(pos[:, 3].astype(np.float32) * np.float32(2.0 ** sim.scale_bits)).astype(np.float64)
        net = np.abs((q[:, None] * F).sum(axis=0)).max()
        scale = (q[:, None] * np.abs(F)).sum(axis=0).max()
        assert scale > 0
        assert net / scale < 1e-5, net / scale
    finally:
        sim.close()


def test_full_size_steps_are_deterministic():
    a, pos, vel = _sim()
    b, _, _ = _sim()
    try:
        a.step(3)
        b.step(3)
        torch.cuda.synchronize()
        assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
    finally:
        a.close()
        b.close()
