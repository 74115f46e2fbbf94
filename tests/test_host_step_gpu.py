"""Steps over particles held in host memory (mog_step_host,
mog_learned_step_host): chunked copies overlapped with the kernels must give
bit for bit what copying the records to the device, stepping there and
copying them back gives."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _sim(k, g, n, seed=0):
    from mog_solver_b200 import Simulation

    return Simulation({"n_grids": k, "grid_size": g, "world_size": 100.0, "num_particles": n,
                       "G": 100.0, "dt": 1e-3, "damping": 0.999, "seed": seed})


def _particles(n, seed):
    from mog_solver_b200 import ics

    pos, vel = ics.clumps(n, 100.0, seed=seed)
    vel[:, :3] = np.random.default_rng(seed).normal(0, 1, (n, 3))
    return pos, vel


def _pinned(a):
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()


@pytest.mark.parametrize("n,k,g,chunks", [(70001, 24, 16, 8), (5000, 7, 8, 3), (30000, 5, 32, 1),
                                          (257, 3, 16, 64)])
def test_plain_host_step_equals_device_step(n, k, g, chunks):
    a, b = _sim(k, g, n), _sim(k, g, n)
    pos, vel = _particles(n, k + g)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    hp, hv = _pinned(pos), _pinned(vel)
    for _ in range(3):
        b.step_host(hp, hv, chunks=chunks)
        a.step()
    torch.cuda.synchronize()
    assert torch.equal(a.pos.cpu(), hp) and torch.equal(a.vel.cpu(), hv)
    assert b.status() == 0


@pytest.mark.parametrize("n,chunks", [(100000, 8), (4097, 3)])
def test_learned_host_step_equals_device_step(n, chunks):
    from mog_solver_b200 import _lib
    from mog_solver_b200.learned import Model
    from mog_solver_b200.train_learned import DEFAULT_MODEL

    model = Model.load(DEFAULT_MODEL)
    a, b = _sim(32, 16, n, 3), _sim(32, 16, n, 3)
    pos, vel = _particles(n, 9)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    hp, hv = _pinned(pos), _pinned(vel)
    lib = _lib.lib()
    stats = []
    try:
        for _ in range(3):
            _lib.check(lib.mog_learned_step(a.handle, model.handle, a.pos.data_ptr(), a.vel.data_ptr(),
                                            n, 1e-3, None), "learned step")
            _lib.check(lib.mog_learned_step_host(b.handle, model.handle, hp.data_ptr(), hv.data_ptr(),
                                                 n, 1e-3, chunks, None), "learned host step")
            torch.cuda.synchronize()
            for s in (a, b):
                out = (ctypes.c_double * 2)()
                _lib.check(lib.mog_learned_spread(s.handle, out, None), "spread")
                stats.append((out[0], out[1]))
        assert torch.equal(a.pos.cpu(), hp) and torch.equal(a.vel.cpu(), hv)
        for sa, sb in zip(stats[::2], stats[1::2]):
            # per-CTA float partial sums are grouped differently: equal to rounding
            assert abs(sa[0] - sb[0]) <= 1e-5 * abs(sa[0]) and abs(sa[1] - sb[1]) <= 1e-5 * abs(sa[1])
    finally:
        model.close()


def test_learned_simulation_host_step_with_gate():
    from mog_solver_b200.learned import LearnedSimulation, Model
    from mog_solver_b200.train_learned import DEFAULT_MODEL

    n = 60000
    model = Model.load(DEFAULT_MODEL)
    cheap_a, cheap_b = _sim(32, 16, n, 3), _sim(32, 16, n, 3)
    big_a, big_b = _sim(48, 16, n, 4), _sim(48, 16, n, 4)
    pos, vel = _particles(n, 11)
    for s in (cheap_a, cheap_b, big_a, big_b):
        s.set_particles(pos, vel)
    # a gate factor of zero always fires: steps 0-1 learned, 2-5 fallback
    la = LearnedSimulation(cheap_a, model, fallback=big_a, gate_every=2, gate_factor=0.0)
    lb = LearnedSimulation(cheap_b, model, fallback=big_b, gate_every=2, gate_factor=0.0)
    hp, hv = _pinned(pos), _pinned(vel)
    la.step(6)
    lb.step_host(hp, hv, n_steps=6, chunks=4)
    torch.cuda.synchronize()
    assert la.fallback_steps == lb.fallback_steps == 4
    assert torch.equal(la.pos.cpu(), hp) and torch.equal(la.vel.cpu(), hv)
    model.close()


def test_host_step_rejects_device_buffers():
    sim = _sim(4, 16, 100)
    sim.init_particles("uniform")
    with pytest.raises(ValueError):
        sim.step_host(sim.pos, sim.vel)
