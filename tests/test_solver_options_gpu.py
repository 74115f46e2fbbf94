"""Solver options and auxiliary subsystems on the GPU, beyond the core
parity suite (test_gpu_parity.py):

* the softened Green's function (softening > 0, the variant commented out
  in greens.glsl:63-115) against the FP64 pipeline;
* checkpoint / resume: save, load into a new Simulation and continue,
  bit-identical to an uninterrupted run;
* failure detection: a bounded device wait that nothing satisfies gives up,
  raises MOG_FLAG_TIMEOUT and leaves the context usable.
"""
import numpy as np
import pytest

from oracle import pipeline as pl

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5  # relative L2 against the FP64 oracle (FP32 path)


def make_sim(k=4, g=16, L=100.0, G=100.0, n=1000, seed=0, dt=1e-5, damping=0.999):
    from mog_solver_b200 import Simulation

    return Simulation({"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": G,
                       "dt": dt, "damping": damping, "seed": seed})


def particles(n, L=100.0, seed=0):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), dtype=np.float32)
    nc = n // 2
    pos[:nc, :3] = rng.normal(L / 2, L / 12, (nc, 3))
    pos[nc:, :3] = rng.uniform(0, L, (n - nc, 3))
    pos[:, :3] = np.mod(pos[:, :3], np.float32(L))
    pos[:, 3] = 1.0 / max(n, 1)
    vel = np.zeros_like(pos)
    vel[:, :3] = rng.normal(0, 1, (n, 3))
    return pos, vel


@pytest.mark.parametrize("g", [16, 32])
def test_softened_solve_matches_fp64(g):
    """softening > 0: the variant commented out in greens.glsl:63-115."""
    from mog_solver_b200 import Simulation

    L, G, n, k, a = 100.0, 100.0, 20000, 3, 0.5
    sim = Simulation({"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": G,
                      "dt": 1e-5, "seed": 1, "softening": a})
    pos, vel = particles(n, L, seed=g + 1)
    sim.set_particles(pos, vel)
    m = sim.mass_grid()
    F = sim.solve_grid(m).cpu().numpy()[..., :3]
    rho = m.cpu().numpy().view(np.uint64).astype(np.float64) * 2.0 ** -sim.scale_bits
    ref = pl.forces_grid_fp64(rho, G, L, softening=a)
    assert pl.relative_l2(F, ref) <= FORCE_TOL
    plain = pl.forces_grid_fp64(rho, G, L)
    assert pl.relative_l2(ref, plain) > 0.05   # the softening changes the field


def test_checkpoint_resume_is_bit_identical(tmp_path):
    """save after 4 steps, load into a new Simulation, 4 more steps == 8
    uninterrupted steps, bit for bit (the deposit is deterministic)."""
    from mog_solver_b200 import Simulation

    n = 20000
    a = make_sim(k=6, g=16, n=n, dt=1e-3, damping=0.999, seed=3)
    pos, vel = particles(n, seed=12)
    a.set_particles(pos, vel)
    a.step(4)
    a.save(tmp_path / "ck.npz")
    a.step(4)
    b = Simulation.load(tmp_path / "ck.npz")
    assert b.steps_taken == 4
    b.step(4)
    torch.cuda.synchronize()
    assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)


def test_bounded_wait_times_out_and_the_context_survives():
    """A device wait that nothing satisfies gives up within its budget,
    raises MOG_FLAG_TIMEOUT, and the next step still runs and matches a
    fresh handle's."""
    import time

    from mog_solver_b200 import FLAG_TIMEOUT, _lib

    n = 4096
    a = make_sim(k=4, g=16, n=n, dt=1e-3)
    b = make_sim(k=4, g=16, n=n, dt=1e-3)
    pos, vel = particles(n, seed=21)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    assert a.status() == 0
    t0 = time.time()
    _lib.check(_lib.lib().mog_selftest_wait_timeout(a.handle, None), "selftest")
    assert a.status() == FLAG_TIMEOUT
    assert time.time() - t0 < 30.0
    assert a.status() == 0  # read and cleared
    a.step(2)
    b.step(2)
    torch.cuda.synchronize()
    assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
    assert a.status() == 0


@pytest.mark.parametrize("g,k", [(16, 32), (16, 13), (8, 40)])
@pytest.mark.parametrize("equal", [True, False])
def test_split_histogram_at_small_grids_is_bit_exact(g, k, equal):
    """Tuning deposit_split = 1: the high-word-only shared histogram at g = 8
    and 16 (low halves as global atomics) gives the integer oracle's grid,
    for power-of-two masses (no low halves) and for unequal ones."""
    import oracle

    n, L = 1 << 18, 100.0  # equal masses 1/n are a power of two: no low halves
    sim = make_sim(k=k, g=g, n=n)
    sim.tune(deposit_split=1)
    pos, vel = particles(n, L, seed=g + k)
    if not equal:
        pos[:, 3] = np.random.default_rng(5).uniform(0.5, 2.0, n).astype(np.float32) / n
    sim.set_particles(pos, vel)
    got = sim.mass_grid().cpu().numpy().view(np.uint64)
    ref = oracle.deposit(pos, sim.rotations, sim.offsets, g, L, oracle.MASS_U64, sim.scale_bits)
    assert sim.tuning()["deposit_split"] == 1
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("g,k", [(16, 32), (8, 40), (32, 6)])
@pytest.mark.parametrize("masses", ["equal", "two", "random"])
def test_count_histogram_is_bit_exact(g, k, masses):
    """Tuning deposit_split = 2: the count histogram (one word per cell counting
    the particles of a CTA's first mass, any other mass as a global atomic)
    gives the integer oracle's grid for equal masses with non-zero low halves,
    for two interleaved masses and for random ones."""
    import oracle

    n, L = 200003, 100.0
    sim = make_sim(k=k, g=g, n=n)
    sim.tune(deposit_split=2)
    pos, vel = particles(n, L, seed=g + k + 1)
    if masses == "equal":
        pos[:, 3] = np.float32(1.0 / n)
    elif masses == "two":
        pos[:, 3] = np.where(np.arange(n) % 7 == 0, 2.0, 1.0).astype(np.float32) / n
    else:
        pos[:, 3] = np.random.default_rng(6).uniform(0.5, 2.0, n).astype(np.float32) / n
    sim.set_particles(pos, vel)
    got = sim.mass_grid().cpu().numpy().view(np.uint64)
    ref = oracle.deposit(pos, sim.rotations, sim.offsets, g, L, oracle.MASS_U64, sim.scale_bits)
    assert sim.tuning()["deposit_split"] == 2
    assert np.array_equal(got, ref)
    assert sim.status() == 0
    sim.close()


@pytest.mark.parametrize("g", [8, 16, 32])
def test_learned_fold_is_bit_identical(g):
    """Tuning learned_fold = 1 (the default): the solve's epilogue writes the cell masses
    (g = 8, 16; a separate pass at g = 32): the learned step's particles and
    its variance-gate statistics are those of the separate pass, bit for bit."""
    import ctypes

    from mog_solver_b200 import _lib
    from mog_solver_b200.learned import Model
    from mog_solver_b200.train_learned import DEFAULT_MODEL

    n = 50000
    model = Model.load(DEFAULT_MODEL)
    a = make_sim(k=32, g=g, n=n, dt=1e-3)
    b = make_sim(k=32, g=g, n=n, dt=1e-3)
    a.tune(learned_fold=-1)
    b.tune(learned_fold=1)
    pos, vel = particles(n, seed=31)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    lib = _lib.lib()
    try:
        for _ in range(3):
            for s in (a, b):
                _lib.check(lib.mog_learned_step(s.handle, model.handle, s.pos.data_ptr(),
                                                s.vel.data_ptr(), n, 1e-3, None), "learned step")
        torch.cuda.synchronize()
        assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
        sa, sb = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
        _lib.check(lib.mog_learned_spread(a.handle, sa, None), "spread")
        _lib.check(lib.mog_learned_spread(b.handle, sb, None), "spread")
        assert list(sa) == list(sb)
        assert a.status() == 0 and b.status() == 0
    finally:
        a.close()
        b.close()
        model.close()


def test_deposit_layout_follows_the_masses():
    """Simulation picks a one-word deposit histogram exactly when every mass
    is the same (deposit_split 1, high words, when every fixed-point low
    half is zero; 2, counts, otherwise), re-checks it when the particles
    change, and leaves a caller's own choice alone; the steps are
    bit-identical either way."""
    n = 1 << 16
    pos, vel = particles(n, seed=41)
    pos[:, 3] = 1.0 / n  # q = 2^52 / 2^16 = 2^36: low halves zero
    a = make_sim(k=8, g=16, n=n)
    b = make_sim(k=8, g=16, n=n)
    try:
        a.set_particles(pos, vel)
        b.set_particles(pos, vel)
        b.tune(deposit_split=-1)
        assert a.tuning()["deposit_split"] == 1 and b.tuning()["deposit_split"] == -1
        a.step(3)
        b.step(3)
        torch.cuda.synchronize()
        assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
        odd = pos.copy()
        odd[:, 3] = np.float32(1.0 / 3.0) / n  # equal, with non-zero low halves
        a.set_particles(odd, vel)
        b.set_particles(odd, vel)
        assert a.tuning()["deposit_split"] == 2
        a.step(3)
        b.step(3)
        torch.cuda.synchronize()
        assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
        uneven = pos.copy()
        uneven[:, 3] = np.linspace(0.5, 1.5, n, dtype=np.float32) / n
        a.set_particles(uneven, vel)
        assert a.tuning()["deposit_split"] == 0
        a.set_particles(pos, vel)
        assert a.tuning()["deposit_split"] == 1
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("g,k,alias", [(16, 32, False), (16, 7, False), (8, 40, False),
                                       (16, 240, False), (16, 32, True)])
def test_split_solve_is_bit_identical(g, k, alias):
    """Tuning solve_split = 1 (a cluster of three CTAs per grid pair, one
    gradient field each, the fields read across the cluster's shared memory)
    gives the forces of the one-CTA-per-pair solve (-1) bit for bit: in the
    grid frame (mog_solve), at the particles, over plain steps (world-frame
    slots, mass grid cleared by the solve) and over learned steps (cell masses
    in the force grid); odd k leaves the last pair one grid."""
    import ctypes

    from mog_solver_b200 import Simulation, _lib
    from mog_solver_b200.learned import Model
    from mog_solver_b200.train_learned import DEFAULT_MODEL

    n = 60000
    pos, vel = particles(n, seed=g + k + 3)
    cfg = {"n_grids": k, "grid_size": g, "world_size": 100.0, "num_particles": n, "G": 100.0,
           "dt": 1e-3, "seed": 4, "reference_texture_aliasing": alias}
    a, b = Simulation(dict(cfg)), Simulation(dict(cfg))
    model = None
    try:
        a.tune(solve_split=-1)
        b.tune(solve_split=1)
        assert a.tuning()["solve_split"] == -1 and b.tuning()["solve_split"] == 1
        a.set_particles(pos, vel)
        b.set_particles(pos, vel)
        m = a.mass_grid()
        assert torch.equal(a.solve_grid(m.clone()), b.solve_grid(m.clone()))
        assert torch.equal(a.forces(), b.forces())
        a.step(3)
        b.step(3)
        torch.cuda.synchronize()
        assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
        if k == 32 and not alias:
            model = Model.load(DEFAULT_MODEL)
            lib = _lib.lib()
            for _ in range(2):
                for s in (a, b):
                    _lib.check(lib.mog_learned_step(s.handle, model.handle, s.pos.data_ptr(),
                                                    s.vel.data_ptr(), n, 1e-3, None), "learned step")
            torch.cuda.synchronize()
            assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)
            sa, sb = (ctypes.c_double * 2)(), (ctypes.c_double * 2)()
            _lib.check(lib.mog_learned_spread(a.handle, sa, None), "spread")
            _lib.check(lib.mog_learned_spread(b.handle, sb, None), "spread")
            assert list(sa) == list(sb)
        assert a.status() == 0 and b.status() == 0
    finally:
        a.close()
        b.close()
        if model is not None:
            model.close()


def test_solve_split_defaults_to_auto_and_checks_its_range():
    """solve_split starts at 0 (auto: the clustered solve while three CTAs per
    grid pair fit one wave of the SMs) and mog_set_tuning refuses values
    outside -1..1."""
    from mog_solver_b200._lib import MogError

    a = make_sim(k=32, g=16, n=1000)
    try:
        assert a.tuning()["solve_split"] == 0
        with pytest.raises(MogError):
            a.tune(solve_split=2)
        assert a.tuning()["solve_split"] == 0
    finally:
        a.close()
