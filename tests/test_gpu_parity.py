"""Parity of the CUDA path (libmog.so through the C ABI) with the oracle.

* mass grids: bit-exact against the C integer-histogram oracle (both index
  modes, both fixed-point modes, equal and unequal masses, odd sizes);
* particle update: bit-exact against the C restatement of update.glsl,
  given the same force grid (direct and shared-memory-staged kernels);
* spectral solve: relative L2 <= 1e-5 against the FP64 ideal pipeline;
* end-to-end forces: relative L2 <= 1e-5 against the FP64 pipeline;
* determinism, CUDA-graph replay, convolution solver, FP64 diagnostics and
  device status flags.
"""
import numpy as np
import pytest

import oracle
from oracle import pipeline as pl

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5  # relative L2 against the FP64 oracle (FP32 path)


def make_sim(k=4, g=16, L=100.0, G=100.0, n=1000, seed=0, mass_mode="u64", index_mode="fast",
             solver="fft", dt=1e-5, damping=0.999, scale_bits=None):
    from mog_solver_b200 import Simulation

    cfg = {"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": G, "dt": dt,
           "damping": damping, "solver": solver, "seed": seed, "mass_mode": mass_mode,
           "index_mode": index_mode, "scale_bits": scale_bits}
    return Simulation(cfg)


def particles(n, L=100.0, seed=0, equal_mass=True, mass=None, clustered=True):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), dtype=np.float32)
    if clustered:
        nc = n // 2
        pos[:nc, :3] = rng.normal(L / 2, L / 12, (nc, 3))
        pos[nc:, :3] = rng.uniform(0, L, (n - nc, 3))
        pos[:, :3] = np.mod(pos[:, :3], np.float32(L))
    else:
        pos[:, :3] = rng.uniform(0, L, (n, 3))
    if mass is not None:
        pos[:, 3] = mass
    elif equal_mass:
        pos[:, 3] = 1.0 / max(n, 1)
    else:
        pos[:, 3] = rng.uniform(0.5, 2.0, n) / max(n, 1)
    vel = np.zeros_like(pos)
    vel[:, :3] = rng.normal(0, 1, (n, 3))
    return pos, vel


MODES = [("u64", "fast"), ("u64", "exact"), ("u32x1000", "fast"), ("u32x1000", "exact")]
SHAPES = [(1, 1, 8), (7, 3, 16), (257, 16, 16), (65536, 16, 16), (5000, 5, 32), (3000, 2, 4),
          (4096, 3, 64)]


# launch shapes that take different code paths; none may change a bit
DEPOSIT_TUNINGS = {
    "sorted+merged": dict(sort_every=1, deposit_aggregate=-1, deposit_sorted=1),
    "unsorted": dict(sort_every=0, deposit_aggregate=0),
    "sorted+plain": dict(sort_every=1, deposit_aggregate=0, deposit_ppt=1, deposit_sorted=1),
    "sorted-update-only": dict(sort_every=1),
    "unsorted+merged": dict(sort_every=0, deposit_aggregate=1, deposit_ppt=2),
    "global": dict(sort_every=0, deposit_grids_per_cta=-1),
    "generic": dict(sort_every=0, deposit_generic=1),
    "fast-ppt1": dict(sort_every=0, deposit_ppt=1, deposit_grids_per_cta=2),
}


@pytest.mark.parametrize("mass_mode,index_mode", MODES)
@pytest.mark.parametrize("n,k,g", SHAPES)
@pytest.mark.parametrize("equal_mass", [True, False])
@pytest.mark.parametrize("tuning", ["sorted+merged", "unsorted", "generic"])
def test_deposit_bit_exact(mass_mode, index_mode, n, k, g, equal_mass, tuning):
    L = 100.0
    sim = make_sim(k=k, g=g, L=L, n=n, mass_mode=mass_mode, index_mode=index_mode, seed=n + k)
    sim.tune(**DEPOSIT_TUNINGS[tuning])
    mass = None
    if mass_mode == "u32x1000":
        mass = 1.0 if equal_mass else np.random.default_rng(1).uniform(0.5, 3.0, n).astype(np.float32)
    pos, vel = particles(n, L, seed=k, equal_mass=equal_mass, mass=mass)
    sim.set_particles(pos, vel)
    got = sim.mass_grid().cpu().numpy()
    mm = oracle.MASS_U64 if mass_mode == "u64" else oracle.MASS_U32
    im = oracle.INDEX_FAST if index_mode == "fast" else oracle.INDEX_EXACT
    bits = sim.scale_bits
    ref = oracle.deposit(pos, sim.rotations, sim.offsets, g, L, mm, bits, im)
    got = got.view(np.uint64 if mm == oracle.MASS_U64 else np.uint32)
    assert got.shape == ref.shape
    assert np.array_equal(got, ref), int((got != ref).sum())
    assert sim.status() == 0


@pytest.mark.parametrize("tuning", sorted(DEPOSIT_TUNINGS))
@pytest.mark.parametrize("mass_mode", ["u64", "u32x1000"])
def test_deposit_tunings_bit_exact(tuning, mass_mode):
    n, k, g, L = 100000, 12, 16, 100.0
    sim = make_sim(k=k, g=g, L=L, n=n, mass_mode=mass_mode)
    sim.tune(**DEPOSIT_TUNINGS[tuning])
    mass = 1.0 if mass_mode == "u32x1000" else None
    for equal in (True, False):
        m = mass if (mass is None or equal) else np.random.default_rng(2).uniform(0.5, 2, n)
        pos, vel = particles(n, L, seed=6, equal_mass=equal, mass=m)
        sim.set_particles(pos, vel)
        got = sim.mass_grid().cpu().numpy()
        mm = oracle.MASS_U64 if mass_mode == "u64" else oracle.MASS_U32
        ref = oracle.deposit(pos, sim.rotations, sim.offsets, g, L, mm, sim.scale_bits)
        assert np.array_equal(got.view(ref.dtype), ref)


@pytest.mark.parametrize("mass_mode", ["u64", "u32x1000"])
def test_deposit_g32_bit_exact(mass_mode):
    """g = 32: the split histogram (u64: high words in shared memory, low
    halves as global atomics) and the one-word histogram (u32)."""
    n, k, g, L = 131072, 5, 32, 100.0  # 2^17: equal masses have a zero low half
    sim = make_sim(k=k, g=g, L=L, n=n, mass_mode=mass_mode)
    for equal in (True, False):
        if mass_mode == "u32x1000":
            m = None if equal else np.random.default_rng(4).uniform(0.5, 2, n)
            pos, vel = particles(n, L, seed=8, equal_mass=equal, mass=1.0 if equal else m)
        else:
            m = None if equal else np.random.default_rng(4).uniform(0.5, 2, n) / n
            pos, vel = particles(n, L, seed=8, equal_mass=equal, mass=m)
        sim.set_particles(pos, vel)
        got = sim.mass_grid().cpu().numpy()
        mm = oracle.MASS_U64 if mass_mode == "u64" else oracle.MASS_U32
        ref = oracle.deposit(pos, sim.rotations, sim.offsets, g, L, mm, sim.scale_bits)
        assert np.array_equal(got.view(ref.dtype), ref)


def test_deposit_repeat_is_identical():
    sim = make_sim(k=32, g=16, n=200000)
    pos, vel = particles(200000, seed=3)
    sim.set_particles(pos, vel)
    a = sim.mass_grid().cpu().numpy()
    b = sim.mass_grid().cpu().numpy()
    assert np.array_equal(a, b)


UPDATE_TUNINGS = {
    "auto": dict(),
    "unsorted": dict(sort_every=0),
    "direct4": dict(update_staged=0, update_direct_ppt=4),
    "direct1-unsorted": dict(update_staged=0, update_direct_ppt=1, sort_every=0),
    "staged768": dict(update_staged=1, update_threads=768, sort_every=0),
    "staged1024-sorted": dict(update_staged=1, update_threads=1024, sort_every=1),
}


@pytest.mark.parametrize("index_mode", ["fast", "exact"])
@pytest.mark.parametrize("n,k,g", [(1, 1, 8), (1000, 3, 16), (200000, 24, 16), (3000, 4, 32),
                                   (160000, 8, 8), (1 << 20, 4, 16)])
@pytest.mark.parametrize("tuning", sorted(UPDATE_TUNINGS))
def test_update_bit_exact(index_mode, n, k, g, tuning):
    """update.glsl from one force grid: GPU (direct or staged) == C oracle."""
    L = 100.0
    sim = make_sim(k=k, g=g, L=L, n=n, index_mode=index_mode, dt=3e-3, damping=0.97)
    sim.tune(**UPDATE_TUNINGS[tuning])
    pos, vel = particles(n, L, seed=11)
    sim.set_particles(pos, vel)
    rng = np.random.default_rng(5)
    f = rng.normal(0, 10, (k, g, g, g, 4)).astype(np.float32)
    sim.update_from_grid(torch.from_numpy(f).cuda(), dt_eff=3e-3)
    im = oracle.INDEX_FAST if index_mode == "fast" else oracle.INDEX_EXACT
    p_ref, v_ref = oracle.update(pos, vel, f, sim.rotations, sim.offsets, g, L, 3e-3, 0.97, im)
    p = sim.pos.cpu().numpy()
    v = sim.vel.cpu().numpy()
    assert np.array_equal(p.view(np.uint32), p_ref.view(np.uint32))
    assert np.array_equal(v.view(np.uint32), v_ref.view(np.uint32))


@pytest.mark.parametrize("mass_mode", ["u64", "u32x1000"])
@pytest.mark.parametrize("k,g", [(1, 2), (3, 4), (5, 8), (16, 16), (3, 32), (2, 64)])
def test_solve_matches_fp64(mass_mode, k, g):
    L, G = 100.0, 100.0
    n = 20000
    sim = make_sim(k=k, g=g, L=L, G=G, n=n, mass_mode=mass_mode)
    mass = 1.0 if mass_mode == "u32x1000" else None
    pos, vel = particles(n, L, seed=g, mass=mass)
    sim.set_particles(pos, vel)
    m = sim.mass_grid()
    F = sim.solve_grid(m).cpu().numpy()
    mm = m.cpu().numpy()
    if mass_mode == "u64":
        rho = mm.view(np.uint64).astype(np.float64) * 2.0 ** -sim.scale_bits
    else:
        rho = mm.view(np.uint32).astype(np.float64) / 1000.0
    ref = pl.forces_grid_fp64(rho, G, L)
    err = pl.relative_l2(F[..., :3], ref)
    assert err <= FORCE_TOL, err
    mag = np.sqrt((F[..., :3].astype(np.float64) ** 2).sum(-1))
    assert np.allclose(F[..., 3], mag, rtol=1e-5, atol=1e-30)


@pytest.mark.parametrize("index_mode", ["fast", "exact"])
def test_forces_match_fp64_pipeline(index_mode):
    """c1-like: N=65,536 uniform, k=16, g=16, G=100."""
    n, k, g, L, G = 65536, 16, 16, 100.0, 100.0
    sim = make_sim(k=k, g=g, L=L, G=G, n=n, index_mode=index_mode)
    pos, vel = particles(n, L, seed=0, clustered=False)
    sim.set_particles(pos, vel)
    acc = sim.forces().cpu().numpy()[:, :3]
    im = oracle.INDEX_FAST if index_mode == "fast" else oracle.INDEX_EXACT
    mass = oracle.deposit(pos, sim.rotations, sim.offsets, g, L, oracle.MASS_U64,
                          sim.scale_bits, im)
    rho = mass.astype(np.float64) * 2.0 ** -sim.scale_bits
    fgrid = pl.forces_grid_fp64(rho, G, L)
    cells = oracle.cells(pos, sim.rotations, sim.offsets, g, L, im)
    ref = pl.gather_fp64(cells, fgrid, sim.rotations)
    err = pl.relative_l2(acc, ref)
    assert err <= FORCE_TOL, err


def test_step_equals_stagewise_oracle():
    """One production step (world-frame forces, fused zeroing) == deposit ->
    solve (grid frame) -> C update oracle, bit for bit."""
    n, k, g, L = 200000, 24, 16, 100.0
    sim = make_sim(k=k, g=g, L=L, n=n, dt=1e-3, damping=0.999)
    pos, vel = particles(n, L, seed=21)
    sim.set_particles(pos, vel)
    F = sim.solve_grid(sim.mass_grid()).cpu().numpy()
    p_ref, v_ref = oracle.update(pos, vel, F, sim.rotations, sim.offsets, g, L, 1e-3, 0.999)
    sim.step()
    assert np.array_equal(sim.pos.cpu().numpy().view(np.uint32), p_ref.view(np.uint32))
    assert np.array_equal(sim.vel.cpu().numpy().view(np.uint32), v_ref.view(np.uint32))
    # and the next step starts from a cleared mass grid
    F2 = sim.solve_grid(sim.mass_grid()).cpu().numpy()
    p2, v2 = oracle.update(p_ref, v_ref, F2, sim.rotations, sim.offsets, g, L, 1e-3, 0.999)
    sim.step()
    assert np.array_equal(sim.pos.cpu().numpy().view(np.uint32), p2.view(np.uint32))


def test_graph_replay_equals_single_steps():
    n, k, g = 30000, 8, 16
    a = make_sim(k=k, g=g, n=n, dt=1e-3)
    b = make_sim(k=k, g=g, n=n, dt=1e-3)
    pos, vel = particles(n, seed=4)
    a.set_particles(pos, vel)
    b.set_particles(pos, vel)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        a.step(5)
        a.step(3)
    s.synchronize()
    for _ in range(8):
        b.step()
    torch.cuda.synchronize()
    assert torch.equal(a.pos, b.pos) and torch.equal(a.vel, b.vel)


def test_ten_steps_track_fp64_pipeline():
    """c1 for 10 steps: the FP32 GPU trajectory stays within 1e-5 (relative
    L2 of the velocity change) of a trajectory driven by FP64 forces."""
    n, k, g, L, G, dt = 65536, 16, 16, 100.0, 100.0, 1e-5
    sim = make_sim(k=k, g=g, L=L, G=G, n=n, dt=dt, damping=0.999)
    pos, vel = particles(n, L, seed=0, clustered=False)
    vel[:] = 0
    sim.set_particles(pos, vel)
    bits = sim.scale_bits
    p, v = pos.astype(np.float64), vel.astype(np.float64)
    for _ in range(10):
        p32 = p.astype(np.float32)
        mass = oracle.deposit(p32, sim.rotations, sim.offsets, g, L, oracle.MASS_U64, bits)
        fgrid = pl.forces_grid_fp64(mass.astype(np.float64) * 2.0 ** -bits, G, L)
        cells = oracle.cells(p32, sim.rotations, sim.offsets, g, L)
        acc = pl.gather_fp64(cells, fgrid, sim.rotations)
        v[:, :3] = (v[:, :3] - acc * dt) * 0.999
        p[:, :3] = np.mod(p[:, :3] + v[:, :3] * dt, L)
    sim.step(10)
    err = pl.relative_l2(sim.vel.cpu().numpy()[:, :3], v[:, :3])
    assert err <= FORCE_TOL, err


def test_convolution_solver_matches_fp64():
    k, g, L, G = 2, 8, 100.0, 5.0
    n = 3000
    sim = make_sim(k=k, g=g, L=L, G=G, n=n, solver="convolution")
    pos, vel = particles(n, L, seed=9)
    sim.set_particles(pos, vel)
    m = sim.mass_grid()
    F = sim.solve_grid(m).cpu().numpy()[..., :3]
    rho = m.cpu().numpy().view(np.uint64).astype(np.float64) * 2.0 ** -sim.scale_bits
    h = L / g
    sh = pl.shift(g)
    d = sh * h
    dz, dy, dx = np.meshgrid(d, d, d, indexing="ij")
    r = np.sqrt(dx * dx + dy * dy + dz * dz)
    with np.errstate(divide="ignore", invalid="ignore"):
        fac = np.where(r > 1e-10, 1.0 / (4 * np.pi * r ** 3), 0.0)
    K = np.stack([dx * fac, dy * fac, dz * fac], -1).astype(np.float32).astype(np.float64)
    ref = np.zeros((k, g, g, g, 3))
    idx = np.arange(g)
    for i in range(k):
        for z in range(g):
            for y in range(g):
                for x in range(g):
                    kk = K[(z - idx)[:, None, None] % g, (y - idx)[None, :, None] % g,
                           (x - idx)[None, None, :] % g]
                    ref[i, z, y, x] = (rho[i][..., None] * kk).sum((0, 1, 2))
    ref *= 2 * np.pi * G * h ** 3
    assert pl.relative_l2(F, ref) <= FORCE_TOL


def test_diagnostics_fp64():
    n = 100000
    sim = make_sim(n=n)
    pos, vel = particles(n, seed=8, equal_mass=False)
    sim.set_particles(pos, vel)
    d = sim.diagnostics()
    m = pos[:, 3].astype(np.float64)
    v = vel[:, :3].astype(np.float64)
    assert np.allclose(d["momentum"], (m[:, None] * v).sum(0), rtol=1e-12, atol=1e-15)
    assert np.isclose(d["kinetic_energy"], 0.5 * (m * (v * v).sum(1)).sum(), rtol=1e-12)
    assert np.isclose(d["mass"], m.sum(), rtol=1e-12)
    com = (m[:, None] * pos[:, :3].astype(np.float64)).sum(0) / m.sum()
    assert np.allclose(d["com"], com, rtol=1e-12)


def test_status_flags():
    from mog_solver_b200 import FLAG_BADMASS, FLAG_NONFINITE, FLAG_OVERFLOW

    n = 1000
    sim = make_sim(n=n, dt=1e-3)
    pos, vel = particles(n, seed=2)
    vel[5, 0] = np.inf
    sim.set_particles(pos, vel)
    sim.step()
    assert sim.status() & FLAG_NONFINITE
    assert sim.status() == 0  # read-and-clear
    pos2 = pos.copy()
    pos2[3, 3] = -1.0
    sim.set_particles(pos2, np.zeros_like(pos2))
    sim.mass_grid()
    assert sim.status() & FLAG_BADMASS
    big = make_sim(n=n, scale_bits=100)
    pos3 = pos.copy()
    pos3[:, 3] = 1.0
    big.set_particles(pos3, np.zeros_like(pos3))
    big.mass_grid()
    assert big.status() & FLAG_OVERFLOW
