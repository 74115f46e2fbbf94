"""The oracle against the reference's own shaders run live (compiled as C++
by oracle/_ref from the reference checkout), on seeded random cases over
more grid sizes, ensemble sizes and masses than the committed fixtures.
Skipped where oracle/_ref was not built (no reference checkout)."""
import numpy as np
import pytest

import oracle
from oracle import pipeline as pl

rh = pytest.importorskip("oracle.ref_harness")
pytestmark = pytest.mark.skipif(not rh.available(), reason="oracle/_ref not built")


def _case(g, k, n, seed, L=100.0):
    from mog_solver_b200.transforms import compute_transforms

    rng = np.random.default_rng(seed)
    off, rot = compute_transforms(k, g, L, seed=seed)
    pos = np.zeros((n, 4), dtype=np.float32)
    half = n // 2
    pos[:half, :3] = rng.normal(L / 2, L / 8, (half, 3))
    pos[half:, :3] = rng.uniform(0, L, (n - half, 3))
    pos[:, :3] = np.mod(pos[:, :3], np.float32(L)).astype(np.float32)
    pos[:, 3] = rng.choice(np.array([0.5, 1.0, 1.5, 3.0], dtype=np.float32), n)
    vel = np.zeros_like(pos)
    vel[:, :3] = rng.normal(0, 1, (n, 3))
    return pos, vel, off, rot, L


CASES = [(2, 3, 500, 1), (4, 2, 2000, 2), (8, 5, 3000, 3), (16, 2, 4000, 4), (32, 1, 3000, 5)]


@pytest.mark.parametrize("g,k,n,seed", CASES)
def test_deposit_bit_exact_with_live_reference(g, k, n, seed):
    pos, _, off, rot, L = _case(g, k, n, seed)
    ref = rh.deposit(pos, off, rot, g, L)
    got = oracle.deposit(pos, rot, off, g, L, oracle.MASS_U32, 0, oracle.INDEX_EXACT)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("g,k,n,seed", CASES)
def test_update_bit_exact_with_live_reference(g, k, n, seed):
    pos, vel, off, rot, L = _case(g, k, n, seed)
    G, dt, damping = 10.0, 1e-3, 0.999
    grad = rh.solve(rh.deposit(pos, off, rot, g, L), L, G)
    p_ref, v_ref = rh.update(pos, vel, off, rot, grad, g, L, dt, damping)
    p, v = oracle.update(pos, vel, grad, rot, off, g, L, dt, damping, oracle.INDEX_EXACT)
    assert np.array_equal(p.view(np.uint32), p_ref.view(np.uint32))
    assert np.array_equal(v.view(np.uint32), v_ref.view(np.uint32))


@pytest.mark.parametrize("g,k,n,seed", CASES)
def test_solve_f32_transcription_with_live_reference(g, k, n, seed):
    """The FP32 NumPy transcription of the shader chain (including the
    reference's texture aliasing at g = 4, 16) against the shaders."""
    pos, _, off, rot, L = _case(g, k, n, seed)
    G = 10.0
    mass = rh.deposit(pos, off, rot, g, L)
    ref = rh.solve(mass, L, G)
    assert pl.relative_l2(pl.forces_grid_f32(mass, G, L), ref) < 1e-6


def test_perlin_sampler_bit_exact_with_live_reference():
    from mog_solver_b200 import ics

    for shape, seed, buf in (("sphere", 99, 0.1), ("cube", 12345, 0.2)):
        ref_p, ref_v = rh.init_particles(2000, 80.0, 3.0, 1.5, seed, 0.75, buf,
                                         1 if shape == "sphere" else 0)
        p, v = ics.perlin_host(2000, 80.0, 0.75, buf, seed, 3.0, 1.5, shape)
        assert np.array_equal(p.view(np.uint32), ref_p.view(np.uint32))
        assert np.array_equal(v.view(np.uint32), ref_v.view(np.uint32))


@pytest.mark.parametrize("g,k,n,seed", [(8, 3, 2000, 11), (16, 2, 3000, 12), (32, 2, 2500, 13)])
def test_oracle_step_composition_tracks_reference_step(g, k, n, seed):
    """Three of the reference's whole steps (step_fft, compiled as C++) against
    the oracle's stages composed the same way: the first mass grid is
    bit-exact, and the particles stay within 1e-5 relative of the reference
    (the FP32 chain matches the shaders to ~1e-7 per step)."""
    pos, vel, off, rot, L = _case(g, k, n, seed)
    G, dt, damping = 10.0, 1e-3, 0.999
    p_ref, v_ref = pos.copy(), vel.copy()
    p, v = pos.copy(), vel.copy()
    for s in range(3):
        p_ref, v_ref, mass_ref = rh.step(p_ref, v_ref, off, rot, g, L, G, dt, damping)
        mass = oracle.deposit(p, rot, off, g, L, oracle.MASS_U32, 0, oracle.INDEX_EXACT)
        if s == 0:
            assert np.array_equal(mass, mass_ref)
        grad = pl.forces_grid_f32(mass, G, L)
        p, v = oracle.update(p, v, grad, rot, off, g, L, dt, damping, oracle.INDEX_EXACT)
    span = np.abs(p_ref[:, :3] - pos[:, :3]).max()
    assert np.abs(p[:, :3] - p_ref[:, :3]).max() <= 1e-5 * max(span, 1e-3) + 1e-5
    assert pl.relative_l2(v[:, :3], v_ref[:, :3]) < 1e-5
