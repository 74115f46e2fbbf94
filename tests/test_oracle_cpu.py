"""CPU checks of the oracle itself (no GPU).

The oracle is the checker of the CUDA path, so it is pinned here first:
known-answer physics of the FP64 pipeline, agreement between the FP32
shader transcription and the FP64 pipeline, and the two cell-index modes.
"""
import numpy as np
import pytest

import oracle
from oracle import pipeline as pl
from mog_solver_b200.transforms import compute_transforms


def _setup(k=4, g=16, L=100.0, seed=0):
    off, rot = compute_transforms(k, g, L, seed=seed)
    return off, rot


def test_oracle_builds(oracle_lib):
    assert oracle.LIB.exists()


def test_fft_forces_blob_newtonian():
    """A compact mass: far field ~ (h^3/2) G M / r^2 along the separation
    (greens.glsl uses -2 pi G on cell masses and pack.glsl divides by g^3).
    A smooth blob is used because the unfiltered spectral derivative of a
    single NGP cell rings at near-Nyquist wave numbers."""
    g, L, G = 32, 100.0, 3.0
    h = L / g
    z, y, x = np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij")
    rho = np.exp(-((x - 16) ** 2 + (y - 16) ** 2 + (z - 16) ** 2) / (2 * 1.5 ** 2))
    rho /= rho.sum()
    F = pl.forces_grid_fp64(rho[None], G, L)[0]
    for d in (4, 6):
        f = F[16, 16, 16 + d]
        expected = (h ** 3 / 2) * G / (d * h) ** 2
        # points away from the mass (update.glsl's vel -= F dt attracts)
        assert f[0] > 0
        assert abs(f[1]) < 1e-12 and abs(f[2]) < 1e-12
        # periodic images and the removed mean change it by a few per cent
        assert abs(f[0] / expected - 1) < 0.1


def test_fft_forces_uniform_lattice_zero():
    g, L = 16, 100.0
    rho = np.full((2, g, g, g), 0.25)
    F = pl.forces_grid_fp64(rho, 7.0, L)
    assert np.abs(F).max() < 1e-12


def test_fft_forces_translation_covariant():
    g, L = 8, 100.0
    rng = np.random.default_rng(1)
    rho = rng.random((1, g, g, g))
    F = pl.forces_grid_fp64(rho, 1.0, L)
    F2 = pl.forces_grid_fp64(np.roll(rho, (1, 2, 3), axis=(1, 2, 3)), 1.0, L)
    assert np.allclose(np.roll(F, (1, 2, 3), axis=(1, 2, 3)), F2, atol=1e-12)


def test_keep_mask_small_world_drops_low_modes():
    # world 2000 (config.yaml): (2 pi / L)^2 < 1e-4 so the fundamental is dropped
    keep = pl.keep_mask(16, 2000.0)
    assert not keep[0, 0, 1] and not keep[0, 0, 0]
    assert pl.keep_mask(16, 100.0)[0, 0, 1]


def test_f32_shader_chain_matches_fp64(oracle_lib):
    """The FP32 transcription (flushes included) agrees with the FP64 ideal
    chain for unit-scale masses (the reference's u32 x1000 regime)."""
    k, g, L, G = 2, 8, 100.0, 10.0
    off, rot = _setup(k, g, L, seed=3)
    rng = np.random.default_rng(3)
    pos = np.zeros((500, 4), dtype=np.float32)
    pos[:, :3] = rng.uniform(20, 80, (500, 3))
    pos[:, 3] = 1.0
    m = oracle.deposit(pos, rot, off, g, L, oracle.MASS_U32, 0, oracle.INDEX_EXACT)
    assert m.sum() == 500 * 1000 * k
    f32 = pl.forces_grid_f32(m, G, L)
    f64 = pl.forces_grid_fp64(m.astype(np.float64) / 1000.0, G, L)
    assert pl.relative_l2(f32[..., :3], f64) < 1e-4


@pytest.mark.parametrize("g", [8, 16, 32])
def test_fast_and_exact_cells_agree(oracle_lib, g):
    """FAST cells equal the shader's EXACT sequence except within ~1 ulp of a
    cell face."""
    k, L = 16, 100.0
    off, rot = _setup(k, g, L, seed=5)
    rng = np.random.default_rng(5)
    pos = np.zeros((20000, 4), dtype=np.float32)
    pos[:, :3] = rng.uniform(0, L, (20000, 3))
    a = oracle.cells(pos, rot, off, g, L, oracle.INDEX_FAST)
    b = oracle.cells(pos, rot, off, g, L, oracle.INDEX_EXACT)
    assert (a < g ** 3).all() and (b < g ** 3).all()
    mismatch = np.mean(a != b)
    assert mismatch < 1e-4, mismatch


def test_deposit_conserves_mass(oracle_lib):
    k, g, L = 3, 16, 100.0
    off, rot = _setup(k, g, L, seed=2)
    rng = np.random.default_rng(2)
    n = 257
    pos = np.zeros((n, 4), dtype=np.float32)
    pos[:, :3] = rng.uniform(0, L, (n, 3))
    pos[:, 3] = 1.0 / 256
    m = oracle.deposit(pos, rot, off, g, L, oracle.MASS_U64, 40, oracle.INDEX_FAST)
    assert m.dtype == np.uint64
    per_grid = m.reshape(k, -1).sum(axis=1)
    assert (per_grid == n * (2 ** 40 // 256)).all()


def test_reference_mass_quantisation_truncates_small_masses(oracle_lib):
    """uint(m * 1000) is 0 for m = 1/65536: the reference's mass grid is empty
    at the benchmark masses (why the u64 fixed-point mode exists)."""
    k, g, L = 2, 8, 100.0
    off, rot = _setup(k, g, L)
    pos = np.array([[10, 20, 30, 1 / 65536]], dtype=np.float32)
    m = oracle.deposit(pos, rot, off, g, L, oracle.MASS_U32, 0, oracle.INDEX_EXACT)
    assert m.sum() == 0


def test_update_oracle_known_answer(oracle_lib):
    """Uniform force grid: every particle feels exactly the rotated constant."""
    k, g, L = 2, 4, 100.0
    off, rot = _setup(k, g, L)
    f = np.zeros((k, g, g, g, 4), dtype=np.float32)
    f[..., 0] = 1.0
    pos = np.array([[10, 20, 30, 1], [50, 50, 50, 1]], dtype=np.float32)
    vel = np.zeros_like(pos)
    acc = oracle.averaged_force(pos, f, rot, off, g, L)
    M = rot.reshape(k, 3, 4)[:, :, :3]
    expect = M[:, :, 0].mean(axis=0)
    assert np.allclose(acc[0, :3], expect, atol=1e-6)
    p2, v2 = oracle.update(pos, vel, f, rot, off, g, L, dt=0.5, damping=1.0)
    assert np.allclose(v2[:, :3], -0.5 * acc[:, :3], atol=1e-6)


def test_direct_sum_two_body():
    L = 100.0
    t = np.array([[50.0, 50.0, 50.0]])
    s = np.array([[53.0, 50.0, 50.0]])
    f = pl.direct_sum_fp64(t, s, np.array([2.0]), L, g_eff=1.5)
    assert np.allclose(f, [[-1.5 * 2.0 / 9.0, 0, 0]])
