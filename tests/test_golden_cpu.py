"""The oracle against fixtures generated from the reference itself
(tests/golden/make_golden.py): the reference's transform sampler and
Green's kernel (main.py imported), and its compute shaders run on small
seeded cases (oracle/_ref).  No GPU."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from oracle import pipeline as pl
from mog_solver_b200.transforms import compute_transforms

GOLD = Path(__file__).resolve().parent / "golden"


def _cases():
    T = np.load(GOLD / "transforms.npz")
    return T, sorted({k.rsplit("_", 1)[0] for k in T.files})


@pytest.mark.parametrize("key", _cases()[1])
def test_transforms_match_reference_sampler(key):
    T, _ = _cases()
    p = key.split("_")
    k, g, L, s = int(p[0][1:]), int(p[1][1:]), float(p[2][1:]), int(p[3][1:])
    off, rot = compute_transforms(k, g, L, seed=s)
    assert np.array_equal(off.view(np.uint32), T[key + "_offsets"].view(np.uint32))
    assert np.array_equal(rot.view(np.uint32), T[key + "_rotations"].view(np.uint32))


@pytest.mark.parametrize("g", [8, 16])
def test_green_kernel_table_matches_reference(g):
    """The real-space kernel of init_greens_kernel (main.py:250-278),
    restated in FP64 the way the library builds it."""
    K = np.load(GOLD / "greens_kernel.npz")[f"g{g}"]
    L = 100.0
    voxel = L / g
    sh = pl.shift(g)
    out = np.zeros((g, g, g, 4), dtype=np.float32)
    for iz in range(g):
        for iy in range(g):
            for ix in range(g):
                rx, ry, rz = sh[ix] * voxel, sh[iy] * voxel, sh[iz] * voxel
                r2 = rx * rx + ry * ry + rz * rz
                r = np.sqrt(r2)
                if r > 1e-10:
                    f = 1.0 / (4.0 * np.pi * r2 * r)
                    out[iz, iy, ix, :3] = (rx * f, ry * f, rz * f)
    assert np.array_equal(out.view(np.uint32), K.view(np.uint32))


@pytest.fixture(params=[8, 16])
def shaders(request):
    d = np.load(GOLD / f"shaders_g{request.param}.npz")
    return request.param, d


def test_oracle_deposit_matches_reference_shader(shaders, oracle_lib):
    g, d = shaders
    L = float(d["params"][0])
    m = oracle.deposit(d["pos"], d["rotations"], d["offsets"], g, L, oracle.MASS_U32, 0,
                       oracle.INDEX_EXACT)
    assert np.array_equal(m, d["mass"])


def test_oracle_update_matches_reference_shader(shaders, oracle_lib):
    g, d = shaders
    L, G, dt, damping = (float(x) for x in d["params"])
    p, v = oracle.update(d["pos"], d["vel"], d["grad"], d["rotations"], d["offsets"], g, L, dt,
                         damping, oracle.INDEX_EXACT)
    assert np.array_equal(p.view(np.uint32), d["pos1"].view(np.uint32))
    assert np.array_equal(v.view(np.uint32), d["vel1"].view(np.uint32))


def test_f32_port_matches_reference_shader_chain(shaders):
    g, d = shaders
    L, G = float(d["params"][0]), float(d["params"][1])
    f = pl.forces_grid_f32(d["mass"], G, L)
    assert pl.relative_l2(f, d["grad"]) < 1e-6


def test_fp64_pipeline_matches_reference_components(shaders):
    """y and z match the FP64 ideal chain; x matches it at g = 8 and is the
    z-gradient at g = 16 (the reference's texture aliasing)."""
    g, d = shaders
    L, G = float(d["params"][0]), float(d["params"][1])
    f64 = pl.forces_grid_fp64(d["mass"].astype(np.float64) / 1000.0, G, L)
    grad = d["grad"]
    assert pl.relative_l2(grad[..., 1], f64[..., 1]) < 1e-5
    assert pl.relative_l2(grad[..., 2], f64[..., 2]) < 1e-5
    if pl.texture_aliasing(g):
        assert np.array_equal(grad[..., 0], grad[..., 2])
        assert pl.relative_l2(grad[..., 0], f64[..., 0]) > 0.5
    else:
        assert pl.relative_l2(grad[..., 0], f64[..., 0]) < 1e-5


def test_two_galaxy_initialiser_matches_reference():
    """ics.reference_two_galaxies == the reference's init_particles2
    (main.py:312-357) after np.random.seed, bit for bit (fixture from the
    reference itself)."""
    from mog_solver_b200 import ics

    d = np.load(GOLD / "two_galaxies.npz")
    keys = sorted({k.rsplit("_", 1)[0] for k in d.files})
    assert keys
    for key in keys:
        n, L, m, seed = d[f"{key}_params"]
        pos, vel = ics.reference_two_galaxies(int(n), float(L), float(m), int(seed))
        assert np.array_equal(pos.view(np.uint32), d[f"{key}_pos"].view(np.uint32)), key
        assert np.array_equal(vel.view(np.uint32), d[f"{key}_vel"].view(np.uint32)), key


def test_perlin_sampler_host_matches_reference_shader():
    """mog_init_particles_host == init_particles.glsl (the reference's GPU
    initial-condition sampler, compiled as C++ by oracle/_ref), bit for bit,
    for the reference's default call and a cube-shaped variant."""
    from mog_solver_b200 import ics

    d = np.load(GOLD / "init_particles.npz")
    for key in sorted({k.rsplit("_", 1)[0] for k in d.files}):
        n, L, noise, contrast, seed, m, buf, shape = d[f"{key}_params"]
        pos, vel = ics.perlin_host(int(n), float(L), float(m), float(buf), int(seed), float(noise),
                                   float(contrast), "sphere" if int(shape) == 1 else "cube")
        assert np.array_equal(pos.view(np.uint32), d[f"{key}_pos"].view(np.uint32)), key
        assert np.array_equal(vel.view(np.uint32), d[f"{key}_vel"].view(np.uint32)), key


def test_perlin_sampler_rejects_bad_arguments():
    import ctypes

    from mog_solver_b200 import _lib

    lib = _lib.lib()
    buf = np.zeros((4, 4), np.float32)
    p = buf.ctypes.data_as(ctypes.c_void_p)
    assert lib.mog_init_particles_host(p, p, 4, -1.0, 4.0, 2.0, 1, 1.0, 0.1, 1) == _lib.MOG_ERR_ARG
    assert lib.mog_init_particles_host(p, p, 4, 100.0, 4.0, 2.0, 1, 1.0, 0.1, 2) == _lib.MOG_ERR_ARG
    assert lib.mog_init_particles_host(None, None, 0, 100.0, 4.0, 2.0, 1, 1.0, 0.1, 1) == _lib.MOG_OK
