"""The CUDA renderer (mog_render) against its host twin (mog_render_host,
pinned to the oracle by tests/test_render_cpu.py): bit-identical images
for every tile-count regime of the sort (one tile: no pass; up to 256
tiles: one pass; more: two), both point-size modes and both targets."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _particles(n, seed, lo=-10.0, hi=110.0):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    half = n // 2
    pos[:half, :3] = rng.normal(50.0, 8.0, (half, 3))  # a dense clump: long tile lists
    pos[half:, :3] = rng.uniform(lo, hi, (n - half, 3))
    pos[:, 3] = 1.0 / max(n, 1)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 3.0, (n, 3))
    return pos, vel


CASES = [
    # n, W, H, point_mode, fmt, speed_scale, camera (rx, ry, dist), point_size, max size
    (20000, 64, 48, "fixed", "rgba8", 0.3, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (20000, 16, 16, "fixed", "rgba8", 0.3, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (5000, 13, 7, "program", "rgba32f", 0.5, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (4096, 640, 360, "program", "rgba8", 1.0, (30.0, 20.0, 2.0), 1.0, 64.0),
    (100000, 333, 201, "fixed", "rgba32f", 0.2, (-100.0, 60.0, 1.5), 2.5, 2047.0),
    (1 << 20, 2560, 1440, "fixed", "rgba8", 0.0, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (0, 100, 50, "fixed", "rgba8", 0.0, (0.0, 0.0, 3.0), 1.0, 2047.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c[0]}_{c[1]}x{c[2]}_{c[3]}_{c[4]}")
def test_cuda_renderer_equals_host_twin(case):
    from mog_solver_b200 import render as R

    n, W, H, mode, fmt, scale, cam, ps, maxps = case
    pos, vel = _particles(n, n + W)
    v, p = R.camera_matrices(*cam, W / H)
    kw = dict(width=W, height=H, world_size=100.0, speed_scale=scale, point_mode=mode,
              point_size=ps, max_point_size=maxps, fmt=fmt, m_view=v, m_proj=p)
    got = R.render(torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda(), **kw)
    torch.cuda.synchronize()
    ref = R.render_host(pos, vel, **kw)
    got = got.cpu().numpy()
    assert got.shape == ref.shape == (H, W, 4)
    assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))


def test_renderer_reuse_across_sizes():
    """One Renderer, growing and shrinking workloads: every frame equals the
    host twin."""
    from mog_solver_b200 import render as R

    r = R.Renderer()
    try:
        for n, W, H in [(1000, 32, 32), (200000, 800, 600), (10, 8, 8), (50000, 1000, 100)]:
            pos, vel = _particles(n, W)
            kw = dict(width=W, height=H, world_size=100.0, speed_scale=0.4)
            got = r.render(torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda(), **kw)
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy(), R.render_host(pos, vel, **kw)), (n, W, H)
    finally:
        r.close()


def test_simulation_render_matches_host():
    from mog_solver_b200 import Simulation, render as R

    sim = Simulation({"n_grids": 4, "grid_size": 16, "world_size": 100.0, "num_particles": 30000,
                      "G": 100.0, "dt": 1e-3, "damping": 0.999, "seed": 0})
    sim.init_particles("two_galaxies", seed=3)
    sim.step(2)
    img = sim.render(width=320, height=180, speed_scale=0.2)
    torch.cuda.synchronize()
    ref = R.render_host(sim.pos.cpu().numpy(), sim.vel.cpu().numpy(), width=320, height=180,
                        world_size=100.0, speed_scale=0.2)
    assert np.array_equal(img.cpu().numpy(), ref)
