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


def _expected_stats(pos, vel, W, H, scale, v, p):
    """(point, tile) pairs and kernel launches of one frame, from the
    oracle's vertex stage and the renderer's binning rule (a one-pixel
    margin around each point's square, 16 x 16 tiles)."""
    from oracle import render as O

    clip, _, _ = O.vertex_stage(pos, vel, v, p, 100.0, scale)
    x, y, z, w = (clip[:, i] for i in range(4))
    keep = (w > 0) & (x >= -w) & (x <= w) & (y >= -w) & (y <= w) & (z >= -w) & (z <= w)
    F = np.float32
    xw = (x[keep] / w[keep]) * F(W * 0.5) + F(W * 0.5)
    yw = (y[keep] / w[keep]) * F(H * 0.5) + F(H * 0.5)
    h = F(1.0) * F(0.5)
    i0 = np.maximum(np.floor(xw - h).astype(int) - 1, 0)
    i1 = np.minimum(np.floor(xw + h).astype(int) + 1, W - 1)
    j0 = np.maximum(np.floor(yw - h).astype(int) - 1, 0)
    j1 = np.minimum(np.floor(yw + h).astype(int) + 1, H - 1)
    ok = (i0 <= i1) & (j0 <= j1)
    pairs = int(((i1 // 16 - i0 // 16 + 1) * (j1 // 16 - j0 // 16 + 1))[ok].sum())

    def scans(m):
        nb = -(-m // 2048)
        return 1 if nb <= 1 else 2 + scans(nb)

    tiles = -(-W // 16) * -(-H // 16)
    passes = -(-int(np.ceil(np.log2(tiles))) // 8) if tiles > 1 else 0
    hn = -(-pairs // 2048) * 256
    launches = 1 + scans(len(pos)) + passes * (2 + scans(hn)) + 3 if pairs else 1 + scans(len(pos)) + 1
    return pairs, launches


def test_renderer_stats():
    from mog_solver_b200 import render as R

    n, W, H, scale = 50000, 700, 300, 0.3
    pos, vel = _particles(n, 11)
    v, p = R.camera_matrices(aspect=W / H)
    r = R.Renderer()
    try:
        r.render(torch.from_numpy(pos).cuda(), torch.from_numpy(vel).cuda(), width=W, height=H,
                 world_size=100.0, speed_scale=scale, m_view=v, m_proj=p)
        torch.cuda.synchronize()
        pairs, launches = _expected_stats(pos, vel, W, H, scale, v, p)
        assert r.stats() == {"pairs": pairs, "launches": launches}
    finally:
        r.close()
