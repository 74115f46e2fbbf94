"""The headless particle renderer on the CPU: the oracle (oracle/render.py)
pinned to the reference's own shaders and camera code, the library's host
twin (mog_render_host, the same arithmetic the CUDA kernels run) equal to
the oracle bit for bit, and known answers for the GL point rules."""
import ctypes
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

from oracle import render as O

GOLD = Path(__file__).resolve().parent / "golden"


def _lib():
    from mog_solver_b200 import _lib

    return _lib


def test_camera_matrices_match_reference_uniform_bytes():
    """camera_matrices == the m_view / m_proj bytes on_render writes
    (main.py:685-700), bit for bit."""
    from mog_solver_b200.render import camera_matrices

    d = np.load(GOLD / "camera.npz")
    keys = sorted({k.split("_", 1)[0] for k in d.files})
    assert len(keys) == 5
    for key in keys:
        rx, ry, dist, aspect = d[f"{key}_params"]
        v, p = camera_matrices(rx, ry, dist, aspect)
        assert np.array_equal(v.view(np.uint32), d[f"{key}_m_view"].view(np.uint32)), key
        assert np.array_equal(p.view(np.uint32), d[f"{key}_m_proj"].view(np.uint32)), key


def test_oracle_vertex_stage_matches_reference_shader():
    """Clip position, the shader's point size and v_speed of the reference's
    vertex shader (compiled as C++), bit for bit."""
    d = np.load(GOLD / "point_shaders.npz")
    cases = sorted({k.rsplit("_", 1)[0] for k in d.files if k.endswith("_clip")})
    assert len(cases) == 6
    for case in cases:
        cam = case.split("_")[0]
        world, scale = d[f"{case}_params"]
        clip, size, v_speed = O.vertex_stage(d["pos"], d["vel"], d[f"{cam}_m_view"],
                                             d[f"{cam}_m_proj"], world, scale)
        assert np.array_equal(clip.view(np.uint32), d[f"{case}_clip"].view(np.uint32)), case
        assert np.array_equal(size.view(np.uint32), d[f"{case}_size"].view(np.uint32)), case
        assert np.array_equal(v_speed.view(np.uint32), d[f"{case}_v_speed"].view(np.uint32)), case


def test_oracle_fragment_stage_matches_reference_shader():
    """Discard decision and colour bit for bit; alpha within 2 ulp (GLSL
    allows exp an error of 3 + 2|x| ulp; the compiled reference uses the C
    library's expf)."""
    d = np.load(GOLD / "point_shaders.npz")
    colour, kept = O.fragment_stage(d["frag_point_coord"], d["frag_v_speed"])
    assert np.array_equal(kept, d["frag_kept"])
    assert kept.sum() > 1000 and (~kept).sum() > 100
    ref = d["frag_colour"][kept]
    got = colour[kept]
    assert np.array_equal(got[:, :3].view(np.uint32), ref[:, :3].view(np.uint32))
    ulp = np.abs(got[:, 3].view(np.int32).astype(np.int64) - ref[:, 3].view(np.int32))
    assert ulp.max() <= 2


def test_exp_within_two_ulp():
    x = np.concatenate([np.linspace(-87.0, 88.0, 200001), np.linspace(-3.5, 0.0, 100001)])
    x = x.astype(np.float32)
    got = O.exp_rn(x)
    ref = np.exp(x.astype(np.float64)).astype(np.float32)
    ulp = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32))
    assert ulp.max() <= 2
    assert O.exp_rn(np.float32(0.0)) == 1.0


def _particles(n, seed, lo=0.0, hi=100.0):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(lo, hi, (n, 3))
    pos[:, 3] = 1.0 / max(n, 1)
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 3.0, (n, 3))
    return pos, vel


CASES = [
    # n, W, H, seed, point_mode, fmt, speed_scale, camera (rx, ry, dist), point_size, max size
    (2000, 64, 48, 0, "fixed", "rgba8", 0.0, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (2000, 64, 48, 1, "fixed", "rgba32f", 0.3, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (500, 64, 48, 2, "program", "rgba8", 0.5, (0.0, 0.0, 3.0), 1.0, 2047.0),
    (300, 97, 53, 3, "program", "rgba32f", 1.0, (30.0, 20.0, 2.0), 1.0, 2047.0),
    (3000, 128, 72, 4, "fixed", "rgba8", 0.2, (0.0, 0.0, 3.0), 3.0, 2047.0),
    (1000, 40, 40, 5, "program", "rgba8", 0.7, (-100.0, 60.0, 1.5), 1.0, 20.0),
    (1500, 17, 33, 6, "fixed", "rgba8", 2.0, (200.0, -30.0, 0.8), 2.5, 2047.0),
    (0, 31, 9, 7, "fixed", "rgba8", 0.0, (0.0, 0.0, 3.0), 1.0, 2047.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"n{c[0]}_{c[1]}x{c[2]}_{c[4]}_{c[5]}")
def test_host_renderer_equals_oracle(case):
    from mog_solver_b200 import render as R

    n, W, H, seed, mode, fmt, scale, cam, ps, maxps = case
    pos, vel = _particles(n, seed, -10.0, 110.0)
    v, p = R.camera_matrices(*cam, W / H)
    kw = dict(width=W, height=H, world_size=100.0, speed_scale=scale, point_mode=mode,
              point_size=ps, max_point_size=maxps, fmt=fmt)
    got = R.render_host(pos, vel, m_view=v, m_proj=p, **kw)
    ref = O.render(pos, vel, m_view=v, m_proj=p, **kw)
    assert got.shape == ref.shape == (H, W, 4)
    assert np.array_equal(got.view(np.uint8), ref.view(np.uint8))
    if n:
        assert (got != got[0, 0]).any()  # something was drawn


# Known answers.  With identity matrices and world_size = W = H = 8 the
# window position of a particle is its (x, y): p = pos / 8 * 2 - 1 and
# x_w = 4 p + 4 are exact.
def _kat(pos, vel=None, **kw):
    from mog_solver_b200 import render as R

    pos = np.asarray(pos, np.float32).reshape(-1, 4)
    vel = np.zeros_like(pos) if vel is None else np.asarray(vel, np.float32).reshape(-1, 4)
    eye = np.eye(4, dtype=np.float32).reshape(16)
    args = dict(width=8, height=8, world_size=8.0, m_view=eye, m_proj=eye)
    args.update(kw)
    return R.render_host(pos, vel, **args)


CLEAR8 = np.array([3, 3, 5, 0], np.uint8)  # round((0.01, 0.01, 0.02, 0) * 255)


def test_point_at_a_pixel_centre_draws_that_pixel():
    img = _kat([2.5, 5.5, 4.0, 1.0])
    changed = np.argwhere((img != CLEAR8).any(axis=2))
    # GL row 5 from the bottom is image row 8 - 1 - 5 = 2
    assert changed.tolist() == [[2, 2]]
    # coord = 0, alpha = 0.8, colour (0.05, 0.1, 0.4) over the clear colour
    assert img[2, 2].tolist() == [11, 21, 83, 163]


def test_point_at_a_pixel_corner_is_discarded():
    """Size 1 on the corner (3, 4): the covered pixel's centre is half a
    pixel away on both axes, gl_PointCoord = (0, 1), r = 2 > 1."""
    img = _kat([3.0, 4.0, 4.0, 1.0])
    assert (img == CLEAR8).all()


def test_points_outside_the_view_volume_are_clipped():
    img = _kat([[2.5, 5.5, 9.0, 1.0], [2.5, 5.5, -0.5, 1.0], [8.5, 1.5, 4.0, 1.0]])
    assert (img == CLEAR8).all()


def test_blending_follows_particle_order():
    """Two points on one pixel with different colours: the later one is on top."""
    pos = [[2.5, 2.5, 4.0, 1.0], [2.5, 2.5, 4.0, 1.0]]
    vel = [[0.0, 0.0, 0.0, 0.0], [100.0, 0.0, 0.0, 0.0]]  # speeds 0 and 100 -> t = 0 and 1
    a = _kat(pos, vel, speed_scale=1.0)
    b = _kat(pos[::-1], vel[::-1], speed_scale=1.0)
    assert not np.array_equal(a, b)
    assert a[5, 2, 0] > a[5, 2, 2]  # the hot core colour (1, 0.9, 0.7) drawn last
    assert b[5, 2, 2] > b[5, 2, 0]  # the cold colour (0.05, 0.1, 0.4) drawn last


def test_program_point_size_draws_a_round_sprite():
    """w = 1, so the shader's size is 800 / 1.1, clamped to 5.  Centred on
    pixel (4, 4), the square [2, 7) holds the centres of pixels 2..6 on each
    axis, at gl_PointCoord offsets u, v in {-0.8, -0.4, 0, 0.4, 0.8}; the
    four corners (r = 1.28) are discarded."""
    img = _kat([4.5, 4.5, 4.0, 1.0], point_mode="program", max_point_size=5.0, fmt="rgba32f")
    drawn = (img[..., 3] > 0).astype(int)
    assert drawn.sum() == 21
    block = drawn[1:6, 2:7]  # GL rows 6..2 are image rows 1..5
    assert block.tolist() == [[0, 1, 1, 1, 0], [1, 1, 1, 1, 1], [1, 1, 1, 1, 1],
                              [1, 1, 1, 1, 1], [0, 1, 1, 1, 0]]
    sprite = img[1:6, 2:7]
    # symmetric up to the rounding of gl_PointCoord (0.5 +- 0.4 are not mirror images in binary32)
    np.testing.assert_allclose(sprite, sprite[:, ::-1], rtol=1e-5)
    np.testing.assert_allclose(sprite, sprite[::-1], rtol=1e-5)
    assert sprite[2, 2, 3] == np.float32(0.8) * np.float32(0.8)  # the centre: r = 0


def test_half_open_square_on_an_even_size():
    """Size 4 centred on the pixel corner (4, 4): the square [2, 6) holds
    centres 2.5..5.5, u, v in {-0.75, -0.25, 0.25, 0.75}; r = 1.125 at the
    corners is discarded: 12 pixels."""
    img = _kat([4.0, 4.0, 4.0, 1.0], point_mode="fixed", point_size=4.0, fmt="rgba32f")
    assert (img[..., 3] > 0).sum() == 12


def test_float_target_alpha_is_the_sprite_alpha():
    img = _kat([2.5, 5.5, 4.0, 1.0], fmt="rgba32f")
    assert img[2, 2, 3] == np.float32(0.8) * np.float32(0.8)  # a * a + 0 * (1 - a)


def test_render_rejects_bad_parameters():
    from mog_solver_b200 import render as R

    lib = _lib().lib()
    pos, vel = _particles(4, 0)
    out = np.zeros((8, 8, 4), np.uint8)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    for field, value in [("width", 0), ("height", -3), ("width", 20000), ("world_size", 0.0),
                         ("point_mode", 2), ("format", 5), ("point_size", 0.5),
                         ("max_point_size", float("nan")), ("speed_scale", float("inf"))]:
        p = R.params(8, 8)
        setattr(p, field, value)
        assert lib.mog_render_host(ctypes.byref(p), ptr(pos), ptr(vel), 4, ptr(out)) == \
            _lib().MOG_ERR_ARG, field
    p = R.params(8, 8)
    p.m_view[3] = float("nan")
    assert lib.mog_render_host(ctypes.byref(p), ptr(pos), ptr(vel), 4, ptr(out)) == _lib().MOG_ERR_ARG
    assert lib.mog_render_host(ctypes.byref(R.params(8, 8)), None, None, 4, ptr(out)) == \
        _lib().MOG_ERR_ARG
    with pytest.raises(ValueError):
        R.params(8, 8, point_mode="sprite")


def test_params_default_is_the_reference_state():
    from mog_solver_b200 import render as R

    p = _lib().RenderParamsC()
    _lib().lib().mog_render_params_default(ctypes.byref(p))
    assert (p.width, p.height) == (2560, 1440)
    assert list(p.clear) == [np.float32(0.01), np.float32(0.01), np.float32(0.02), 0.0]
    assert (p.point_mode, p.point_size, p.speed_scale, p.format) == (0, 1.0, 0.0, 0)
    q = R.params()
    v, m = R.camera_matrices()
    assert np.array_equal(np.array(q.m_view, np.float32), v)
    assert np.array_equal(np.array(q.m_proj, np.float32), m)


def test_write_png_round_trip(tmp_path):
    from mog_solver_b200 import render as R

    pos, vel = _particles(500, 3)
    img = R.render_host(pos, vel, width=40, height=30, world_size=100.0)
    R.write_png(tmp_path / "f.png", img)
    data = (tmp_path / "f.png").read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    w, h, depth, colour = struct.unpack(">IIBB", data[16:26])
    assert (w, h, depth, colour) == (40, 30, 8, 6)
    idat_len = struct.unpack(">I", data[33:37])[0]
    raw = zlib.decompress(data[41:41 + idat_len])
    rows = np.frombuffer(raw, np.uint8).reshape(30, 1 + 40 * 4)
    assert (rows[:, 0] == 0).all()
    assert np.array_equal(rows[:, 1:].reshape(30, 40, 4), img)


def test_write_png_rejects_other_images(tmp_path):
    from mog_solver_b200 import render as R

    with pytest.raises(ValueError):
        R.write_png(tmp_path / "f.png", np.zeros((4, 4, 4), np.float32))
    with pytest.raises(ValueError):
        R.write_png(tmp_path / "f.png", np.zeros((4, 4, 3), np.uint8))
    with pytest.raises(ValueError):
        R.params(8, 8, fmt="rgb565")
