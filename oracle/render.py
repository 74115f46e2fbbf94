"""The reference's particle draw under OpenGL's point rules, in NumPy —
TEST INFRASTRUCTURE ONLY (the checker of the CUDA renderer and of its host
twin; never part of the product).

What is restated:

* the reference's vertex and fragment shaders (main.py:359-410): position
  to clip space through m_proj * m_view, the shader's point size
  800 / (w + 0.1), the speed colour ramp getCosmicColor, the round sprite
  alpha exp(-r * 3.5) * 0.8 with discard outside the unit disc;
* the GL 4.6 core rules the draw relies on (on_render, main.py:678-703):
  point clipping to the view volume, the viewport transform, the square of
  pixel centres a point covers, gl_PointCoord with its upper-left origin,
  and SRC_ALPHA / ONE_MINUS_SRC_ALPHA blending in primitive order, with an
  8-bit target rounding after every blend.

Arithmetic: every operation is a binary32 NumPy operation in the order the
shaders write it (matrix products as ((c0 x + c1 y) + c2 z) + c3 w); exp is
Cody and Waite's reduction by ln 2 (split as in the Cephes library) with a
degree-7 Taylor polynomial, which is within GLSL's error bound for exp.
Where GL leaves a choice to the implementation this file makes the one the
library documents: pixel centres on the square's low edges are inside,
those on its high edges are not; the size is clamped to [1, max size].

Parity pins: the shader arithmetic is checked against the reference's own
vertex and fragment shaders compiled as C++ (oracle/_ref; golden fixture
tests/golden/point_shaders.npz); the camera matrices against the bytes the
reference's on_render writes (tests/golden/camera.npz).  The GL rules are
restated from the specification and pinned by known-answer tests.
"""
from __future__ import annotations

import numpy as np

F = np.float32


def exp_rn(x):
    """e^x, binary32, by the method above (x clamped to [-87, 88])."""
    x = np.clip(np.asarray(x, F), F(-87.0), F(88.0))
    k = np.rint(x * F(1.44269504088896341))
    f = (x - k * F(0.693359375)) - k * F(-2.12194440e-4)
    p = F(1.0) / F(5040.0)
    for c in (F(1.0) / F(720.0), F(1.0) / F(120.0), F(1.0) / F(24.0), F(1.0) / F(6.0), F(0.5),
              F(1.0), F(1.0)):
        p = p * f + c
    scale = ((k.astype(np.int32) + 127).astype(np.uint32) << 23).view(F)
    return (p * scale).astype(F)


def mat_vec(M, x, y, z, w):
    """Column-major 4x4 M (16 floats) times (x, y, z, w), GLSL association."""
    M = np.asarray(M, F)
    return [((M[r] * x + M[4 + r] * y) + M[8 + r] * z) + M[12 + r] * w for r in range(4)]


def mat_mul(A, B):
    """A * B for column-major 4x4 matrices."""
    B = np.asarray(B, F)
    out = np.zeros(16, F)
    for c in range(4):
        out[4 * c:4 * c + 4] = mat_vec(A, B[4 * c], B[4 * c + 1], B[4 * c + 2], B[4 * c + 3])
    return out


def mix(x, y, a):
    return x * (F(1.0) - a) + y * a


def cosmic_colour(t):
    """getCosmicColor (main.py:392-405) for an array of t in [0, 1]."""
    t = np.asarray(t, F)
    ramps = [((0.05, 0.1, 0.4), (0.6, 0.0, 0.7), t / F(0.3)),
             ((0.6, 0.0, 0.7), (1.0, 0.4, 0.0), (t - F(0.3)) / F(0.4)),
             ((1.0, 0.4, 0.0), (1.0, 0.9, 0.7), (t - F(0.7)) / F(0.3))]
    seg = np.where(t < F(0.3), 0, np.where(t < F(0.7), 1, 2))
    out = np.zeros(t.shape + (3,), F)
    for s, (lo, hi, a) in enumerate(ramps):
        for ch in range(3):
            v = mix(F(lo[ch]), F(hi[ch]), a)
            out[..., ch] = np.where(seg == s, v, out[..., ch])
    return out


def vertex_stage(pos, vel, m_view, m_proj, world, speed_scale):
    """The vertex shader: clip position (n, 4), the shader's point size,
    v_speed."""
    pos = np.asarray(pos, F)
    vel = np.asarray(vel, F)
    M = mat_mul(m_proj, m_view)
    p = [(pos[:, i] / F(world)) * F(2.0) - F(1.0) for i in range(3)]
    clip = np.stack(mat_vec(M, p[0], p[1], p[2], F(1.0)), axis=1).astype(F)
    size = F(800.0) / (clip[:, 3] + F(0.1))
    speed = np.sqrt((vel[:, 0] * vel[:, 0] + vel[:, 1] * vel[:, 1]) + vel[:, 2] * vel[:, 2])
    v_speed = np.clip(np.sqrt(speed) * F(speed_scale), F(0.0), F(1.0))
    return clip, size.astype(F), v_speed.astype(F)


def fragment_stage(point_coord, v_speed):
    """The fragment shader for gl_PointCoord (m, 2): (rgba (m, 4), kept)."""
    pc = np.asarray(point_coord, F)
    u = pc[:, 0] * F(2.0) - F(1.0)
    v = pc[:, 1] * F(2.0) - F(1.0)
    r = u * u + v * v
    rgba = np.zeros((pc.shape[0], 4), F)
    rgba[:, :3] = cosmic_colour(v_speed)
    rgba[:, 3] = exp_rn(-r * F(3.5)) * F(0.8)
    return rgba, ~(r > F(1.0))


def render(pos, vel, *, width, height, world_size, speed_scale, m_view, m_proj,
           clear=(0.01, 0.01, 0.02, 0.0), point_mode="fixed", point_size=1.0,
           max_point_size=2047.0, fmt="rgba8"):
    """The frame: (height, width, 4), top row first; uint8 codes for rgba8,
    float32 for rgba32f."""
    W, H = int(width), int(height)
    clip, shader_size, v_speed = vertex_stage(pos, vel, m_view, m_proj, world_size, speed_scale)
    x, y, z, w = (clip[:, i] for i in range(4))
    keep = (w > 0) & (x >= -w) & (x <= w) & (y >= -w) & (y <= w) & (z >= -w) & (z <= w)
    size = shader_size if point_mode == "program" else np.full(len(w), F(point_size), F)
    size = np.minimum(np.maximum(size, F(1.0)), F(max_point_size))
    hw, hh = F(W) * F(0.5), F(H) * F(0.5)
    with np.errstate(all="ignore"):
        xw = (x / w) * hw + hw
        yw = (y / w) * hh + hh
    rgba8 = fmt == "rgba8"

    def to8(c):
        return np.rint(np.clip(np.asarray(c, F), F(0.0), F(1.0)) * F(255.0)).astype(F)

    fb = np.empty((H, W, 4), F)  # rows from the bottom, as GL numbers them
    fb[...] = to8(np.array(clear, F)) if rgba8 else np.array(clear, F)
    colour = cosmic_colour(v_speed)
    for q in np.nonzero(keep)[0]:
        s, cx, cy = size[q], xw[q], yw[q]
        h = s * F(0.5)
        lo_x, hi_x, lo_y, hi_y = cx - h, cx + h, cy - h, cy + h
        i0, i1 = max(int(np.floor(lo_x)) - 1, 0), min(int(np.floor(hi_x)) + 1, W - 1)
        j0, j1 = max(int(np.floor(lo_y)) - 1, 0), min(int(np.floor(hi_y)) + 1, H - 1)
        if i0 > i1 or j0 > j1:
            continue
        xc = np.arange(i0, i1 + 1).astype(F) + F(0.5)
        yc = np.arange(j0, j1 + 1).astype(F) + F(0.5)
        X, Y = np.meshgrid(xc, yc)
        inside = (X >= lo_x) & (X < hi_x) & (Y >= lo_y) & (Y < hi_y)
        ps = F(0.5) + (X - cx) / s
        pt = F(0.5) - (Y - cy) / s
        u = ps * F(2.0) - F(1.0)
        v = pt * F(2.0) - F(1.0)
        r = u * u + v * v
        hit = inside & ~(r > F(1.0))
        if not hit.any():
            continue
        a = exp_rn(-r[hit] * F(3.5)) * F(0.8)
        jj, ii = np.nonzero(hit)
        jj, ii = jj + j0, ii + i0
        src = [colour[q, 0], colour[q, 1], colour[q, 2], a]
        for ch in range(4):
            d = fb[jj, ii, ch]
            if rgba8:
                d = d / F(255.0)
            out = src[ch] * a + d * (F(1.0) - a)
            fb[jj, ii, ch] = to8(out) if rgba8 else out
    img = fb[::-1]
    return img.astype(np.uint8) if rgba8 else np.ascontiguousarray(img)
