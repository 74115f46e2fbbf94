"""Headless particle renderer: the reference's particle draw without a window.

The reference draws every particle as a GL point each frame (vertex and
fragment shaders at main.py:359-423, on_render at main.py:678-703).  This
module draws the same picture with CUDA kernels into a device tensor, under
OpenGL's rules for points (see ``csrc/render_math.cuh``), and can write it
to a PNG file:

    img = render(sim.pos, sim.vel, world_size=sim.cfg.world_size)   # (H, W, 4) uint8, CUDA
    write_png("frame.png", img)

``camera_matrices`` builds the two matrix uniforms exactly as on_render
does, from the orbit camera's angles and distance (main.py:135-137 and
685-697).  ``render_host`` is the same image computed on the host (no GPU).
"""
from __future__ import annotations

import ctypes
import struct
import zlib
from pathlib import Path

import numpy as np

from . import _lib

WINDOW_SIZE = (2560, 1440)  # main.py:104


def perspective(fovy: float, aspect: float, near: float, far: float) -> np.ndarray:
    """The projection on_render uses (main.py:70-80), as a float32 4x4
    array whose C-order bytes are the m_proj uniform."""
    f = 1.0 / np.tan(np.radians(fovy) / 2.0)
    rows = [[f / aspect, 0.0, 0.0, 0.0], [0.0, f, 0.0, 0.0],
            [0.0, 0.0, (far + near) / (near - far), -1.0],
            [0.0, 0.0, (2.0 * far * near) / (near - far), 0.0]]
    return np.array(rows, dtype=np.float32)


def look_at(eye: np.ndarray, target: np.ndarray, up: np.ndarray) -> np.ndarray:
    """The view matrix on_render uses (main.py:83-98): float32 throughout,
    returned transposed so that its C-order bytes are the m_view uniform."""
    fwd = eye - target
    fwd = fwd / np.linalg.norm(fwd)
    side = np.cross(up, fwd)
    side = side / np.linalg.norm(side)
    upv = np.cross(fwd, side)
    m = np.identity(4, dtype=np.float32)
    for r, axis in enumerate((side, upv, fwd)):
        m[r, :3] = axis
        m[r, 3] = -np.dot(axis, eye)
    return m.T


def camera_matrices(cam_rot_x: float = 0.0, cam_rot_y: float = 0.0, cam_dist: float = 3.0,
                    aspect: float = WINDOW_SIZE[0] / WINDOW_SIZE[1]):
    """(m_view, m_proj) as 16 float32 each, column-major: the uniform bytes
    on_render writes for an orbit camera (main.py:685-700; the reference
    starts at angles 0, 0 and distance 3, main.py:135-137)."""
    ax = np.radians(cam_rot_x)
    ay = np.radians(np.clip(cam_rot_y, -89, 89))
    eye = np.array([cam_dist * np.sin(ax) * np.cos(ay), cam_dist * np.sin(ay),
                    cam_dist * np.cos(ax) * np.cos(ay)], dtype=np.float32)
    view = look_at(eye, np.zeros(3, np.float32), np.array([0, 1, 0], np.float32))
    proj = perspective(45.0, aspect, 0.1, 100.0)
    return (np.frombuffer(view.tobytes(), np.float32).copy(),
            np.frombuffer(proj.tobytes(), np.float32).copy())


def params(width: int = WINDOW_SIZE[0], height: int = WINDOW_SIZE[1], *, world_size: float = 100.0,
           cam_rot_x: float = 0.0, cam_rot_y: float = 0.0, cam_dist: float = 3.0,
           speed_scale: float = 0.0, point_mode: str = "fixed", point_size: float = 1.0,
           max_point_size: float = 2047.0, fmt: str = "rgba8",
           clear=(0.01, 0.01, 0.02, 0.0), m_view=None, m_proj=None) -> _lib.RenderParamsC:
    """mog_render_params for one frame.  point_mode "fixed" draws every
    point point_size pixels wide (the reference's GL state: it never enables
    GL_PROGRAM_POINT_SIZE); "program" uses the shader's 800 / (w + 0.1)."""
    if point_mode not in ("fixed", "program"):
        raise ValueError("point_mode must be 'fixed' or 'program'")
    if fmt not in ("rgba8", "rgba32f"):
        raise ValueError("fmt must be 'rgba8' or 'rgba32f'")
    p = _lib.RenderParamsC()
    _lib.lib().mog_render_params_default(ctypes.byref(p))
    p.width, p.height = int(width), int(height)
    p.world_size = float(world_size)
    p.speed_scale = float(speed_scale)
    if m_view is None or m_proj is None:
        v, pr = camera_matrices(cam_rot_x, cam_rot_y, cam_dist, width / height)
        m_view = v if m_view is None else m_view
        m_proj = pr if m_proj is None else m_proj
    p.m_view[:] = [float(x) for x in np.asarray(m_view, np.float32).reshape(16)]
    p.m_proj[:] = [float(x) for x in np.asarray(m_proj, np.float32).reshape(16)]
    p.clear[:] = [float(x) for x in clear]
    p.point_mode = 0 if point_mode == "fixed" else 1
    p.point_size = float(point_size)
    p.max_point_size = float(max_point_size)
    p.format = _lib.RENDER_RGBA8 if fmt == "rgba8" else _lib.RENDER_RGBA32F
    return p


class Renderer:
    """Owns the renderer's device scratch (mog_renderer_create)."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().mog_renderer_create(ctypes.byref(self._h)), "mog_renderer_create")

    def close(self) -> None:
        if self._h:
            _lib.lib().mog_renderer_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def render(self, pos, vel, p: _lib.RenderParamsC | None = None, out=None, **kw):
        """Image (height, width, 4) on the particles' device, top row first:
        uint8 for rgba8, float32 for rgba32f."""
        import torch

        p = params(**kw) if p is None else p
        if pos.shape != vel.shape or pos.dim() != 2 or pos.shape[1] != 4:
            raise ValueError("pos and vel must both be (N, 4)")
        if not (pos.is_cuda and vel.is_cuda and pos.dtype == torch.float32 and
                vel.dtype == torch.float32):
            raise ValueError("pos and vel must be float32 CUDA tensors")
        pos, vel = pos.contiguous(), vel.contiguous()
        dtype = torch.uint8 if p.format == _lib.RENDER_RGBA8 else torch.float32
        if out is None:
            out = torch.empty((p.height, p.width, 4), dtype=dtype, device=pos.device)
        elif out.shape != (p.height, p.width, 4) or out.dtype != dtype or not out.is_contiguous():
            raise ValueError("out must be a contiguous (height, width, 4) tensor of the format's type")
        with torch.cuda.device(pos.device):
            stream = ctypes.c_void_p(torch.cuda.current_stream(pos.device).cuda_stream)
            _lib.check(_lib.lib().mog_render(self._h, ctypes.byref(p), pos.data_ptr(),
                                             vel.data_ptr(), int(pos.shape[0]), out.data_ptr(),
                                             stream), "mog_render")
        return out

    def stats(self) -> dict:
        """The last frame's (point, tile) pair count and kernel launches."""
        pairs, launches = ctypes.c_int64(), ctypes.c_int32()
        _lib.check(_lib.lib().mog_renderer_stats(self._h, ctypes.byref(pairs),
                                                 ctypes.byref(launches)), "mog_renderer_stats")
        return {"pairs": pairs.value, "launches": launches.value}


_renderers: dict[int, Renderer] = {}


def render(pos, vel, **kw):
    """One frame of device particles with a Renderer shared per device (see
    params for the keywords)."""
    import torch

    dev = pos.device.index if pos.device.index is not None else torch.cuda.current_device()
    if dev not in _renderers:
        with torch.cuda.device(dev):
            _renderers[dev] = Renderer()
    return _renderers[dev].render(pos, vel, **kw)


def render_host(pos: np.ndarray, vel: np.ndarray, p: _lib.RenderParamsC | None = None, **kw):
    """The same image from host arrays, computed on the host."""
    p = params(**kw) if p is None else p
    pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 4)
    vel = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 4)
    if pos.shape != vel.shape:
        raise ValueError("pos and vel must have the same shape")
    dtype = np.uint8 if p.format == _lib.RENDER_RGBA8 else np.float32
    out = np.empty((p.height, p.width, 4), dtype=dtype)
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a.size else None
    _lib.check(_lib.lib().mog_render_host(ctypes.byref(p), ptr(pos), ptr(vel), pos.shape[0],
                                          out.ctypes.data_as(ctypes.c_void_p)), "mog_render_host")
    return out


def write_png(path: str | Path, image) -> None:
    """An (H, W, 4) uint8 image (numpy or torch, top row first) as an RGBA PNG."""
    img = image.cpu().numpy() if hasattr(image, "cpu") else np.asarray(image)
    if img.dtype != np.uint8 or img.ndim != 3 or img.shape[2] != 4:
        raise ValueError("write_png takes an (H, W, 4) uint8 image")
    h, w = img.shape[:2]
    raw = b"".join(b"\x00" + img[r].tobytes() for r in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return (struct.pack(">I", len(data)) + tag + data +
                struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF))

    png = (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)) +
           chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b""))
    Path(path).write_bytes(png)
