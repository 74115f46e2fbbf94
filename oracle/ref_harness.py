"""ctypes wrapper of oracle/_ref/libmogref.so — TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.

The library runs the reference's own compute shaders (compiled as C++ by
ref_build.py) with the dispatch order, bindings and texture ping-pong of
Simulation.step_fft (main.py:592-669).  It exists only where it was built
from a reference checkout; callers check ``available()``.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from .ref_build import LIB

_lib = None


def available() -> bool:
    return LIB.exists()


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        h = ctypes.CDLL(str(LIB))
        P, I, F = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        h.ref_threads.argtypes = [I]
        h.ref_threads.restype = I
        h.ref_deposit.argtypes = [P, I, P, P, I, I, F, F, P]
        h.ref_deposit.restype = None
        h.ref_solve.argtypes = [P, I, I, F, F, P]
        h.ref_solve.restype = None
        h.ref_update.argtypes = [P, P, I, P, P, I, I, F, F, F, F, P]
        h.ref_update.restype = None
        h.ref_step.argtypes = [P, P, I, P, P, I, I, F, F, F, F, F, P]
        U = ctypes.c_uint32
        h.ref_init_particles.argtypes = [P, P, I, F, F, F, U, F, F, U]
        h.ref_step.restype = None
        h.ref_point_vertex.argtypes = [P, P, I, F, F, P, P, P]
        h.ref_point_vertex.restype = None
        h.ref_point_fragment.argtypes = [P, P, I, P]
        h.ref_point_fragment.restype = None
        _lib = h
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def voxel(world: float, g: int) -> float:
    return float(np.float32(world / g))  # main.py:118, passed as a float uniform


def threads(n: int = 0) -> int:
    return lib().ref_threads(n)


def deposit(pos4, off4, rot12, g: int, world: float) -> np.ndarray:
    pos = _f32(pos4).copy()
    off, rot = _f32(off4), _f32(rot12)
    k = off.shape[0]
    out = np.zeros((k, g, g, g), dtype=np.uint32)
    lib().ref_deposit(_p(pos), pos.shape[0], _p(off), _p(rot), k, g, world, voxel(world, g),
                      _p(out))
    return out


def solve(mass_u32, world: float, G: float) -> np.ndarray:
    """Gradient texture (k, g, g, g, 4) = (fx, fy, fz, |f|) from a uint32 grid."""
    m = np.ascontiguousarray(mass_u32, dtype=np.uint32).copy()
    k, g = m.shape[0], m.shape[-1]
    out = np.empty((k, g, g, g, 4), dtype=np.float32)
    lib().ref_solve(_p(m), k, g, world, G, _p(out))
    return out


def update(pos4, vel4, off4, rot12, grad, g: int, world: float, dt: float, damping: float):
    pos, vel = _f32(pos4).copy(), _f32(vel4).copy()
    off, rot, grad = _f32(off4), _f32(rot12), _f32(grad)
    k = off.shape[0]
    lib().ref_update(_p(pos), _p(vel), pos.shape[0], _p(off), _p(rot), k, g, world,
                     voxel(world, g), dt, damping, _p(grad))
    return pos, vel


def step(pos4, vel4, off4, rot12, g: int, world: float, G: float, dt: float, damping: float):
    """One step_fft; returns (pos, vel, mass grid)."""
    pos, vel = _f32(pos4).copy(), _f32(vel4).copy()
    off, rot = _f32(off4), _f32(rot12)
    k = off.shape[0]
    mass = np.zeros((k, g, g, g), dtype=np.uint32)
    lib().ref_step(_p(pos), _p(vel), pos.shape[0], _p(off), _p(rot), k, g, world,
                   voxel(world, g), G, dt, damping, _p(mass))
    return pos, vel, mass


def init_particles(n: int, world: float, noise_scale: float = 4.0, contrast: float = 2.0,
                   seed: int = 12345, mass: float = 1.0, spawn_buffer: float = 0.1,
                   shape: int = 1):
    """init_particles.glsl (DIM 3) as init_particles_gpu dispatches it; returns
    (pos, vel) float32 (n, 4)."""
    pos = np.zeros((n, 4), dtype=np.float32)
    vel = np.zeros((n, 4), dtype=np.float32)
    lib().ref_init_particles(_p(pos), _p(vel), n, float(world), float(noise_scale),
                             float(contrast), int(seed) & 0xFFFFFFFF, float(mass),
                             float(spawn_buffer), int(shape))
    return pos, vel


def point_vertex(pos4, vel4, world: float, speed_scale: float, m_view, m_proj):
    """The reference's particle vertex shader (main.py:360-383): (gl_Position
    (n, 4), gl_PointSize (n), v_speed (n))."""
    pos, vel = _f32(pos4), _f32(vel4)
    out = np.zeros((pos.shape[0], 6), dtype=np.float32)
    lib().ref_point_vertex(_p(pos), _p(vel), pos.shape[0], float(world), float(speed_scale),
                           _p(_f32(m_view)), _p(_f32(m_proj)), _p(out))
    return out[:, :4], out[:, 4], out[:, 5]


def point_fragment(point_coord, v_speed):
    """The reference's particle fragment shader (main.py:385-410): (fragColor
    (m, 4), kept (m) bool)."""
    pc, vs = _f32(point_coord), _f32(v_speed)
    out = np.zeros((vs.shape[0], 5), dtype=np.float32)
    lib().ref_point_fragment(_p(pc), _p(vs), vs.shape[0], _p(out))
    return out[:, :4], out[:, 4] > 0.5


def time_steps(pos4, vel4, off4, rot12, w: dict, steps: int):
    """(particle seconds per step, grid seconds per step, threads) on all cores."""
    nthr = threads(os.cpu_count() or 1)
    pos, vel = _f32(pos4).copy(), _f32(vel4).copy()
    off, rot = _f32(off4), _f32(rot12)
    k, g, L = off.shape[0], w["g"], w["L"]
    mass = np.zeros((k, g, g, g), dtype=np.uint32)
    grad = np.empty((k, g, g, g, 4), dtype=np.float32)
    h = lib()
    vx = voxel(L, g)
    t_part = t_grid = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        h.ref_deposit(_p(pos), pos.shape[0], _p(off), _p(rot), k, g, L, vx, _p(mass))
        t1 = time.perf_counter()
        h.ref_solve(_p(mass), k, g, L, w["G"], _p(grad))
        t2 = time.perf_counter()
        h.ref_update(_p(pos), _p(vel), pos.shape[0], _p(off), _p(rot), k, g, L, vx, w["dt"],
                     w["damping"], _p(grad))
        t3 = time.perf_counter()
        t_part += (t1 - t0) + (t3 - t2)
        t_grid += t2 - t1
    return t_part / steps, t_grid / steps, nthr
