"""Oracle for the MOG force-and-step path — TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; it is the checker of the CUDA path, never part
of it.  Contents:

* ``liboracle()``      C restatement of the deposit / update shaders
                       (mog_oracle.c, built with -ffp-contract=off): the
                       bit-exact gate for mass grids and particle updates;
* ``pipeline``         NumPy FP64 "ideal pipeline" (same transforms, NGP and
                       Green's function, exact FFT): the 1e-5 force gate;
                       NumPy FP32 transcription of the reference's shader
                       chain with its flush quirks; FP64 direct-sum yardstick;
* ``mlp``              NumPy FP64 forward/backward of the learned correction;
* ``render``           NumPy restatement of the reference's particle draw
                       under OpenGL's point rules (the renderer's checker);
* ``_ref``             (built in the source container only) the reference's
                       own GLSL compute shaders, and the vertex and fragment
                       shaders of its particle draw, compiled as C++ through
                       a GLSL compatibility header, used to pin the above.

Parity anchors: the transforms come from the reference's own
``RandomSE3Sampler`` (golden fixtures in tests/golden, generated by
importing the reference), and the shader outputs on small cases come from
``_ref`` (same fixtures).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libmogoracle.so"
SRC = HERE / "mog_oracle.c"
CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-std=c11"]


def build_oracle(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        subprocess.run(["gcc", *CFLAGS, "-o", str(tmp), str(SRC), "-lm"], check=True)
        tmp.replace(LIB)
    return LIB


_lib = None


def liboracle() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build_oracle()
        lib = ctypes.CDLL(str(LIB))
        P = ctypes.c_void_p
        I = ctypes.c_int
        F = ctypes.c_float
        I64 = ctypes.c_int64
        lib.oracle_fast_rows.argtypes = [P, P, I, F, I, P]
        lib.oracle_fast_rows.restype = None
        lib.oracle_cells.argtypes = [P, I64, P, P, I, I, F, I, P]
        lib.oracle_cells.restype = None
        lib.oracle_deposit.argtypes = [P, I64, P, P, I, I, F, I, I, I, P]
        lib.oracle_deposit.restype = I
        lib.oracle_update.argtypes = [P, P, I64, P, P, P, I, I, F, I, F, F, P]
        lib.oracle_update.restype = I
        lib.oracle_mass_values.argtypes = [P, I64, I, I, P]
        lib.oracle_mass_values.restype = None
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


MASS_U64, MASS_U32 = 0, 1
INDEX_FAST, INDEX_EXACT = 0, 1


def fast_rows(rot12, off4, world: float, g: int) -> np.ndarray:
    rot12, off4 = _f32(rot12), _f32(off4)
    k = rot12.shape[0]
    out = np.empty((k, 12), dtype=np.float32)
    liboracle().oracle_fast_rows(_p(rot12), _p(off4), k, float(world), g, _p(out))
    return out


def cells(pos4, rot12, off4, g: int, world: float, index_mode: int = INDEX_FAST) -> np.ndarray:
    """(n, k) uint32 cell index (x fastest) of every particle in every grid."""
    pos4, rot12, off4 = _f32(pos4), _f32(rot12), _f32(off4)
    n, k = pos4.shape[0], rot12.shape[0]
    out = np.empty((n, k), dtype=np.uint32)
    liboracle().oracle_cells(_p(pos4), n, _p(rot12), _p(off4), k, g, float(world), index_mode,
                             _p(out))
    return out


def deposit(pos4, rot12, off4, g: int, world: float, mass_mode: int = MASS_U64,
            scale_bits: int = 32, index_mode: int = INDEX_FAST) -> np.ndarray:
    """(k, g, g, g) integer mass grid (uint64 or uint32)."""
    pos4, rot12, off4 = _f32(pos4), _f32(rot12), _f32(off4)
    k = rot12.shape[0]
    dt = np.uint64 if mass_mode == MASS_U64 else np.uint32
    out = np.empty((k, g, g, g), dtype=dt)
    rc = liboracle().oracle_deposit(_p(pos4), pos4.shape[0], _p(rot12), _p(off4), k, g,
                                    float(world), mass_mode, scale_bits, index_mode, _p(out))
    assert rc == 0
    return out


def update(pos4, vel4, force4, rot12, off4, g: int, world: float, dt: float, damping: float,
           index_mode: int = INDEX_FAST):
    """One update.glsl pass from a grid-frame force grid; returns (pos, vel)."""
    pos = _f32(pos4).copy()
    vel = _f32(vel4).copy()
    force4, rot12, off4 = _f32(force4), _f32(rot12), _f32(off4)
    k = rot12.shape[0]
    rc = liboracle().oracle_update(_p(pos), _p(vel), pos.shape[0], _p(force4), _p(rot12),
                                   _p(off4), k, g, float(world), index_mode, float(dt),
                                   float(damping), None)
    assert rc == 0
    return pos, vel


def averaged_force(pos4, force4, rot12, off4, g: int, world: float,
                   index_mode: int = INDEX_FAST) -> np.ndarray:
    """avgForce of update.glsl:81 at every particle, (n, 4) float32."""
    pos = _f32(pos4).copy()
    force4, rot12, off4 = _f32(force4), _f32(rot12), _f32(off4)
    k = rot12.shape[0]
    acc = np.empty_like(pos)
    rc = liboracle().oracle_update(_p(pos), None, pos.shape[0], _p(force4), _p(rot12), _p(off4),
                                   k, g, float(world), index_mode, 0.0, 1.0, _p(acc))
    assert rc == 0
    return acc


def mass_values(mass: np.ndarray, mass_mode: int, scale_bits: int) -> np.ndarray:
    """Cell values as float32, exactly as the solver reads them."""
    m = np.ascontiguousarray(mass)
    out = np.empty(m.shape, dtype=np.float32)
    liboracle().oracle_mass_values(_p(m), m.size, mass_mode, scale_bits, _p(out))
    return out
