"""ctypes bindings for libmog.so (the C ABI declared in include/mog.h).

The library is loaded from this package directory.  There is no fallback:
if it is missing or fails to load, every call raises ``MogLibraryError``.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libmog.so"

# status codes (include/mog.h)
MOG_OK = 0
MOG_ERR_CONFIG = 1
MOG_ERR_CUDA = 2
MOG_ERR_OVERFLOW = 3
MOG_ERR_NONFINITE = 4
MOG_ERR_TIMEOUT = 5
MOG_ERR_ARG = 6
MOG_ERR_UNSUPPORTED = 7

SOLVER_FFT = 0
SOLVER_CONVOLUTION = 1
MASS_U64_FIXED = 0
MASS_U32_X1000 = 1
INDEX_FAST = 0
INDEX_EXACT = 1
DFT_FFT32 = 0
DFT_TC_BF16X3 = 1

COMPAT_FFT_TEXTURE_ALIAS = 1

MODEL_PARAMS = 5187
MODEL_NORM = 28

FLAG_NONFINITE = 1
FLAG_OVERFLOW = 2
FLAG_TIMEOUT = 4
FLAG_BADMASS = 8
FLAG_BOUNDS = 16  # only from a library built with --check

# Every symbol include/mog.h declares.
EXPORTS = (
    "mog_config_default", "mog_create", "mog_destroy", "mog_step", "mog_step_n",
    "mog_step_profiled", "mog_forces", "mog_deposit", "mog_solve", "mog_update", "mog_get_status",
    "mog_selftest_wait_timeout", "mog_shard_init", "mog_shard_export", "mog_shard_connect",
    "mog_shard_connect_local", "mog_shard_deposit", "mog_shard_exchange", "mog_shard_finish",
    "mog_shard_step",
    "mog_get_tuning", "mog_set_tuning", "mog_diagnostics", "mog_direct_sum",
    "mog_direct_sum_noalloc", "mog_green_table", "mog_init_particles", "mog_init_particles_host",
    "mog_init_two_galaxies", "mog_init_two_galaxies_host",
    "mog_batch_create", "mog_batch_step", "mog_batch_destroy", "mog_batch_set_tuning",
    "mog_batch_get_tuning",
    "mog_model_create", "mog_model_destroy", "mog_model_set", "mog_model_get",
    "mog_model_train_step", "mog_features", "mog_learned_forces", "mog_learned_step",
    "mog_learned_step_profiled", "mog_learned_spread", "mog_step_host", "mog_learned_step_host",
    "mog_render_params_default", "mog_renderer_create", "mog_renderer_destroy", "mog_render",
    "mog_renderer_stats", "mog_render_host",
    "mog_strerror", "mog_last_error", "mog_version",
)


class MogLibraryError(RuntimeError):
    """libmog.so is missing or could not be loaded."""


class MogError(RuntimeError):
    """A libmog call returned a non-zero status."""

    def __init__(self, code: int, where: str, detail: str):
        self.code = code
        super().__init__(f"{where}: {detail} (status {code})")


class MogConfigC(ctypes.Structure):
    _fields_ = [
        ("n_grids", ctypes.c_int32),
        ("grid_size", ctypes.c_int32),
        ("world_size", ctypes.c_float),
        ("G", ctypes.c_float),
        ("dt", ctypes.c_float),
        ("damping", ctypes.c_float),
        ("solver", ctypes.c_int32),
        ("mass_mode", ctypes.c_int32),
        ("scale_bits", ctypes.c_int32),
        ("index_mode", ctypes.c_int32),
        ("dft_prec", ctypes.c_int32),
        ("compat_flags", ctypes.c_int32),
        ("num_particles", ctypes.c_int64),
        ("softening", ctypes.c_float),
    ]


class MogTuningC(ctypes.Structure):
    _fields_ = [
        ("deposit_threads", ctypes.c_int32),
        ("deposit_grids_per_cta", ctypes.c_int32),
        ("deposit_chunks", ctypes.c_int32),
        ("deposit_ppt", ctypes.c_int32),
        ("update_staged", ctypes.c_int32),
        ("update_ctas", ctypes.c_int32),
        ("sort_every", ctypes.c_int32),
        ("update_direct_ppt", ctypes.c_int32),
        ("deposit_aggregate", ctypes.c_int32),
        ("deposit_generic", ctypes.c_int32),
        ("deposit_sorted", ctypes.c_int32),
        ("update_threads", ctypes.c_int32),
        ("deposit_split", ctypes.c_int32),
        ("learned_fold", ctypes.c_int32),
        ("learned_ctas_per_sm", ctypes.c_int32),
        ("solve_split", ctypes.c_int32),
    ]


class MogBatchTuningC(ctypes.Structure):
    """mog_batch_tuning (include/mog.h)."""

    _fields_ = [
        ("work_queue", ctypes.c_int32),
        ("deposit_chunk", ctypes.c_int32),
        ("active_work_queue", ctypes.c_int32),
        ("deposit_split", ctypes.c_int32),
    ]


RENDER_RGBA8 = 0
RENDER_RGBA32F = 1


class RenderParamsC(ctypes.Structure):
    """mog_render_params (include/mog.h)."""

    _fields_ = [
        ("width", ctypes.c_int32),
        ("height", ctypes.c_int32),
        ("world_size", ctypes.c_float),
        ("speed_scale", ctypes.c_float),
        ("m_view", ctypes.c_float * 16),
        ("m_proj", ctypes.c_float * 16),
        ("clear", ctypes.c_float * 4),
        ("point_mode", ctypes.c_int32),
        ("point_size", ctypes.c_float),
        ("max_point_size", ctypes.c_float),
        ("format", ctypes.c_int32),
    ]


_lib = None


def _declare(lib: ctypes.CDLL) -> None:
    P = ctypes.c_void_p
    I64 = ctypes.c_int64
    F = ctypes.c_float
    I = ctypes.c_int
    lib.mog_config_default.argtypes = [ctypes.POINTER(MogConfigC)]
    lib.mog_create.argtypes = [ctypes.POINTER(MogConfigC), P, P, ctypes.POINTER(P)]
    lib.mog_destroy.argtypes = [P]
    lib.mog_step.argtypes = [P, P, P, I64, F, P]
    lib.mog_step_n.argtypes = [P, P, P, I64, F, ctypes.c_int32, P]
    lib.mog_step_profiled.argtypes = [P, P, P, I64, F, ctypes.POINTER(ctypes.c_float), P]
    lib.mog_forces.argtypes = [P, P, P, I64, P]
    lib.mog_deposit.argtypes = [P, P, I64, P, P]
    lib.mog_solve.argtypes = [P, P, P, P]
    lib.mog_update.argtypes = [P, P, P, I64, P, F, P]
    lib.mog_get_tuning.argtypes = [P, ctypes.POINTER(MogTuningC)]
    lib.mog_set_tuning.argtypes = [P, ctypes.POINTER(MogTuningC)]
    lib.mog_get_status.argtypes = [P, ctypes.POINTER(ctypes.c_uint32), P]
    lib.mog_selftest_wait_timeout.argtypes = [P, P]
    lib.mog_shard_init.argtypes = [P, ctypes.c_int32, ctypes.c_int32]
    lib.mog_shard_export.argtypes = [P, P, P]
    lib.mog_shard_connect.argtypes = [P, P, P]
    lib.mog_shard_connect_local.argtypes = [P, ctypes.POINTER(P)]
    lib.mog_shard_deposit.argtypes = [P, P, I64, P]
    lib.mog_shard_exchange.argtypes = [P, P]
    lib.mog_shard_finish.argtypes = [P, P, P, I64, F, P]
    lib.mog_shard_step.argtypes = [P, P, P, I64, F, P]
    lib.mog_diagnostics.argtypes = [P, P, P, I64, ctypes.POINTER(ctypes.c_double), P]
    D = ctypes.c_double
    lib.mog_direct_sum.argtypes = [P, I64, P, I64, D, D, D, P, P]
    lib.mog_direct_sum_noalloc.argtypes = [P, I64, P, I64, D, D, D, P, P]
    lib.mog_green_table.argtypes = [ctypes.c_int32, F, F, F, P]
    U32 = ctypes.c_uint32
    lib.mog_init_particles.argtypes = [P, P, I64, F, F, F, U32, F, F, ctypes.c_int32, P]
    lib.mog_init_particles_host.argtypes = [P, P, I64, F, F, F, U32, F, F, ctypes.c_int32]
    lib.mog_init_two_galaxies.argtypes = [P, P, I64, F, F, ctypes.c_uint64, P]
    lib.mog_init_two_galaxies_host.argtypes = [P, P, I64, F, F, ctypes.c_uint64]
    FP = ctypes.POINTER(ctypes.c_float)
    lib.mog_batch_create.argtypes = [P, ctypes.c_int32, ctypes.POINTER(P)]
    lib.mog_batch_step.argtypes = [P, P, P, P, P, ctypes.c_int32, P]
    lib.mog_batch_destroy.argtypes = [P]
    lib.mog_batch_set_tuning.argtypes = [P, ctypes.POINTER(MogBatchTuningC)]
    lib.mog_batch_get_tuning.argtypes = [P, ctypes.POINTER(MogBatchTuningC)]
    lib.mog_model_create.argtypes = [ctypes.POINTER(P)]
    lib.mog_model_destroy.argtypes = [P]
    lib.mog_model_set.argtypes = [P, P, P]
    lib.mog_model_get.argtypes = [P, P, P]
    lib.mog_model_train_step.argtypes = [P, P, P, P, ctypes.c_int32, F, FP, P, P]
    lib.mog_features.argtypes = [P, P, P, I64, P, P, P]
    lib.mog_learned_forces.argtypes = [P, P, P, P, I64, P]
    lib.mog_learned_step.argtypes = [P, P, P, P, I64, F, P]
    lib.mog_learned_step_profiled.argtypes = [P, P, P, P, I64, F, ctypes.POINTER(ctypes.c_float), P]
    lib.mog_learned_spread.argtypes = [P, ctypes.POINTER(ctypes.c_double), P]
    lib.mog_step_host.argtypes = [P, P, P, I64, F, ctypes.c_int32, P]
    lib.mog_learned_step_host.argtypes = [P, P, P, P, I64, F, ctypes.c_int32, P]
    RP = ctypes.POINTER(RenderParamsC)
    lib.mog_render_params_default.argtypes = [RP]
    lib.mog_render_params_default.restype = None
    lib.mog_renderer_create.argtypes = [ctypes.POINTER(P)]
    lib.mog_renderer_destroy.argtypes = [P]
    lib.mog_render.argtypes = [P, RP, P, P, I64, P, P]
    lib.mog_render_host.argtypes = [RP, P, P, I64, P]
    lib.mog_renderer_stats.argtypes = [P, ctypes.POINTER(I64), ctypes.POINTER(ctypes.c_int32)]
    lib.mog_strerror.argtypes = [I]
    lib.mog_strerror.restype = ctypes.c_char_p
    lib.mog_last_error.argtypes = []
    lib.mog_last_error.restype = ctypes.c_char_p
    lib.mog_version.argtypes = []
    lib.mog_version.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name not in ("mog_strerror", "mog_last_error", "mog_version", "mog_render_params_default"):
            getattr(lib, name).restype = ctypes.c_int


def lib() -> ctypes.CDLL:
    """Load libmog.so (once).  Raises MogLibraryError if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("MOG_LIBRARY", LIB_PATH))
    if not path.exists():
        raise MogLibraryError(
            f"{path} is not built; run `python -m mog_solver_b200.build` (CUDA is required, "
            "there is no CPU fallback)")
    try:
        handle = ctypes.CDLL(str(path))
    except OSError as exc:  # pragma: no cover - depends on the environment
        raise MogLibraryError(f"cannot load {path}: {exc}") from exc
    _declare(handle)
    _lib = handle
    return handle


def check(code: int, where: str) -> None:
    if code != MOG_OK:
        detail = lib().mog_last_error().decode() or lib().mog_strerror(code).decode()
        raise MogError(code, where, detail)


def default_config() -> MogConfigC:
    c = MogConfigC()
    check(lib().mog_config_default(ctypes.byref(c)), "mog_config_default")
    return c
