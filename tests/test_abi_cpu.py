"""The C-ABI library loads and exports every entry point include/mog.h
declares; host-side validation works without a GPU (no compute calls)."""
import ctypes
import re
from pathlib import Path

import pytest

from mog_solver_b200 import _lib
from mog_solver_b200.build import build

ROOT = Path(__file__).resolve().parent.parent


def _declared_functions():
    text = (ROOT / "include" / "mog.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(mog_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build()
    return _lib.lib()


def test_header_and_binding_agree():
    assert _declared_functions() == sorted(_lib.EXPORTS)


def test_every_declared_symbol_is_exported(lib):
    for name in _declared_functions():
        assert hasattr(lib, name), name


def test_checked_library_exports_every_symbol():
    """libmog_check.so (the -DMOG_CHECK build) has the same C ABI."""
    checked = ctypes.CDLL(str(build(check=True)))
    for name in _declared_functions():
        assert hasattr(checked, name), name


def test_config_default_matches_reference_defaults(lib):
    c = _lib.default_config()
    # main.py:179-189 defaults, damping 1.0 (main.py:667)
    assert c.n_grids == 16 and c.grid_size == 16
    assert c.world_size == 100.0 and c.G == 1.0
    assert abs(c.dt - 1e-5) < 1e-12 and c.damping == 1.0
    assert c.solver == _lib.SOLVER_FFT


@pytest.mark.parametrize("field,value", [
    ("n_grids", 0), ("grid_size", 12), ("grid_size", 128), ("world_size", -1.0),
    ("solver", 7), ("mass_mode", 3), ("scale_bits", 101), ("index_mode", 2),
])
def test_create_rejects_bad_config_without_touching_the_gpu(lib, field, value):
    c = _lib.default_config()
    setattr(c, field, value)
    k = max(c.n_grids, 1)
    rot = (ctypes.c_float * (12 * k))()
    off = (ctypes.c_float * (4 * k))()
    h = ctypes.c_void_p()
    rc = lib.mog_create(ctypes.byref(c), rot, off, ctypes.byref(h))
    assert rc in (_lib.MOG_ERR_CONFIG, _lib.MOG_ERR_UNSUPPORTED)
    assert not h.value
    assert lib.mog_last_error().decode()


def test_create_rejects_nonfinite_transforms(lib):
    c = _lib.default_config()
    rot = (ctypes.c_float * (12 * c.n_grids))()
    rot[3] = float("nan")
    off = (ctypes.c_float * (4 * c.n_grids))()
    h = ctypes.c_void_p()
    assert lib.mog_create(ctypes.byref(c), rot, off, ctypes.byref(h)) == _lib.MOG_ERR_CONFIG


def test_null_arguments(lib):
    assert lib.mog_step(None, None, None, 0, 0.0, None) == _lib.MOG_ERR_ARG
    assert lib.mog_create(None, None, None, None) == _lib.MOG_ERR_ARG
    assert lib.mog_destroy(None) == _lib.MOG_OK


def test_strerror(lib):
    for code in range(8):
        assert lib.mog_strerror(code)
    assert b"sm_100a" in lib.mog_version()


@pytest.mark.parametrize("g,softening", [(8, 0.0), (16, 0.0), (16, 0.5), (32, 1.5)])
def test_green_table_matches_fp64(lib, g, softening):
    """mog_green_table (host): the solve's Green's factors, plain and with the
    reference's commented-out spectral softening, against the FP64 oracle."""
    import numpy as np

    from oracle import pipeline as pl

    out = np.empty(g ** 3, dtype=np.float32)
    assert lib.mog_green_table(g, 100.0, 3.0, softening, out.ctypes.data_as(ctypes.c_void_p)) == 0
    ref = pl.green_fp64(g, 100.0, 3.0, softening).ravel()
    assert np.array_equal(out == 0, ref == 0)
    nz = ref != 0
    assert np.abs(out[nz] / ref[nz] - 1).max() <= 1e-7


def test_green_table_rejects_bad_arguments(lib):
    import numpy as np

    out = np.empty(8, dtype=np.float32)
    assert lib.mog_green_table(3, 100.0, 1.0, 0.0, out.ctypes.data_as(ctypes.c_void_p)) == _lib.MOG_ERR_ARG
    assert lib.mog_green_table(2, 100.0, 1.0, -1.0, out.ctypes.data_as(ctypes.c_void_p)) == _lib.MOG_ERR_ARG


def test_config_softening_key():
    from mog_solver_b200.config import MogConfig

    base = {"grid_size": 16, "world_size": 100.0, "num_particles": 10, "G": 1.0, "dt": 1e-3}
    assert MogConfig.from_dict(base).softening == 0.0
    assert MogConfig.from_dict({**base, "softening": 0.5}).softening == 0.5
    with pytest.raises(ValueError):
        MogConfig.from_dict({**base, "softening": -1.0})
    with pytest.raises(ValueError):
        MogConfig.from_dict({**base, "softening": 0.5, "solver": "convolution"})
