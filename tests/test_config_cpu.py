"""The configuration surface against the reference's own load_config
(fixture tests/golden/config.json, made by running it) and its parse rules
(main.py:115-126): keys, defaults, the int(float(...)) particle count, the
voxel size, and the values this library rejects before touching a GPU."""
import json
import math
from pathlib import Path

import pytest

from mog_solver_b200.config import REFERENCE_DEFAULTS, MogConfig, load_config

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "config.json").read_text())


def test_in_code_defaults_are_the_references():
    assert REFERENCE_DEFAULTS == GOLD["defaults"]
    assert load_config(None) == GOLD["defaults"]
    assert load_config("/nonexistent/config.yaml") == GOLD["defaults"]


def test_reference_config_file_parses_like_the_reference(tmp_path):
    """The reference's config.yaml through our loader and parser: YAML reads
    3e6 as a string, which int(float(...)) turns into 3,000,000 (main.py:119)."""
    import yaml

    p = tmp_path / "config.yaml"
    p.write_text(yaml.safe_dump(GOLD["config_yaml"]).replace("'3e6'", "3e6"))
    raw = load_config(p)
    assert raw == GOLD["config_yaml"]
    c = MogConfig.from_dict(raw)
    assert (c.n_grids, c.grid_size, c.world_size, c.num_particles) == (120, 16, 2000.0, 3_000_000)
    assert (c.G, c.dt, c.damping, c.solver) == (10.0, 1e-5, 0.998, "fft")
    assert (c.particle_mass, c.spawn_buffer) == (1.0, 0.25)
    assert c.voxel_size == 2000.0 / 16  # main.py:118


def test_defaults_parse():
    c = MogConfig.from_dict(load_config(None))
    assert (c.n_grids, c.grid_size, c.world_size, c.num_particles) == (16, 16, 100.0, 100000)
    assert (c.G, c.dt, c.solver) == (1.0, 1e-5, "fft")
    assert c.damping == 1.0  # main.py:667
    assert c.spawn_buffer == 0.1  # main.py:289
    assert c.mass_mode == "u64" and c.scale_bits is None and c.softening == 0.0


@pytest.mark.parametrize("value,expect", [("3e6", 3_000_000), ("1.5e3", 1500), (2.9, 2), (7, 7),
                                          ("100000", 100000)])
def test_particle_count_is_int_of_float(value, expect):
    base = dict(GOLD["defaults"], num_particles=value)
    assert MogConfig.from_dict(base).num_particles == expect


def test_n_grids_defaults_to_16_and_solver_to_fft():
    base = {k: v for k, v in GOLD["defaults"].items() if k not in ("n_grids", "solver")}
    c = MogConfig.from_dict(base)
    assert c.n_grids == 16  # main.py:115
    # the reference parses a missing key as "convolution" but its step runs
    # the FFT chain (main.py:125, 671-672); here the config runs what it ran
    assert c.solver == "fft"
    assert MogConfig.from_dict(dict(base, solver="convolution")).solver == "convolution"
    assert MogConfig.from_dict(dict(base, solver="spectral")).solver == "fft"  # only "convolution" counts


@pytest.mark.parametrize("key", ["grid_size", "world_size", "num_particles", "G", "dt"])
def test_keys_the_reference_indexes_are_required(key):
    base = {k: v for k, v in GOLD["defaults"].items() if k != key}
    with pytest.raises(KeyError):
        MogConfig.from_dict(base)


@pytest.mark.parametrize("field,value", [("grid_size", 12), ("grid_size", 128), ("grid_size", 1),
                                         ("n_grids", 0), ("world_size", -1.0),
                                         ("num_particles", -5), ("mass_mode", "f32"),
                                         ("index_mode", "rounded"), ("dft_precision", "fp8"),
                                         ("scale_bits", 101), ("softening", -0.5),
                                         ("softening", math.inf)])
def test_invalid_values_are_rejected(field, value):
    with pytest.raises(ValueError):
        MogConfig.from_dict(dict(GOLD["defaults"], **{field: value}))


def test_softening_needs_the_fft_solver():
    with pytest.raises(ValueError):
        MogConfig.from_dict(dict(GOLD["defaults"], solver="convolution", softening=0.5))


def test_round_trip_through_a_checkpoint_header():
    c = MogConfig.from_dict(dict(GOLD["defaults"], seed=4, mass_mode="u32x1000", softening=0.5))
    assert MogConfig(**json.loads(json.dumps(c.to_dict()))) == c
