"""Configuration surface: the reference's config.yaml keys and parse rules.

Mirrors ``Simulation.load_config`` (main.py:174-189) and the parameter parse
in ``Simulation.__init__`` (main.py:115-126):

* ``load_config(path)`` returns the YAML mapping when the file exists and
  otherwise the reference's in-code defaults (main.py:179-189);
* ``n_grids`` defaults to 16 (main.py:115), ``num_particles`` accepts strings
  such as ``"3e6"`` through ``int(float(...))`` (main.py:119), ``damping``
  defaults to 1.0 (main.py:667) and ``spawn_buffer`` to 0.1 (main.py:289);
* ``voxel_size = world_size / grid_size`` (main.py:118).

One deliberate difference: a config without a ``solver`` key runs the FFT
solver.  The reference parses a missing key as ``"convolution"``
(main.py:125) but its ``step()`` always runs the FFT chain (main.py:671-672),
so FFT is what such a config actually executed.

Keys this library adds: ``seed`` (transform sampler seed), ``mass_mode``
(``u64`` | ``u32x1000``), ``scale_bits`` (u64 fixed-point scale, ``None`` =
chosen from the total mass), ``index_mode`` (``fast`` | ``exact``),
``dft_precision`` (``fp32`` | ``bf16x3``), ``reference_texture_aliasing``
(reproduce the reference's x <- z force aliasing at g = 4, 16, 64; see
include/mog.h MOG_COMPAT_FFT_TEXTURE_ALIAS).
"""
from __future__ import annotations

import dataclasses
import math
from pathlib import Path
from typing import Any, Mapping

# main.py:179-189
REFERENCE_DEFAULTS: dict[str, Any] = {
    "n_grids": 16,
    "grid_size": 16,
    "world_size": 100.0,
    "num_particles": 100000,
    "G": 1.0,
    "dt": 0.00001,
    "particle_mass": 1.0,
    "solver": "fft",
    "record": True,
}


def load_config(path: str | Path | None = None) -> dict[str, Any]:
    """YAML mapping at ``path`` if it exists, else the reference defaults."""
    if path is not None:
        p = Path(path)
        if p.exists():
            import yaml

            with open(p) as f:
                data = yaml.safe_load(f)
            return dict(data or {})
    return dict(REFERENCE_DEFAULTS)


_SOLVERS = ("fft", "convolution")
_MASS_MODES = ("u64", "u32x1000")
_INDEX_MODES = ("fast", "exact")
_DFT = ("fp32", "bf16x3")


@dataclasses.dataclass
class MogConfig:
    n_grids: int = 16
    grid_size: int = 16
    world_size: float = 100.0
    num_particles: int = 100000
    G: float = 1.0
    dt: float = 0.00001
    damping: float = 1.0
    solver: str = "fft"
    particle_mass: float = 1.0
    spawn_buffer: float = 0.1
    seed: int | None = None
    mass_mode: str = "u64"
    scale_bits: int | None = None
    index_mode: str = "fast"
    dft_precision: str = "fp32"
    reference_texture_aliasing: bool = False
    softening: float = 0.0

    @property
    def voxel_size(self) -> float:
        return self.world_size / self.grid_size  # main.py:118

    @classmethod
    def from_dict(cls, cfg: Mapping[str, Any]) -> "MogConfig":
        """Parse a config mapping with the reference's rules (main.py:115-126)."""
        if "grid_size" not in cfg or "world_size" not in cfg or "num_particles" not in cfg:
            missing = [k for k in ("grid_size", "world_size", "num_particles") if k not in cfg]
            raise KeyError(f"config is missing required keys {missing} (main.py:116-119 index them)")
        if "G" not in cfg or "dt" not in cfg:
            missing = [k for k in ("G", "dt") if k not in cfg]
            raise KeyError(f"config is missing required keys {missing} (main.py:120-121 index them)")
        solver = cfg.get("solver", "fft")
        # The reference only tests solver == "convolution" (main.py:126);
        # every other value runs the FFT chain.
        solver = "convolution" if solver == "convolution" else "fft"
        out = cls(
            n_grids=int(cfg.get("n_grids", 16)),
            grid_size=int(cfg["grid_size"]),
            world_size=float(cfg["world_size"]),
            num_particles=int(float(cfg["num_particles"])),
            G=float(cfg["G"]),
            dt=float(cfg["dt"]),
            damping=float(cfg.get("damping", 1.0)),
            solver=solver,
            particle_mass=float(cfg.get("particle_mass", 1.0)),
            spawn_buffer=float(cfg.get("spawn_buffer", 0.1)),
            seed=None if cfg.get("seed") is None else int(cfg["seed"]),
            mass_mode=str(cfg.get("mass_mode", "u64")),
            scale_bits=None if cfg.get("scale_bits") is None else int(cfg["scale_bits"]),
            index_mode=str(cfg.get("index_mode", "fast")),
            dft_precision=str(cfg.get("dft_precision", "fp32")),
            reference_texture_aliasing=bool(cfg.get("reference_texture_aliasing", False)),
            softening=float(cfg.get("softening", 0.0)),
        )
        out.validate()
        return out

    def validate(self) -> None:
        g = self.grid_size
        if self.n_grids <= 0:
            raise ValueError("n_grids must be positive")
        if g < 2 or g > 64 or g & (g - 1):
            raise ValueError("grid_size must be a power of two in [2, 64] (the radix-2 FFT of fft_batched.glsl needs a power of two)")
        if not self.world_size > 0:
            raise ValueError("world_size must be positive")
        if self.num_particles < 0:
            raise ValueError("num_particles must be >= 0")
        if self.solver not in _SOLVERS:
            raise ValueError(f"solver must be one of {_SOLVERS}")
        if self.mass_mode not in _MASS_MODES:
            raise ValueError(f"mass_mode must be one of {_MASS_MODES}")
        if self.index_mode not in _INDEX_MODES:
            raise ValueError(f"index_mode must be one of {_INDEX_MODES}")
        if self.dft_precision not in _DFT:
            raise ValueError(f"dft_precision must be one of {_DFT}")
        if self.scale_bits is not None and not 0 <= self.scale_bits <= 100:
            raise ValueError("scale_bits must be in [0, 100]")
        if not (math.isfinite(self.softening) and self.softening >= 0):
            raise ValueError("softening must be finite and >= 0")
        if self.softening > 0 and self.solver != "fft":
            raise ValueError("softening applies to the fft solver only")

    def to_dict(self) -> dict[str, Any]:
        return dataclasses.asdict(self)
