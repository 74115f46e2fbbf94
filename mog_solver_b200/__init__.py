"""Mixture-of-Grids force-and-step path for NVIDIA B200 (sm_100a).

Python host layer over libmog.so (include/mog.h):

    from mog_solver_b200 import Simulation, load_config
    sim = Simulation(load_config("config.yaml"), seed=0)
    sim.init_particles("disks")
    sim.step()

The package mirrors the reference's operator surface (tbmo/mog-solver
main.py: ``load_config``, ``RandomSE3Sampler``, ``compute_transforms``,
``Simulation.step``); every force evaluation runs in hand-written CUDA.
"""
from ._lib import (MogError, MogLibraryError, FLAG_BADMASS, FLAG_BOUNDS, FLAG_NONFINITE,
                   FLAG_OVERFLOW, FLAG_TIMEOUT)
from .config import MogConfig, REFERENCE_DEFAULTS, load_config
from .transforms import RandomSE3Sampler, compute_transforms, rotation_matrices
from .simulation import Simulation, auto_scale_bits

__all__ = [
    "MogConfig", "MogError", "MogLibraryError", "REFERENCE_DEFAULTS", "RandomSE3Sampler",
    "Simulation", "auto_scale_bits", "compute_transforms", "load_config", "rotation_matrices",
    "FLAG_BADMASS", "FLAG_BOUNDS", "FLAG_NONFINITE", "FLAG_OVERFLOW", "FLAG_TIMEOUT",
]
__version__ = "0.1.0"
