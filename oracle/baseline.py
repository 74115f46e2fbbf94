"""Timed CPU baseline of the reference's path — TEST/BENCH INFRASTRUCTURE ONLY.

Used by bench.py's CPU-baseline leg and ``--impl reference``.  Two kinds:

* ``reference``: the reference's own GLSL compute shaders compiled as C++
  (oracle/_ref, built from the sources in the reference checkout by
  oracle/ref_build.py), run by the harness with OpenMP over all host threads;
* ``port``: the C restatement (deposit and update, mog_oracle.c) plus the
  NumPy FP32 transcription of the spectral shader chain, one thread.

Both run the reference's arithmetic (uint x1000 masses, exact op order)
on a bounded sample: the full k grids of g^3 cells, and the first
``sample_n`` particles of the workload.  The per-step time of the full
workload is extrapolated as t_grid + t_particles(sample) * N / sample_n.
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import pipeline as pl


def _workload_particles(w: dict, n: int):
    from mog_solver_b200 import ics
    from mog_solver_b200.transforms import compute_transforms

    off, rot = compute_transforms(w["k"], w["g"], w["L"], seed=0)
    if w["ic"] == "disks":
        h = w["L"] / w["g"]
        pos, vel = ics.two_disks(w["n"], w["L"], seed=w["seed"], g_eff=w["G"] * h ** 3 / 2)
    else:
        pos, vel = ics.uniform_cube(w["n"], w["L"], seed=w["seed"])
    idx = np.random.default_rng(7).choice(w["n"], size=min(n, w["n"]), replace=False)
    pos = pos[idx].copy()
    vel = vel[idx].copy()
    pos[:, 3] = 1.0  # the reference's particle_mass (config.yaml:8)
    return pos, vel, off, rot


def _time_port(w: dict, sample_n: int, steps: int):
    import oracle

    pos, vel, off, rot = _workload_particles(w, sample_n)
    g, L = w["g"], w["L"]
    t_part = t_grid = 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        mass = oracle.deposit(pos, rot, off, g, L, oracle.MASS_U32, 0, oracle.INDEX_EXACT)
        t1 = time.perf_counter()
        F = pl.forces_grid_f32(mass, w["G"], L)
        t2 = time.perf_counter()
        pos, vel = oracle.update(pos, vel, F, rot, off, g, L, w["dt"], w["damping"],
                                 oracle.INDEX_EXACT)
        t3 = time.perf_counter()
        t_part += (t1 - t0) + (t3 - t2)
        t_grid += t2 - t1
    return t_part / steps, t_grid / steps, 1


def _time_ref(w: dict, sample_n: int, steps: int):
    from . import ref_harness

    pos, vel, off, rot = _workload_particles(w, sample_n)
    return ref_harness.time_steps(pos, vel, off, rot, w, steps)


def time_reference(w: dict, budget_s: float = 20.0, steps: int | None = None) -> dict:
    kind = "port"
    runner = _time_port
    try:
        from . import ref_harness

        if ref_harness.available():
            kind, runner = "reference", _time_ref
    except ImportError:
        pass
    sample_n = min(w["n"], 16384)
    # one probe step to size the sample within the budget
    tp, tg, cores = runner(w, sample_n, 1)
    n_steps = steps if steps else 3
    per_particle = tp / sample_n
    room = budget_s / max(n_steps, 1) - tg
    if room > 0 and per_particle > 0:
        sample_n = int(min(w["n"], max(4096, room / per_particle)))
    tp, tg, cores = runner(w, sample_n, max(1, min(n_steps, 3)))
    t_step = tg + tp * (w["n"] / sample_n)
    return {
        "value": w["n"] / t_step,
        "ms_per_step": t_step * 1e3,
        "cores": cores,
        "kind": kind,
        "sample_n": sample_n,
        "sample": (f"{sample_n} of {w['n']} particles of the workload with all {w['k']} grids of "
                   f"{w['g']}^3 cells, uint x1000 masses; time per step = grid time + particle "
                   f"time scaled by {w['n'] / sample_n:.1f}; host threads {cores} "
                   f"of {os.cpu_count()}"),
    }
