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


def time_reference(w: dict, budget_s: float = 20.0, steps: int = 3, warmup: int = 0) -> dict:
    """Run ``warmup`` untimed steps, then time exactly ``steps`` steps, all on
    one particle sample sized (from a one-step probe) so that the
    ``warmup + steps`` steps take about ``budget_s`` seconds."""
    kind = "port"
    runner = _time_port
    try:
        from . import ref_harness

        if ref_harness.available():
            kind, runner = "reference", _time_ref
    except ImportError:
        pass
    steps = max(1, int(steps))
    warmup = max(0, int(warmup))
    sample_n = min(w["n"], 16384)
    tp, tg, cores = runner(w, sample_n, 1)
    per_particle = tp / sample_n
    room = budget_s / (steps + warmup) - tg
    if room > 0 and per_particle > 0:
        sample_n = int(min(w["n"], max(4096, room / per_particle)))
    if warmup:
        runner(w, sample_n, warmup)
    t0 = time.perf_counter()
    tp, tg, cores = runner(w, sample_n, steps)
    timed_s = time.perf_counter() - t0
    t_step = tg + tp * (w["n"] / sample_n)
    return {
        "value": w["n"] / t_step,
        "ms_per_step": t_step * 1e3,
        "cores": cores,
        "kind": kind,
        "sample_n": sample_n,
        "steps_timed": steps,
        "warmup_run": warmup,
        "timed_seconds": timed_s,
        "sample": (f"{steps} timed steps (after {warmup} untimed) on {sample_n} of {w['n']} "
                   f"particles of the workload with all {w['k']} grids of {w['g']}^3 cells, "
                   f"uint x1000 masses; time per step = grid time + particle time scaled by "
                   f"{w['n'] / sample_n:.1f}; host threads {cores} of {os.cpu_count()}"),
    }
