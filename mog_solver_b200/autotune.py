"""Autotuner for the launch shapes of a Simulation (no counterpart in the
reference, whose dispatch shapes are fixed in main.py:596-668).

The knobs of ``mog_tuning`` (include/mog.h) never change a result — every
variant is bit-identical (tests/test_gpu_parity.py checks that) — only its
speed.  ``autotune(sim)`` measures candidate shapes with
``mog_step_profiled`` (per-kernel device times), one knob group at a time
(coordinate search: deposit shape, gather variant, spatial ordering), keeps
the fastest, restores the particles it advanced, and caches the choice in
a JSON file keyed by device, particle-count bucket, k, g and modes.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import math
import os
from pathlib import Path

import numpy as np

from . import _lib
from .simulation import Simulation, torch_device

CACHE = Path(os.environ.get("MOG_TUNING_CACHE", Path(__file__).resolve().parent / "tuning_cache.json"))


def _key(sim: Simulation) -> str:
    import torch

    c = sim.cfg
    name = torch.cuda.get_device_name(sim.device).replace(" ", "_")
    bucket = 1 << max(0, math.ceil(math.log2(max(1, sim.n_particles))))
    return f"{name}|n{bucket}|k{c.n_grids}|g{c.grid_size}|{c.mass_mode}|{c.index_mode}|{c.solver}"


def _measure(sim: Simulation, reps: int) -> np.ndarray:
    """Mean per-phase device ms over `reps` profiled steps (after 2 warm-ups)."""
    lib = _lib.lib()
    h = sim.handle
    ph = (ctypes.c_float * 4)()
    rows = []
    with torch_device(sim.device):
        for i in range(reps + 2):
            _lib.check(lib.mog_step_profiled(h, sim.pos.data_ptr(), sim.vel.data_ptr(),
                                             sim.n_particles, float(sim.cfg.dt), ph,
                                             sim._stream()), "mog_step_profiled")
            if i >= 2:
                rows.append(list(ph))
    return np.array(rows).mean(axis=0)


def _candidates(sim: Simulation) -> dict[str, list[dict]]:
    g = sim.cfg.grid_size
    # every candidate sets every deposit knob it could inherit from an earlier trial
    dep = [dict(deposit_grids_per_cta=gpc, deposit_ppt=ppt, deposit_threads=thr, deposit_chunks=0,
                deposit_split=0)
           for gpc, ppt, thr in itertools.product([0, 3, 6] if g <= 16 else [0],
                                                  [2, 4], [512, 1024])]
    dep.append(dict(deposit_grids_per_cta=-1, deposit_split=0))
    if g in (8, 16) and sim.cfg.mass_mode == "u64":
        # high-word-only histograms: more grids per CTA, low halves as global atomics
        dep += [dict(deposit_split=1, deposit_grids_per_cta=0, deposit_ppt=4, deposit_threads=thr,
                     deposit_chunks=0) for thr in (512, 1024)]
    if g in (8, 16, 32) and sim.cfg.mass_mode == "u64":
        # count histograms: one word per cell, other masses than a CTA's
        # first as global atomics
        dep += [dict(deposit_split=2, deposit_grids_per_cta=0, deposit_ppt=4, deposit_threads=1024,
                     deposit_chunks=0)]
    upd = [dict(update_staged=0, update_direct_ppt=1), dict(update_staged=0, update_direct_ppt=4)]
    if g <= 16:
        upd += [dict(update_staged=1, update_threads=t) for t in (512, 768, 1024)]
    order = [dict(sort_every=0), dict(sort_every=16)]
    return {"deposit": dep, "update": upd, "order": order}


def _batch_key(batch) -> str:
    import torch

    name = torch.cuda.get_device_name(batch.sims[0].device).replace(" ", "_")
    parts = []
    for s in batch.sims:
        c = s.cfg
        bucket = 1 << max(0, math.ceil(math.log2(max(1, s.n_particles))))
        parts.append(f"n{bucket}k{c.n_grids}g{c.grid_size}{c.mass_mode}")
    return "batch|" + name + "|" + ",".join(parts)


def autotune_batch(batch, reps: int = 3, cache: Path | None = CACHE, force: bool = False) -> dict:
    """Pick and apply the fastest launch shapes of a Batch (work queue on or
    off, particles per deposit tile) by timing whole ensemble steps with
    CUDA events; the particles every trial advanced are restored."""
    import torch

    key = _batch_key(batch)
    table = {}
    if cache is not None and cache.exists():
        try:
            table = json.loads(cache.read_text())
        except (OSError, json.JSONDecodeError):
            table = {}
    if key in table and not force:
        batch.tune(**table[key]["tuning"])
        return table[key]
    saved = [(s.pos.clone(), s.vel.clone()) for s in batch.sims]
    cands = [dict(work_queue=1, deposit_chunk=c, deposit_split=sp)
             for sp in (0, 1) for c in (131072, 262144, 393216)]
    cands.append(dict(work_queue=0, deposit_chunk=0, deposit_split=0))
    results = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    try:
        for cand in cands:
            batch.tune(**cand)
            batch.step(2)  # capture + warm-up
            torch.cuda.synchronize()
            e0.record()
            batch.step(reps)
            e1.record()
            e1.synchronize()
            results.append((e0.elapsed_time(e1) / reps, cand))
            for s, (p, v) in zip(batch.sims, saved):
                s.pos.copy_(p)
                s.vel.copy_(v)
    finally:
        for s, (p, v) in zip(batch.sims, saved):
            s.pos.copy_(p)
            s.vel.copy_(v)
    ms, best = min(results, key=lambda r: r[0])
    batch.tune(**best)
    entry = {"tuning": best, "step_ms": ms,
             "trials": [{"tuning": c, "step_ms": t} for t, c in results]}
    if cache is not None:
        table[key] = entry
        try:
            cache.write_text(json.dumps(table, indent=1, sort_keys=True))
        except OSError:
            pass
    return entry


def autotune(sim: Simulation, reps: int = 4, cache: Path | None = CACHE, force: bool = False) -> dict:
    """Pick and apply the fastest launch shapes for sim's current particles."""
    key = _key(sim)
    table = {}
    if cache is not None and cache.exists():
        try:
            table = json.loads(cache.read_text())
        except (OSError, json.JSONDecodeError):
            table = {}
    if key in table and not force:
        sim.tune(**table[key]["tuning"])
        return table[key]
    p0, v0 = sim.pos.clone(), sim.vel.clone()
    best: dict = {}
    phase = {"deposit": 1, "update": 3, "order": None}
    try:
        for group, cands in _candidates(sim).items():
            results = []
            for cand in cands:
                trial = {**best, **cand}
                try:
                    sim.tune(**trial)
                    ms = _measure(sim, reps)
                except _lib.MogError:
                    continue
                t = float(ms.sum()) if phase[group] is None else float(ms[phase[group]])
                results.append((t, cand))
                sim.pos.copy_(p0)
                sim.vel.copy_(v0)
            if results:
                best.update(min(results, key=lambda r: r[0])[1])
        sim.tune(**best)
        total = float(_measure(sim, reps).sum())
    finally:
        sim.pos.copy_(p0)
        sim.vel.copy_(v0)
    entry = {"tuning": best, "step_ms": total}
    if cache is not None:
        table[key] = entry
        try:
            cache.write_text(json.dumps(table, indent=1, sort_keys=True))
        except OSError:
            pass
    return entry
