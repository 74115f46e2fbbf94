#!/usr/bin/env python
"""Throughput of the Mixture-of-Grids force-and-step path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--workload learned|c2|c3|c4|c1|render] [--impl ours|reference]

Default workload (``learned``, one GPU): the headline metric, particle-steps/s
of the learned k = 32 step at the RMS force error of plain k = 240, on the
colliding-disk set: N = 1,048,576 particles, grids of 16^3, G = 100,
dt = 1e-5, damping 0.999 (seeded synthetic particles: two exponential disks
with scale radius 8 and sech^2 height 0.5, centres 40 apart, relative speed
5).  Before timing, the RMS force error of learned k = 32 and of plain
k = 240 against the FP64 direct sum is measured on 16,384 sampled particles
at softening 0, h/4 and h/2 and reported in ``accuracy``, beside the cheap
ensemble's plain mean and its least-squares correction alone, and again
after 100 steps of each method (``accuracy.after_100_steps``).  ``value`` is
the learned step's particle-steps/s with the particles resident in HBM
(device time of K steps, CUDA events, L2 flushed between steps); the plain
k = 240 step is timed the same way and reported under ``plain_k240``.
``e2e`` is the learned path through its public API
(``LearnedSimulation.step_host``, with its variance gate) with the particles
in pinned host memory: every step copies them in and back, in chunks
overlapped with the kernels.  On one GPU the default run then times c1, c3,
c4 and the render frame in short runs of their own and embeds their lines
under ``other_workloads`` (``--no-extra`` skips them).

``c2`` times the plain k = 240 step alone, ``c1`` the small uniform-cube
case, ``c3`` the batched uneven ensemble and ``c4`` the plain k = 240, g = 32
step with the DFT passes on the tensor cores (BF16 hi+lo x3), ``render`` one
headless frame of the colliding-disk set (the reference's particle draw,
2560 x 1440, 1-pixel points, 8-bit target).  Under torchrun (N > 1) every
rank advances its own independent simulation of the same size (replicas;
the step has no cross-GPU exchange) and the time is the maximum over ranks.

``--impl reference`` times the reference's own shader code on the host cores
(the GLSL compute shaders compiled as C++ by oracle/, OpenMP over all
threads) on a bounded sample of the plain k = 240 workload (the reference
has no learned path); without that build it falls back to the C/NumPy
restatement in oracle/.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-steps/s at fixed RMS force error vs FP64 direct sum: learned k=32 vs plain k=240"
# the force the plain path computes at g = 16: the reference's step_fft hands
# one scratch texture to both the x and the z inverse transform
# (main.py:638-646), so its shaders store the z gradient as Fx at g = 4, 16,
# 64; this library computes the intended x gradient unless
# reference_texture_aliasing is set
FFT_ALIASING = ("off: the intended x gradient (the reference's shaders store the z gradient as "
                "Fx at g = 4, 16, 64 through a shared scratch texture, main.py:638-646; "
                "config reference_texture_aliasing reproduces that)")
UNIT = "particle-steps/s"
# pieces the host-buffer steps move their particles in (4 overlapped best on
# the B200's host link: 1.15 ms per learned step at N = 2^20 against 1.50 ms
# for copy in, step, copy out)
E2E_CHUNKS = 4
# The comparison leg of the learned workload: both steps with the deposit's
# two-word shared histogram (mog_tuning.deposit_split = -1).  By default the
# Python layer picks the high-word histogram for these particles (every mass
# is 1/N with N = 2^20, so every fixed-point low half is zero); launch shapes
# never change a result.
TWO_WORD = {"deposit_split": -1}

WORKLOADS = {
    "learned": dict(desc="learned k=32 vs plain k=240, g=16, two colliding exponential disks, "
                         "N=1,048,576",
                    n=1 << 20, k=240, k_small=32, g=16, L=100.0, G=100.0, dt=1e-5, damping=0.999,
                    ic="disks", seed=1),
    "c2": dict(desc="plain MOG k=240 g=16, two colliding exponential disks, N=1,048,576",
               n=1 << 20, k=240, g=16, L=100.0, G=100.0, dt=1e-5, damping=0.999, ic="disks",
               seed=1),
    "c3": dict(desc="batched uneven ensemble: 8 simulations (N 65,536..2,097,152; (k,g) round-robin "
                    "over (64,16),(128,16),(240,16),(64,32),(128,32)), Plummer spheres a=5, one CUDA "
                    "graph per ensemble step",
               sims=[(65536, 64, 16), (131072, 128, 16), (262144, 240, 16), (524288, 64, 32),
                     (1048576, 128, 32), (1048576, 64, 16), (2097152, 128, 16),
                     (2097152, 240, 16)],
               L=100.0, G=100.0, dt=1e-5, damping=0.999, ic="plummer", seed=0),
    "c4": dict(desc="plain MOG k=240 g=32 with the DFT passes on the tensor cores (BF16 hi+lo x3), "
                    "two colliding exponential disks, N=1,048,576",
               n=1 << 20, k=240, g=32, L=100.0, G=100.0, dt=1e-5, damping=0.999, ic="disks",
               seed=1, dft="bf16x3"),
    "render": dict(desc="headless frame of the particle draw (main.py:359-423 under GL point rules): "
                        "two colliding exponential disks, N=1,048,576, 2560x1440, default camera, "
                        "1-pixel points, RGBA8 target",
                   n=1 << 20, k=16, g=16, L=100.0, G=100.0, dt=1e-5, damping=0.999, ic="disks",
                   seed=1, width=2560, height=1440, speed_scale=0.2, frame=True),
    "c1": dict(desc="plain MOG k=16 g=16, uniform cube, N=65,536",
               n=1 << 16, k=16, g=16, L=100.0, G=100.0, dt=1e-5, damping=0.999, ic="uniform",
               seed=0),
}

CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def step_bytes(n: int, k: int, g: int) -> int:
    """Algorithmic bytes of one plain step: B = 64 N + 16 N k + 20 k g^3."""
    return 64 * n + 16 * n * k + 20 * k * g ** 3


def launches_per_step(g: int) -> int:
    return 3 if g <= 16 else 10   # deposit, solve (1 fused or 8 passes), update


def phase_bytes(w: dict) -> dict:
    """Algorithmic bytes per launch of each kernel.

    order (when enabled): the spatial permutation and sorted copy of the
    positions (16 N); deposit: position read (16 N) + one 4-byte cell update per (particle,
    grid) (4 N k) + mass-grid write (4 k g^3); solve: mass read + 3 force
    components written (16 k g^3); update: position and velocity read and
    written (64 N) + one 12-byte force read per (particle, grid) (12 N k).
    The whole step uses B = 64 N + 16 N k + 20 k g^3 (the deposit's
    position read is counted once, inside the 64 N).
    """
    n, k, g3 = w["n"], w["k"], w["g"] ** 3
    return {"order": 16 * n,
            "deposit": 16 * n + 4 * n * k + 4 * k * g3,
            "solve": 16 * k * g3,
            "update": 64 * n + 12 * n * k,
            "step": 64 * n + 16 * n * k + 20 * k * g3}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def dft_tensor_flops(k: int, g: int) -> float:
    """Tensor-core FLOPs of one solve with the BF16 x3 DFT passes: per
    128-line tile a (128 x 2g) . (2g x 2g) real GEMM, three products; lines
    per field pass = pairs g^2; one forward field and three inverse fields,
    three axes each."""
    pairs = (k + 1) // 2
    lines = pairs * g * g
    return 2.0 * lines * (2 * g) * (2 * g) * 3 * (3 + 9)


def profiled_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from a committed ncu summary, if one exists."""
    p = ROOT / "profiles" / f"traffic_{kernel}_{workload}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={CLOCK_FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0:  # sampling has started
                time.sleep(0.01)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        return False

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_particles(w: dict, sim, seed_offset: int = 0):
    from mog_solver_b200 import ics

    n, L = w["n"], w["L"]
    if w["ic"] == "disks":
        return ics.two_disks(n, L, seed=w["seed"] + seed_offset, g_eff=sim.effective_g())
    return ics.uniform_cube(n, L, seed=w["seed"] + seed_offset)


def cpu_baseline(w: dict, budget_s: float = 20.0, steps: int = 3, warmup: int = 0) -> dict:
    """Time the reference's CPU path on a bounded sample of the workload."""
    import oracle.baseline as ob

    return ob.time_reference(w, budget_s=budget_s, steps=steps, warmup=warmup)


def run_reference(args, w: dict) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # every declared step runs (warm-up untimed, then exactly --steps timed),
    # each on one particle sample sized so the whole run stays within ~2 min
    res = cpu_baseline(w, budget_s=min(120.0, max(30.0, 3.0 * (args.steps + args.warmup))),
                       steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT,
        "n_gpus": args.gpus, "steps": res["steps_timed"], "warmup": res["warmup_run"],
        "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": w["desc"] + ("; the reference's plain k=240 step (it has no learned "
                                            "path)" if "k_small" in w else ""),
                   "n": w["n"], "k": w["k"], "g": w["g"], "sample_particles": res["sample_n"],
                   "timed_seconds": round(res["timed_seconds"], 3)},
        "cpu_baseline": {"value": res["value"], "unit": UNIT, "cores": res["cores"],
                         "kind": res["kind"], "sample": res["sample"]},
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, w: dict) -> None:
    import ctypes

    import torch
    import torch.distributed as dist

    from mog_solver_b200 import Simulation, _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)

    cfg = {"n_grids": w["k"], "grid_size": w["g"], "world_size": w["L"], "num_particles": w["n"],
           "G": w["G"], "dt": w["dt"], "damping": w["damping"], "solver": "fft", "seed": 0,
           "index_mode": args.index_mode, "dft_precision": w.get("dft", "fp32")}
    sim = Simulation(cfg, device=dev)
    pos, vel = make_particles(w, sim, seed_offset=rank)
    sim.set_particles(pos, vel)
    tuning = json.loads(args.tuning) if args.tuning else {}
    if tuning:
        sim.tune(**tuning)
    if args.autotune:
        from mog_solver_b200.autotune import autotune

        tuning = autotune(sim, cache=None)["tuning"]
    n = sim.n_particles
    lib = _lib.lib()
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    phase = (ctypes.c_float * 4)()
    dt_eff = float(w["dt"])

    def barrier():
        if world > 1:
            dist.barrier()

    torch.cuda.synchronize()  # particles were uploaded on the default stream

    with torch.cuda.stream(stream):
        h = sim.handle
        sptr = ctypes.c_void_p(stream.cuda_stream)
        for _ in range(args.warmup):
            _lib.check(lib.mog_step(h, sim.pos.data_ptr(), sim.vel.data_ptr(), n, dt_eff, sptr),
                       "warmup")
        stream.synchronize()
        barrier()
        torch.cuda.synchronize()
        step_ms, phases = [], []
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            for _ in range(args.steps):
                flush.zero_()  # evict L2 between timed steps
                ev0.record(stream)
                _lib.check(lib.mog_step_profiled(h, sim.pos.data_ptr(), sim.vel.data_ptr(), n,
                                                 dt_eff, phase, sptr), "timed step")
                ev1.record(stream)
                ev1.synchronize()
                step_ms.append(ev0.elapsed_time(ev1))
                phases.append(list(phase))
        torch.cuda.synchronize()
        barrier()
        sim.check()

        # end to end through the public API, host buffers every step
        host_pos = torch.empty((n, 4), dtype=torch.float32).pin_memory()
        host_vel = torch.empty((n, 4), dtype=torch.float32).pin_memory()
        host_pos.copy_(sim.pos)
        host_vel.copy_(sim.vel)
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sim.step_host(host_pos, host_vel, n_steps=args.warmup, chunks=E2E_CHUNKS)  # warm-up
        torch.cuda.synchronize()
        e2e_ms = []
        for _ in range(args.steps):
            flush.zero_()
            e0.record(stream)
            # copies in and out inside the call, overlapped with the deposit
            # and the copy-out of finished chunks (mog_step_host)
            sim.step_host(host_pos, host_vel, chunks=E2E_CHUNKS)
            e1.record(stream)
            e1.synchronize()
            e2e_ms.append(e0.elapsed_time(e1))
        barrier()

    tot = torch.tensor([sum(step_ms), sum(e2e_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    total_ms, total_e2e = float(tot[0]), float(tot[1])
    value = n * world * args.steps / (total_ms / 1e3)
    e2e = n * world * args.steps / (total_e2e / 1e3)
    ph = np.array(phases)
    mean_ph = ph.mean(axis=0)
    names = ["order", "deposit", "solve", "update"]
    dom = int(np.argmax(mean_ph))
    pb = phase_bytes(w)
    peaks = measured_peaks()
    achieved = pb[names[dom]] / (mean_ph[dom] / 1e3) / 1e9
    step_gbs = pb["step"] / (float(np.mean(step_ms)) / 1e3) / 1e9
    clk = clocks.summary()

    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            r = cpu_baseline(w)
            base = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                    "sample": r["sample"]}
        launches = (3 if w["g"] <= 16 else 10) if w.get("dft") != "bf16x3" else 11
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded two-disk set)"
            if w["ic"] == "disks" else "synthetic (seeded uniform cube)",
            "config": {"workload": w["desc"] + " (plain path; learned k=32 not in this line)",
                       "n": w["n"], "k": w["k"], "g": w["g"], "G": w["G"], "dt": w["dt"],
                       "damping": w["damping"], "index_mode": args.index_mode,
                       "mass_mode": "u64 fixed point", "texture_aliasing": FFT_ALIASING,
                       "parallelism":
                       "single GPU" if world == 1 else f"{world} independent replicas",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "tuning": sim.tuning()},
            "phase_ms": {nm: float(v) for nm, v in zip(names, mean_ph)},
            "roofline": {"bound": "hbm", "kernel": names[dom], "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                         "algorithmic_bytes": pb[names[dom]],
                         "traffic": profiled_traffic(names[dom], args.workload),
                         "step_achieved": step_gbs, "step_frac": step_gbs / peaks["hbm_gbs"]},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 2 * 16 * n,
                    "d2h_bytes_per_step": 2 * 16 * n, "ms_per_step": total_e2e / args.steps},
            "gpu_launches": launches * args.steps,
            "clocks": clk,
        }
        if w.get("dft") == "bf16x3":
            fl = dft_tensor_flops(w["k"], w["g"])
            tf = fl / (mean_ph[2] / 1e3) / 1e12
            line["dft"] = {"precision": "BF16 hi+lo x3, FP32 accumulation (tcgen05)",
                           "solve_ms": float(mean_ph[2]), "tensor_flops_per_solve": fl,
                           "achieved_tflops": tf, "peak_tflops": peaks["bf16_tflops"],
                           "frac": tf / peaks["bf16_tflops"],
                           "note": "whole solve (load, 6 DFT passes, Green's multiply, store) "
                                   "timed; tensor-pipe share in profiles/"}
        if base is not None:
            line["cpu_baseline"] = base
        print(json.dumps(line), flush=True)
    sim.close()
    if world > 1:
        dist.destroy_process_group()


def learned_bytes(n: int, k: int, g: int) -> dict:
    """Algorithmic bytes per launch of the learned step's kernels.

    deposit: position read (16 N) + one 4-byte cell update per (particle,
    grid) (4 N k) + mass-grid write (4 k g^3); solve: mass read + force grid
    written (16 k g^3); cell masses: mass read + w lane written (8 k g^3);
    learned kernel: position and velocity read and written (64 N) + one
    16-byte read per (particle, grid) (16 N k: the world-frame force and the
    cell mass the features need), the same convention as the plain gather's
    12 bytes of force per (particle, grid).  Whole step:
    64 N + 20 N k + 28 k g^3 (the deposit's position read inside the 64 N).
    """
    g3 = g ** 3
    return {"deposit": 16 * n + 4 * n * k + 4 * k * g3, "solve": 16 * k * g3,
            "cell_masses": 8 * k * g3, "learned": 64 * n + 16 * n * k,
            "step": 64 * n + 20 * n * k + 28 * k * g3}


def learned_model():
    """The committed model (trained on the GPU by train_learned.py), or one
    trained here on the same recipe when the file is missing."""
    from mog_solver_b200.learned import Model, generate_dataset, train
    from mog_solver_b200.train_learned import DEFAULT_MODEL

    if DEFAULT_MODEL.exists():
        return Model.load(DEFAULT_MODEL), str(DEFAULT_MODEL.relative_to(ROOT))
    data = generate_dataset()
    model = Model(seed=0)
    train(model, data)
    del data
    return model, "trained in this run (64 clump sets x 262,144, 2,000 Adam steps)"


def run_learned(args, w: dict) -> dict | None:
    import ctypes

    import torch
    import torch.distributed as dist

    from mog_solver_b200 import Simulation, _lib, ics
    from mog_solver_b200.learned import (LearnedSimulation, direct_sum, features, learned_forces,
                                         rms_error)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)

    def cfg(k, seed):
        return {"n_grids": k, "grid_size": w["g"], "world_size": w["L"], "num_particles": w["n"],
                "G": w["G"], "dt": w["dt"], "damping": w["damping"], "solver": "fft", "seed": seed}

    cheap = Simulation(cfg(w["k_small"], 1000), device=dev)
    big = Simulation(cfg(w["k"], 2000), device=dev)
    pos, vel = ics.two_disks(w["n"], w["L"], seed=w["seed"] + rank, g_eff=big.effective_g())
    cheap.set_particles(pos, vel)
    big.set_particles(pos, vel)
    tuning = json.loads(args.tuning) if args.tuning else {}
    if tuning:  # launch shapes for both ensembles (results never depend on them)
        cheap.tune(**tuning)
        big.tune(**{k: v for k, v in tuning.items() if k != "learned_fold"})
    model, model_src = learned_model()
    n = cheap.n_particles
    lib = _lib.lib()

    # accuracy against the FP64 direct sum (untimed): at the initial
    # particles, and after 100 steps of each method from them (each judged
    # at its own particles); with the cheap ensemble's plain mean and its
    # least-squares correction alone beside the learned force
    h = w["L"] / w["g"]
    tid = torch.from_numpy(np.random.default_rng(0).choice(n, 16384, replace=False)).to(dev)

    def judge(learned_pos, plain_pos):
        mean, feat = features(cheap, model, pos=learned_pos)
        ls = mean.clone()
        ls[:, :3] += feat[:, 12:15]
        cols = {"learned_k32": learned_forces(cheap, model, pos=learned_pos)[tid],
                "ls_only_k32": ls[tid], "plain_k32": mean[tid]}
        f_big = big.forces(pos=plain_pos)[tid]
        T, Tb = learned_pos[tid].contiguous(), plain_pos[tid].contiguous()
        out = {}
        for name, soft in (("0", 0.0), ("h/4", h / 4), ("h/2", h / 2)):
            D = direct_sum(T, learned_pos, w["L"], big.effective_g(), soft)
            Db = D if plain_pos is learned_pos else direct_sum(Tb, plain_pos, w["L"],
                                                              big.effective_g(), soft)
            row = {k2: rms_error(v, D) for k2, v in cols.items()}
            row["plain_k240"] = rms_error(f_big, Db)
            row["ratio"] = row["learned_k32"] / row["plain_k240"]
            out[f"soft={name}"] = row
        out["vs_k240_force"] = {k2: rms_error(v, f_big) for k2, v in cols.items()} \
            if plain_pos is learned_pos else None
        return out

    accuracy = judge(cheap.pos, cheap.pos)
    within = all(v["ratio"] <= 1.10 for k2, v in accuracy.items() if k2.startswith("soft"))
    # 100 steps of each method from the same particles (config 5's evaluation)
    p_l, v_l = cheap.pos.clone(), cheap.vel.clone()
    p_b, v_b = cheap.pos.clone(), cheap.vel.clone()
    for _ in range(100):
        _lib.check(_lib.lib().mog_learned_step(cheap.handle, model.handle, p_l.data_ptr(),
                                                v_l.data_ptr(), n, float(w["dt"]), None), "eval")
        _lib.check(_lib.lib().mog_step(big.handle, p_b.data_ptr(), v_b.data_ptr(), n,
                                       float(w["dt"]), None), "eval")
    torch.cuda.synchronize()
    after = judge(p_l, p_b)
    after.pop("vs_k240_force")
    after["trajectory_rms_vs_plain_k240"] = float(torch.sqrt(((p_l[:, :3] - p_b[:, :3]) ** 2)
                                                             .sum(1).mean()).item())
    accuracy_100 = after

    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    phase = (ctypes.c_float * 4)()
    dt_eff = float(w["dt"])
    p0, v0 = cheap.pos.clone(), cheap.vel.clone()

    def barrier():
        if world > 1:
            dist.barrier()

    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        sptr = ctypes.c_void_p(stream.cuda_stream)
        hc, hb, hm = cheap.handle, big.handle, model.handle
        for _ in range(args.warmup):
            _lib.check(lib.mog_learned_step(hc, hm, cheap.pos.data_ptr(), cheap.vel.data_ptr(), n,
                                            dt_eff, sptr), "warmup")
            _lib.check(lib.mog_step(hb, big.pos.data_ptr(), big.vel.data_ptr(), n, dt_eff, sptr),
                       "warmup")
        stream.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        learn_ms, plain_ms = [], []
        with ClockSampler(local) as clocks:
            for _ in range(args.steps):
                flush.zero_()  # evict L2 between timed steps
                ev0.record(stream)
                _lib.check(lib.mog_learned_step(hc, hm, cheap.pos.data_ptr(), cheap.vel.data_ptr(),
                                                n, dt_eff, sptr), "timed learned step")
                ev1.record(stream)
                ev1.synchronize()
                learn_ms.append(ev0.elapsed_time(ev1))
            torch.cuda.synchronize()
            barrier()
            for _ in range(args.steps):
                flush.zero_()
                ev0.record(stream)
                _lib.check(lib.mog_step(hb, big.pos.data_ptr(), big.vel.data_ptr(), n, dt_eff, sptr),
                           "timed plain step")
                ev1.record(stream)
                ev1.synchronize()
                plain_ms.append(ev0.elapsed_time(ev1))
            # both steps once more with the two-word deposit histogram
            saved_c, saved_b = cheap.tuning(), big.tuning()
            cheap.tune(**TWO_WORD)
            big.tune(**TWO_WORD)
            for _ in range(args.warmup):
                _lib.check(lib.mog_learned_step(hc, hm, cheap.pos.data_ptr(), cheap.vel.data_ptr(), n,
                                                dt_eff, sptr), "warmup")
                _lib.check(lib.mog_step(hb, big.pos.data_ptr(), big.vel.data_ptr(), n, dt_eff, sptr),
                           "warmup")
            torch.cuda.synchronize()
            barrier()
            dlearn_ms, dplain_ms = [], []
            for _ in range(args.steps):
                flush.zero_()
                ev0.record(stream)
                _lib.check(lib.mog_learned_step(hc, hm, cheap.pos.data_ptr(), cheap.vel.data_ptr(),
                                                n, dt_eff, sptr), "timed default learned step")
                ev1.record(stream)
                ev1.synchronize()
                dlearn_ms.append(ev0.elapsed_time(ev1))
            for _ in range(args.steps):
                flush.zero_()
                ev0.record(stream)
                _lib.check(lib.mog_step(hb, big.pos.data_ptr(), big.vel.data_ptr(), n, dt_eff, sptr),
                           "timed default plain step")
                ev1.record(stream)
                ev1.synchronize()
                dplain_ms.append(ev0.elapsed_time(ev1))
            cheap.tune(**saved_c)
            big.tune(**saved_b)
        torch.cuda.synchronize()
        barrier()
        # per-kernel device times from separate profiled steps (events
        # between the kernels; not part of the timed region above)
        learn_ph, plain_ph = [], []
        for _ in range(min(args.steps, 50)):
            flush.zero_()
            _lib.check(lib.mog_learned_step_profiled(hc, hm, cheap.pos.data_ptr(),
                                                     cheap.vel.data_ptr(), n, dt_eff, phase, sptr),
                       "profiled learned step")
            learn_ph.append(list(phase))
            flush.zero_()
            _lib.check(lib.mog_step_profiled(hb, big.pos.data_ptr(), big.vel.data_ptr(), n, dt_eff,
                                             phase, sptr), "profiled plain step")
            plain_ph.append(list(phase))
        cheap.check()
        big.check()

        # end to end through the public API (variance gate every 10 steps),
        # host buffers every step
        cheap.pos.copy_(p0)
        cheap.vel.copy_(v0)
        ls = LearnedSimulation(cheap, model, fallback=big, gate_every=10)
        host_pos = torch.empty((n, 4), dtype=torch.float32).pin_memory()
        host_vel = torch.empty((n, 4), dtype=torch.float32).pin_memory()
        host_pos.copy_(p0)
        host_vel.copy_(v0)
        # warm-up: the first call allocates the handle's device copies
        ls.step_host(host_pos, host_vel, n_steps=args.warmup, chunks=E2E_CHUNKS)
        torch.cuda.synchronize()
        barrier()
        e2e_ms = []
        for _ in range(args.steps):
            flush.zero_()
            ev0.record(stream)
            # the records travel host -> device -> host inside the call, in
            # chunks overlapped with the kernels (mog_learned_step_host)
            ls.step_host(host_pos, host_vel, chunks=E2E_CHUNKS)
            ev1.record(stream)
            ev1.synchronize()
            e2e_ms.append(ev0.elapsed_time(ev1))
        barrier()

    tot = torch.tensor([sum(learn_ms), sum(plain_ms), sum(e2e_ms), sum(dlearn_ms), sum(dplain_ms)],
                       dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    t_learn, t_plain, t_e2e, t_dlearn, t_dplain = (float(x) for x in tot)
    value = n * world * args.steps / (t_learn / 1e3)
    plain_value = n * world * args.steps / (t_plain / 1e3)
    e2e = n * world * args.steps / (t_e2e / 1e3)
    lph = np.array(learn_ph).mean(axis=0)
    pph = np.array(plain_ph).mean(axis=0)
    lnames = ["deposit", "solve", "cell_masses", "learned"]
    pnames = ["order", "deposit", "solve", "update"]
    lb = learned_bytes(n, w["k_small"], w["g"])
    pb = phase_bytes(w)
    peaks = measured_peaks()
    ldom, pdom = int(np.argmax(lph)), int(np.argmax(pph))
    l_ach = lb[lnames[ldom]] / (lph[ldom] / 1e3) / 1e9
    p_ach = pb[pnames[pdom]] / (pph[pdom] / 1e3) / 1e9
    clk = clocks.summary()

    if rank == 0:
        base = None
        if world == 1 and not args.no_cpu_baseline:
            r = cpu_baseline(w)
            base = {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": r["kind"],
                    "sample": r["sample"] + "; the reference's plain k=240 step (it has no "
                                            "learned path)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_learn / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded two-disk set)",
            "config": {"workload": w["desc"], "n": w["n"], "k_small": w["k_small"], "k": w["k"],
                       "g": w["g"], "G": w["G"], "dt": w["dt"], "damping": w["damping"],
                       "network": "12-64-64-3 GELU, FP16 tensor-core inference, FP32 features",
                       "model": model_src, "index_mode": "fast", "mass_mode": "u64 fixed point",
                       "texture_aliasing": FFT_ALIASING,
                       "tuning": tuning or "library defaults",
                       "deposit_layout": {1: "high words only (deposit_split 1), chosen by "
                                             "Simulation: every mass is 1/N, N = 2^20, a "
                                             "fixed-point value with a zero low half",
                                          2: "counts of the equal masses (deposit_split 2), "
                                             "chosen by Simulation"}.get(
                                             cheap.tuning()["deposit_split"], "two words per cell"),
                       "parallelism": "single GPU" if world == 1 else f"{world} independent replicas",
                       "l2": "flushed between timed steps (256 MiB write)"},
            "accuracy": {"yardstick": "relative RMS force error vs FP64 periodic direct sum, 16,384 "
                                  "sampled particles, all sources",
                         **accuracy, "learned_within_10pct_of_plain_k240": within,
                         "after_100_steps": accuracy_100},
            "plain_k240": {"value": plain_value, "unit": UNIT,
                           "ms_per_step": t_plain / args.steps,
                           "phase_ms": {nm: float(v) for nm, v in zip(pnames, pph)},
                           "speedup_learned_over_plain": value / plain_value,
                           "two_word_histogram": {
                               "ms_per_step": t_dplain / args.steps,
                               "value": n * world * args.steps / (t_dplain / 1e3)},
                           "roofline": {"bound": "hbm", "kernel": pnames[pdom], "achieved": p_ach,
                                        "peak": peaks["hbm_gbs"], "unit": "GB/s",
                                        "frac": p_ach / peaks["hbm_gbs"],
                                        "algorithmic_bytes": pb[pnames[pdom]],
                                        "traffic": profiled_traffic(pnames[pdom], "c2")}},
            "phase_ms": {nm: float(v) for nm, v in zip(lnames, lph)},
            "two_word_histogram": {
                "tuning": TWO_WORD, "ms_per_step": t_dlearn / args.steps,
                "value": n * world * args.steps / (t_dlearn / 1e3),
                "plain_k240_ms_per_step": t_dplain / args.steps,
                "speedup_learned_over_plain": t_dplain / t_dlearn},
            "roofline": {"bound": "hbm", "kernel": lnames[ldom], "achieved": l_ach,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": l_ach / peaks["hbm_gbs"], "peak_source": peaks["source"],
                         "algorithmic_bytes": lb[lnames[ldom]],
                         "traffic": profiled_traffic(lnames[ldom], "learned"),
                         "note": "effective bytes: 64 N + 16 N k, one 16-byte (force, cell mass) "
                                 "read per (particle, grid) served from L1/L2, like the plain "
                                 "gather's 12 bytes; the kernel is bound by instruction issue "
                                 "(feature statistics over 32 gathered grids)"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 2 * 16 * n,
                    "d2h_bytes_per_step": 2 * 16 * n, "ms_per_step": t_e2e / args.steps,
                    "api": f"LearnedSimulation.step_host (mog_learned_step_host, {E2E_CHUNKS} "
                           "chunks, pinned host buffers)",
                    "gate": f"variance gate every 10 steps, {ls.fallback_steps} fallback steps, "
                            f"last relative spread {ls.last_ratio} vs training {ls.train_ratio}"},
            "gpu_launches": (4 if tuning.get("learned_fold") == -1 or w["g"] not in (8, 16) else 3)
                            * args.steps,
            "clocks": clk,
        }
        if base is not None:
            line["cpu_baseline"] = base
    model.close()
    cheap.close()
    big.close()
    if world > 1:
        dist.destroy_process_group()
    return line if rank == 0 else None


# The other configurations, timed after the headline in short runs of their
# own (one process each, the GPU otherwise idle): c1 the small uniform cube,
# c3 the batched uneven ensemble, c4 the tensor-core DFT at g = 32, and one
# headless frame.  Their lines are embedded whole under "other_workloads".
EXTRA_WORKLOADS = (("c1", 50), ("c3", 10), ("c4", 20), ("render", 10))


def run_extra_workloads() -> dict:
    out = {}
    for name, steps in EXTRA_WORKLOADS:
        cmd = [sys.executable, str(ROOT / "bench.py"), "--workload", name, "--steps", str(steps),
               "--warmup", "3", "--no-cpu-baseline"]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(ROOT))
            lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
            out[name] = json.loads(lines[-1]) if r.returncode == 0 and lines else \
                {"error": f"exit {r.returncode}: {r.stderr[-300:]}"}
        except subprocess.TimeoutExpired:
            out[name] = {"error": "timed out after 300 s"}
    return out


def run_batch(args, w: dict) -> None:
    import torch

    from mog_solver_b200 import Simulation, ics
    from mog_solver_b200.batch import Batch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    sims = []
    for i, (n, k, g) in enumerate(w["sims"]):
        s = Simulation({"n_grids": k, "grid_size": g, "world_size": w["L"], "num_particles": n,
                        "G": w["G"], "dt": w["dt"], "damping": w["damping"], "seed": 100 + i},
                       device=dev)
        pos, vel = ics.plummer(n, w["L"], seed=w["seed"] + i + 1000 * rank)
        s.set_particles(pos, vel)
        sims.append(s)
    torch.cuda.synchronize()
    batch = Batch(sims)
    if args.tuning:
        batch.tune(**json.loads(args.tuning))
    tuned = None
    if args.autotune:
        from mog_solver_b200.autotune import autotune_batch

        tuned = autotune_batch(batch, reps=2, cache=None)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    n_tot = sum(s.n_particles for s in sims)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            batch.step(1)
        stream.synchronize()
        if world > 1:
            torch.distributed.barrier()
        times = []
        with ClockSampler(local) as clocks:
            for _ in range(args.steps):
                flush.zero_()
                e0.record(stream)
                batch.step(1)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        # end to end: all particles copied from pinned host memory and back every step
        hp = [torch.empty((s.n_particles, 4), dtype=torch.float32).pin_memory() for s in sims]
        hv = [torch.empty((s.n_particles, 4), dtype=torch.float32).pin_memory() for s in sims]
        for s, a, b in zip(sims, hp, hv):
            a.copy_(s.pos)
            b.copy_(s.vel)
        torch.cuda.synchronize()
        e2e = []
        for _ in range(args.steps):
            e0.record(stream)
            for s, a, b in zip(sims, hp, hv):
                s.pos.copy_(a, non_blocking=True)
                s.vel.copy_(b, non_blocking=True)
            batch.step(1)
            for s, a, b in zip(sims, hp, hv):
                a.copy_(s.pos, non_blocking=True)
                b.copy_(s.vel, non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            e2e.append(e0.elapsed_time(e1))
    tot = torch.tensor([sum(times), sum(e2e)], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(tot, op=torch.distributed.ReduceOp.MAX)
    total_ms, total_e2e = float(tot[0]), float(tot[1])
    for s in sims:
        s.check()
    btune = batch.tuning()
    if rank == 0:
        peaks = measured_peaks()
        B = sum(step_bytes(n, k, g) for n, k, g in w["sims"])
        ms = total_ms / args.steps
        achieved = B / (ms / 1e3) / 1e9
        line = {
            "metric": METRIC, "value": n_tot * world * args.steps / (total_ms / 1e3), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Plummer spheres)",
            "config": {"workload": w["desc"], "sims": w["sims"], "particles": n_tot,
                       "parallelism": "single GPU" if world == 1 else f"{world} independent replicas",
                       "l2": "flushed between timed steps (256 MiB write)",
                       "autotuned": bool(args.autotune), "batch_tuning": btune,
                       **({"autotune_trials": tuned["trials"]} if tuned else {})},
            "roofline": {"bound": "hbm", "kernel": "whole ensemble step", "achieved": achieved,
                         "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                         "peak_source": peaks["source"], "algorithmic_bytes": B, "traffic": None},
            "e2e": {"value": n_tot * world * args.steps / (total_e2e / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": 32 * n_tot, "d2h_bytes_per_step": 32 * n_tot,
                    "ms_per_step": total_e2e / args.steps},
            # work queue: one deposit and one gather launch for the whole
            # batch, plus each simulation's solve
            "gpu_launches": ((2 + sum(launches_per_step(g) - 2 for _, _, g in w["sims"]))
                             if btune["active_work_queue"] else
                             sum(launches_per_step(g) for _, _, g in w["sims"])) * args.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line), flush=True)
    batch.close()
    for s in sims:
        s.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def render_cpu_baseline(w: dict, pos, vel, budget_s: float = 15.0) -> dict:
    """The oracle's draw (oracle/render.py, one core) on a growing prefix of
    the particles until the budget is used; the frame time is extrapolated
    linearly in the particle count (its cost is per point)."""
    import oracle.render as orc
    from mog_solver_b200.render import camera_matrices

    v, p = camera_matrices(aspect=w["width"] / w["height"])
    kw = dict(width=w["width"], height=w["height"], world_size=w["L"],
              speed_scale=w["speed_scale"], m_view=v, m_proj=p)
    t0 = time.perf_counter()
    orc.render(pos[:0], vel[:0], **kw)
    t_clear = time.perf_counter() - t0
    m, t_pts = 1024, 0.0
    while True:
        t0 = time.perf_counter()
        orc.render(pos[:m], vel[:m], **kw)
        t_pts = time.perf_counter() - t0 - t_clear
        if t_pts * 4 > budget_s or m >= len(pos):
            break
        m *= 4
    frame_s = t_clear + max(t_pts, 0.0) * len(pos) / m
    return {"value": 1.0 / frame_s, "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": f"first {m} of {len(pos)} particles drawn by the NumPy restatement "
                      f"(oracle/render.py), time scaled to all particles"}


def run_render(args, w: dict) -> None:
    import torch

    from mog_solver_b200 import Simulation, render as R

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    dev = torch.device("cuda", local)
    sim = Simulation({"n_grids": w["k"], "grid_size": w["g"], "world_size": w["L"],
                      "num_particles": w["n"], "G": w["G"], "dt": w["dt"],
                      "damping": w["damping"], "seed": w["seed"]}, device=dev)
    pos_h, vel_h = make_particles(w, sim, seed_offset=1000 * rank)
    sim.set_particles(pos_h, vel_h)
    W, H = w["width"], w["height"]
    p = R.params(W, H, world_size=w["L"], speed_scale=w["speed_scale"])
    r = R.Renderer()
    img = torch.empty((H, W, 4), dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hp = torch.from_numpy(np.ascontiguousarray(pos_h, np.float32)).pin_memory()
    hv = torch.from_numpy(np.ascontiguousarray(vel_h, np.float32)).pin_memory()
    himg = torch.empty((H, W, 4), dtype=torch.uint8).pin_memory()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            r.render(sim.pos, sim.vel, p=p, out=img)
        stream.synchronize()
        if world > 1:
            torch.distributed.barrier()
        times = []
        with ClockSampler(local) as clocks:
            for _ in range(args.steps):
                flush.zero_()
                e0.record(stream)
                r.render(sim.pos, sim.vel, p=p, out=img)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
        stats = r.stats()
        e2e = []
        for _ in range(args.steps):
            e0.record(stream)
            sim.pos.copy_(hp, non_blocking=True)
            sim.vel.copy_(hv, non_blocking=True)
            r.render(sim.pos, sim.vel, p=p, out=img)
            himg.copy_(img, non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            e2e.append(e0.elapsed_time(e1))
    tot = torch.tensor([sum(times), sum(e2e)], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(tot, op=torch.distributed.ReduceOp.MAX)
    total_ms, total_e2e = float(tot[0]), float(tot[1])
    if rank == 0:
        peaks = measured_peaks()
        n = w["n"]
        B = 32 * n + 4 * W * H  # particles read once, image written once
        ms = total_ms / args.steps
        achieved = B / (ms / 1e3) / 1e9
        line = {
            "metric": "frames/s of the headless particle draw", "unit": "frames/s",
            "value": world * args.steps / (total_ms / 1e3), "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (u8 target)",
            "data": "synthetic (seeded colliding disks)",
            "config": {"workload": w["desc"], "n": n, "width": W, "height": H,
                       "pairs_per_frame": stats["pairs"],
                       "parallelism": "single GPU" if world == 1 else f"{world} independent replicas",
                       "l2": "flushed between timed frames (256 MiB write)"},
            "roofline": {"bound": "hbm", "kernel": "whole frame (6 kernels and the scans)",
                         "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                         "algorithmic_bytes": B, "traffic": None},
            "e2e": {"value": world * args.steps / (total_e2e / 1e3), "unit": "frames/s",
                    "h2d_bytes_per_step": 32 * n, "d2h_bytes_per_step": 4 * W * H,
                    "ms_per_step": total_e2e / args.steps},
            "gpu_launches": stats["launches"] * args.steps,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = render_cpu_baseline(w, pos_h, vel_h)
        print(json.dumps(line), flush=True)
    r.close()
    sim.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="learned", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--index-mode", default="fast", choices=["fast", "exact"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default="", help="JSON object of mog_tuning fields to apply")
    ap.add_argument("--autotune", action="store_true", help="pick launch shapes before timing")
    ap.add_argument("--no-extra", action="store_true",
                    help="default workload: skip the short c1 / c3 / c4 / render runs")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        if w.get("frame"):
            print(json.dumps({"impl": "reference", "unavailable": "the reference draws with OpenGL "
                              "(main.py:359-423, 678-703); there is no graphics stack here: "
                              "unavailable on this box"}))
            return
        if "sims" in w:
            print(json.dumps({"impl": "reference", "unavailable": "the reference runs one "
                              "simulation per window; no batched path to time"}))
            return
        run_reference(args, w)
    elif w.get("frame"):
        run_render(args, w)
    elif "sims" in w:
        run_batch(args, w)
    elif "k_small" in w:
        line = run_learned(args, w)
        if line is not None:
            if int(os.environ.get("WORLD_SIZE", "1")) == 1 and not args.no_extra:
                line["other_workloads"] = run_extra_workloads()
            print(json.dumps(line), flush=True)
    else:
        run_ours(args, w)


if __name__ == "__main__":
    main()
