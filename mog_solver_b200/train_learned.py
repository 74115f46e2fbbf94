"""Train and evaluate the learned correction (k = 32 -> k = 240, g = 16).

    python -m mog_solver_b200.train_learned [--sets 64] [--n 262144] [--steps 2000]
           [--out mog_solver_b200/models/learned_k32_g16.npz] [--report report.json]

Training data are pairs the method generates itself: 64 seeded Gaussian-clump
sets (20 clumps, log-uniform widths 1..8, 10 % uniform background) and 32
randomly oriented disk pairs (ics.rotated_disk_pair: scale radius, thickness
and separation drawn around the benchmark's, never at them), features of a
k = 32 ensemble and the k = 240 force minus the k = 32 base force
(learned.generate_dataset).  Adam, lr 1e-3, batch 8192.  The network's
output scale is then chosen on held-out validation sets (a clump set and a
disk pair with seeds outside the training ones): the alpha in {0.25, 0.5,
0.75, 1} whose learned force is closest to k = 240, or 0 (the
least-squares force alone) when none is (learned.select_output_scale).

Evaluation on the colliding-disk set (N = 1,048,576): relative RMS error
against the FP64 direct sum (mog_direct_sum, 16,384 sampled targets, all
sources; softening 0, h/4, h/2) and against plain k = 240, for plain
k = 240, plain k = 32 and learned k = 32; and device time per step of the
plain k = 240 step and the learned k = 32 step.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
DEFAULT_MODEL = HERE / "models" / "learned_k32_g16.npz"


def evaluate(model, n: int = 1 << 20, k_small: int = 32, k_big: int = 240, g: int = 16,
             world: float = 100.0, G: float = 100.0, steps_timed: int = 50, targets: int = 16384,
             small_seed: int = 1000, big_seed: int = 2000) -> dict:
    import torch

    from . import _lib, ics
    from .learned import _cfg, direct_sum, features, learned_forces, rms_error
    from .simulation import Simulation

    small = Simulation(_cfg(k_small, g, world, G, n, small_seed))
    big = Simulation(_cfg(k_big, g, world, G, n, big_seed))
    pos, vel = ics.two_disks(n, world, seed=1, g_eff=big.effective_g())
    small.set_particles(pos, vel)
    big.set_particles(pos, vel)
    h = world / g
    tid = torch.from_numpy(np.random.default_rng(0).choice(n, targets, replace=False)).cuda()
    P = small.pos
    T = P[tid].contiguous()
    f_big = big.forces()
    f_small = small.forces()
    f_learn = learned_forces(small, model)
    # the least-squares correction alone (feature slots 12-14), without the network
    mean, feat = features(small, model)
    f_reg = mean.clone()
    f_reg[:, :3] += feat[:, 12:15]
    report = {"n": n, "k_small": k_small, "k_big": k_big, "g": g, "targets": targets}
    for soft_name, soft in (("0", 0.0), ("h/4", h / 4), ("h/2", h / 2)):
        D = direct_sum(T, P, world, big.effective_g(), soft)
        report[f"rms_vs_direct[soft={soft_name}]"] = {
            "plain_k240": rms_error(f_big[tid], D), "plain_k32": rms_error(f_small[tid], D),
            "learned_k32": rms_error(f_learn[tid], D),
            "regression_only_k32": rms_error(f_reg[tid], D)}
    report["rms_vs_k240"] = {"plain_k32": rms_error(f_small, f_big), "learned_k32": rms_error(f_learn, f_big),
                             "regression_only_k32": rms_error(f_reg, f_big)}

    # device time per step (L2 flushed between steps)
    lib = _lib.lib()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    sptr = ctypes.c_void_p(stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(steps_timed):
            flush.zero_()
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
        return tot / steps_timed

    def plain_step():
        _lib.check(lib.mog_step(big.handle, big.pos.data_ptr(), big.vel.data_ptr(), n, 1e-5, sptr), "step")

    def learned_step():
        _lib.check(lib.mog_learned_step(small.handle, model.handle, small.pos.data_ptr(),
                                        small.vel.data_ptr(), n, 1e-5, sptr), "learned step")

    ms_big = timed(plain_step)
    ms_learn = timed(learned_step)
    report["ms_per_step"] = {"plain_k240": ms_big, "learned_k32": ms_learn}
    report["particle_steps_per_s"] = {"plain_k240": n / (ms_big / 1e3), "learned_k32": n / (ms_learn / 1e3)}
    report["speedup_learned_over_plain_k240"] = ms_big / ms_learn
    small.close()
    big.close()
    return report


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--sets", type=int, default=64)
    ap.add_argument("--disk-sets", type=int, default=32)
    ap.add_argument("--n", type=int, default=262144)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--out", default=str(DEFAULT_MODEL))
    ap.add_argument("--report", default="")
    ap.add_argument("--eval-only", action="store_true")
    args = ap.parse_args()

    from . import ics
    from .learned import Model, generate_dataset, select_output_scale, train

    t0 = time.time()
    if args.eval_only:
        model = Model.load(args.out)
        hist, stats = [], {}
    else:
        data = generate_dataset(n_sets=args.sets, n=args.n, disk_sets=args.disk_sets)
        t1 = time.time()
        model = Model(seed=0)
        hist = train(model, data, steps=args.steps, batch=args.batch, lr=args.lr)
        stats = dict(data.stats, dataset_seconds=t1 - t0, train_seconds=time.time() - t1)
        val = [ics.clumps(args.n, 100.0, seed=900)[0], ics.rotated_disk_pair(args.n, 100.0, seed=990)[0]]
        stats["output_scale_selection"] = select_output_scale(model, val)
        Path(args.out).parent.mkdir(parents=True, exist_ok=True)
        model.save(args.out)
        del data
    rep = evaluate(model)
    # the network against the method without it (least squares alone), on a
    # held-out clump set and on the evaluation disks, both at N = 2^20
    from .learned import residual_errors

    held = [ics.clumps(1 << 20, 100.0, seed=901)[0], ics.two_disks(1 << 20, 100.0, seed=1)[0]]
    rep["ablation_vs_k240"] = dict(zip(["clumps_seed901", "disks"],
                                       residual_errors(model, held, alphas=(1.0,))))
    rep["training"] = {"sets": args.sets, "disk_sets": args.disk_sets, "n": args.n,
                       "steps": args.steps, "batch": args.batch,
                       "lr": args.lr, "loss_history": hist, **stats}
    text = json.dumps(rep, indent=2)
    print(text)
    if args.report:
        Path(args.report).write_text(text)
    model.close()


if __name__ == "__main__":
    main()
