"""A few steps of a fixed workload, for running under a profiler.

    python -m mog_solver_b200.profile_step [--path plain|learned|render|batch] [--steps 6]
                                           [--n N] [--k K] [--g 16|32] [--dft fp32|bf16x3]
                                           [--width W] [--height H] [--tuning JSON]

plain:   k = 240 grids of 16^3 (or --k, --g, --dft), the colliding-disk set
         (N = 1,048,576, seeded two exponential disks), mog_step;
learned: k = 32 grids of 16^3, the same particles, mog_learned_step with the
         committed model (models/learned_k32_g16.npz);
render:  frames of the same particles drawn headless (mog_render) at
         --width x --height (default 2560 x 1440), default camera, 1-pixel
         points, 8-bit target;
batch:   the batched uneven ensemble of 8 Plummer-sphere simulations
         (N 65,536..2,097,152, (k, g) round-robin over (64,16), (128,16),
         (240,16), (64,32), (128,32)) divided in size by --n-div, stepped
         with mog_batch_step (the work-queue launches).
--tuning: mog_tuning fields as JSON (plain and learned paths).
Everything is set up first; the steps run back to back on the default
stream and the status flags are checked at the end.
"""
from __future__ import annotations

import argparse


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--path", default="plain", choices=["plain", "learned", "render", "batch"])
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--k", type=int, default=0, help="grids (default 240 plain, 32 learned)")
    ap.add_argument("--g", type=int, default=16)
    ap.add_argument("--dft", default="fp32", choices=["fp32", "bf16x3"])
    ap.add_argument("--width", type=int, default=2560)
    ap.add_argument("--height", type=int, default=1440)
    ap.add_argument("--tuning", default="", help="JSON object of mog_tuning fields")
    ap.add_argument("--n-div", type=int, default=1, help="batch: divide every N by this")
    a = ap.parse_args()

    import json

    import torch

    from . import _lib, ics
    from .learned import Model
    from .simulation import Simulation
    from .train_learned import DEFAULT_MODEL

    if a.path == "batch":
        from .batch import Batch

        sims = []
        for i, (n, kk, gg) in enumerate([(65536, 64, 16), (131072, 128, 16), (262144, 240, 16),
                                         (524288, 64, 32), (1048576, 128, 32), (1048576, 64, 16),
                                         (2097152, 128, 16), (2097152, 240, 16)]):
            n = max(256, n // a.n_div)
            s = Simulation({"n_grids": kk, "grid_size": gg, "world_size": 100.0, "num_particles": n,
                            "G": 100.0, "dt": 1e-5, "damping": 0.999, "seed": 100 + i})
            s.set_particles(*ics.plummer(n, 100.0, seed=i))
            sims.append(s)
        b = Batch(sims)
        b.step(a.steps)
        torch.cuda.synchronize()
        for s in sims:
            s.check()
        print(f"batch: {a.steps} ensemble steps, {b.tuning()}")
        b.close()
        return
    k, seed = (240, 2000) if a.path == "plain" else (32, 1000)
    k = a.k or k
    sim = Simulation({"n_grids": k, "grid_size": a.g, "world_size": 100.0, "num_particles": a.n,
                      "G": 100.0, "dt": 1e-5, "damping": 0.999, "seed": seed,
                      "dft_precision": a.dft})
    pos, vel = ics.two_disks(a.n, 100.0, seed=1, g_eff=sim.effective_g())
    sim.set_particles(pos, vel)
    if a.tuning:
        sim.tune(**json.loads(a.tuning))
    lib = _lib.lib()
    model = Model.load(DEFAULT_MODEL) if a.path == "learned" else None
    torch.cuda.synchronize()
    if a.path == "render":
        from .render import Renderer, params

        r = Renderer()
        p = params(a.width, a.height, world_size=100.0, speed_scale=0.2)
        img = torch.empty((a.height, a.width, 4), dtype=torch.uint8, device=sim.pos.device)
        for _ in range(a.steps):
            r.render(sim.pos, sim.vel, p=p, out=img)
        torch.cuda.synchronize()
        print(f"render: {a.steps} frames of N={a.n} at {a.width}x{a.height}: {r.stats()}")
        r.close()
        return
    for _ in range(a.steps):
        if model is None:
            _lib.check(lib.mog_step(sim.handle, sim.pos.data_ptr(), sim.vel.data_ptr(), a.n, 1e-5,
                                    None), "mog_step")
        else:
            _lib.check(lib.mog_learned_step(sim.handle, model.handle, sim.pos.data_ptr(),
                                            sim.vel.data_ptr(), a.n, 1e-5, None), "mog_learned_step")
    torch.cuda.synchronize()
    sim.check()
    print(f"{a.path}: {a.steps} steps of N={a.n}, k={k}, g={a.g}, dft={a.dft}: ok")


if __name__ == "__main__":
    main()
