"""The bounds-checked build (libmog_check.so, nvcc -DMOG_CHECK) on small and
odd shapes: no kernel may compute an index outside its buffer (the checked
kernels raise MOG_FLAG_BOUNDS and skip the access), and the checked library
must give bit-for-bit the trajectories of the production library.  Each
library is loaded in its own child process (ctypes loads one per process)."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent

# (n, k, g, tuning): N = 1, 7, 257 and k = 1, 3 as in the reference's
# smallest cases, every grid size the fast kernels specialise, and the
# launch shapes that take the sorted, merged, global and generic paths
CASES = [
    (1, 1, 8, {}),
    (7, 3, 16, {}),
    (257, 3, 4, {}),
    (257, 1, 32, {}),
    (4099, 5, 16, {"sort_every": 1, "deposit_aggregate": -1, "deposit_sorted": 1}),
    (4099, 3, 16, {"sort_every": 0, "deposit_grids_per_cta": -1}),
    (4099, 3, 8, {"sort_every": 0, "deposit_generic": 1}),
    (3001, 2, 64, {}),
    (20000, 7, 16, {"sort_every": 1}),
]

CHILD = r"""
import hashlib, json, sys
import numpy as np
import torch
from mog_solver_b200 import Simulation, _lib

cases = json.loads(sys.argv[1])
out = {}
for idx, (n, k, g, tuning) in enumerate(cases):
    for mass_mode in ("u64", "u32x1000"):
        sim = Simulation({"n_grids": k, "grid_size": g, "world_size": 100.0, "num_particles": n,
                          "G": 100.0, "dt": 1e-3, "damping": 0.999, "seed": idx,
                          "mass_mode": mass_mode})
        if tuning:
            sim.tune(**tuning)
        rng = np.random.default_rng(idx)
        pos = np.zeros((n, 4), np.float32)
        pos[:, :3] = np.mod(rng.normal(50, 15, (n, 3)), 100.0)
        pos[:, 3] = 1.0 if mass_mode == "u32x1000" else rng.uniform(0.5, 2.0, n) / n
        vel = np.zeros_like(pos)
        vel[:, :3] = rng.normal(0, 1, (n, 3))
        sim.set_particles(pos, vel)
        mass = sim.mass_grid().cpu().numpy()
        sim.step()
        sim.step(3)
        torch.cuda.synchronize()
        key = f"{idx}_{mass_mode}"
        digest = lambda t: hashlib.sha256(t.cpu().numpy().tobytes()).hexdigest()
        out[key] = {"status": int(sim.status()), "mass": hashlib.sha256(mass.tobytes()).hexdigest(),
                    "pos": digest(sim.pos), "vel": digest(sim.vel)}
        sim.close()
print("RESULT" + json.dumps(out))
"""


def _run(library):
    env = dict(os.environ, MOG_LIBRARY=str(library), PYTHONPATH=str(ROOT))
    r = subprocess.run([sys.executable, "-c", CHILD, json.dumps(CASES)], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("RESULT")][-1]
    return json.loads(line[len("RESULT"):])


def test_checked_build_raises_no_bounds_flag_and_matches_production():
    from mog_solver_b200 import FLAG_BOUNDS
    from mog_solver_b200.build import build

    plain = _run(build())
    checked = _run(build(check=True))
    assert plain.keys() == checked.keys()
    for key in plain:
        assert checked[key]["status"] & FLAG_BOUNDS == 0, key
        assert checked[key]["status"] == plain[key]["status"], key
        for field in ("mass", "pos", "vel"):
            assert checked[key][field] == plain[key][field], (key, field)
