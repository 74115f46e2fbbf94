"""The spectral solve with its DFT passes on the tensor cores
(dft_precision bf16x3: BF16 hi + lo split, three products, FP32
accumulation in tensor memory) against the FP64 oracle pipeline and the
FP32 FFT path.  Tolerance: 1e-4 relative L2 against FP64 (the FP32 FFT path
holds 1e-5)."""
import json
import os

import numpy as np
import pytest

from oracle import pipeline as pl

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TC_TOL = 1e-4


def _sim(k, g, n, prec, L=100.0, G=100.0, seed=0):
    from mog_solver_b200 import Simulation

    return Simulation({"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": G,
                       "dt": 1e-5, "damping": 0.999, "seed": seed, "dft_precision": prec})


def _clustered(n, L, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[: n // 2, :3] = np.mod(rng.normal(L / 2, L / 10, (n // 2, 3)), L)
    pos[n // 2:, :3] = rng.uniform(0, L, (n - n // 2, 3))
    pos[:, 3] = 1.0 / n
    return pos


@pytest.mark.parametrize("g,k", [(16, 3), (16, 4), (32, 3)])
def test_tc_solve_matches_fp64(g, k):
    """Grid-frame solve of the same mass grid; k = 3 leaves a pair with one grid."""
    n, L, G = 30000, 100.0, 100.0
    tc = _sim(k, g, n, "bf16x3")
    ff = _sim(k, g, n, "fp32")
    pos = _clustered(n, L, g + k)
    tc.set_particles(pos)
    ff.set_particles(pos)
    m = tc.mass_grid()
    assert torch.equal(m, ff.mass_grid())
    F_tc = tc.solve_grid(m).cpu().numpy()[..., :3]
    F_ff = ff.solve_grid(m).cpu().numpy()[..., :3]
    rho = m.cpu().numpy().view(np.uint64).astype(np.float64) * 2.0 ** -tc.scale_bits
    ref = pl.forces_grid_fp64(rho, G, L)
    e_tc, e_ff = pl.relative_l2(F_tc, ref), pl.relative_l2(F_ff, ref)
    assert e_tc <= TC_TOL, e_tc
    assert e_ff <= 1e-5, e_ff
    assert pl.relative_l2(F_tc, F_ff) <= TC_TOL
    tc.check()
    tc.close()
    ff.close()


def test_tc_step_matches_fft_step():
    """World-frame forces and one full step: tensor-core DFT vs FP32 FFT."""
    n, k, g = 50000, 6, 32
    tc = _sim(k, g, n, "bf16x3")
    ff = _sim(k, g, n, "fp32")
    pos = _clustered(n, 100.0, 5)
    tc.set_particles(pos)
    ff.set_particles(pos)
    a_tc = tc.forces()[:, :3].double()
    a_ff = ff.forces()[:, :3].double()
    assert float(torch.linalg.norm(a_tc - a_ff) / torch.linalg.norm(a_ff)) <= TC_TOL
    tc.step(3)
    ff.step(3)
    torch.cuda.synchronize()
    tc.check()
    d = float(torch.linalg.norm((tc.pos - ff.pos)[:, :3].double()))
    assert np.isfinite(d) and d < 1e-3


def test_tc_rejects_other_sizes():
    from mog_solver_b200 import _lib

    with pytest.raises(_lib.MogError):
        _sim(2, 8, 100, "bf16x3").handle


def test_c4_precision_report():
    """The precision study of the tensor-core DFT on the colliding-disk set:
    N = 1,048,576, k = 240, g = 32; forces of one solve against the FP64
    oracle pipeline for the BF16 x3 and FP32 FFT paths (relative L2 and max
    error).  Writes the numbers to $MOG_REPORT_DIR/dft_precision_c4.json
    when that variable is set."""
    from mog_solver_b200 import ics

    n, k, g, L, G = 1 << 20, 240, 32, 100.0, 100.0
    tc = _sim(k, g, n, "bf16x3")
    ff = _sim(k, g, n, "fp32")
    pos, vel = ics.two_disks(n, L, seed=1, g_eff=tc.effective_g())
    tc.set_particles(pos, vel)
    ff.set_particles(pos, vel)
    m = tc.mass_grid()
    F_tc = tc.solve_grid(m).cpu().numpy()[..., :3].astype(np.float64)
    F_ff = ff.solve_grid(m).cpu().numpy()[..., :3].astype(np.float64)
    rho = m.cpu().numpy().view(np.uint64).astype(np.float64) * 2.0 ** -tc.scale_bits
    ref = pl.forces_grid_fp64(rho, G, L)
    scale = np.abs(ref).max()
    rep = {"workload": "two colliding disks, N=1,048,576, k=240, g=32, one solve",
           "bf16x3": {"rel_l2": pl.relative_l2(F_tc, ref),
                      "max_abs_over_max_ref": float(np.abs(F_tc - ref).max() / scale)},
           "fp32_fft": {"rel_l2": pl.relative_l2(F_ff, ref),
                        "max_abs_over_max_ref": float(np.abs(F_ff - ref).max() / scale)}}
    out = os.environ.get("MOG_REPORT_DIR")
    if out:
        os.makedirs(out, exist_ok=True)
        with open(os.path.join(out, "dft_precision_c4.json"), "w") as f:
            json.dump(rep, f, indent=1)
    assert rep["bf16x3"]["rel_l2"] <= TC_TOL, rep
    assert rep["fp32_fft"]["rel_l2"] <= 1e-5, rep
    tc.close()
    ff.close()
