"""Register budgets of the headline kernels, from ptxas's resource report
(`-Xptxas -v`, compiled for sm_100a here; no GPU needed).

learned_kernel runs two CTAs of 256 threads per SM, so it has exactly 128
registers a thread; a change anywhere in its inputs (a field added to the
Ensemble it takes by value once made it spill 220 bytes and run 20 %
slower) can push it over.  This test fails on any spill in the learned
step's instantiation.
"""
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "mog_solver_b200" / "csrc"
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"

pytestmark = pytest.mark.skipif(not Path(NVCC).exists(), reason="nvcc not available")


def _resources(src: str) -> dict[str, tuple[int, int]]:
    """{mangled kernel name: (registers, spill store bytes)} for one source file."""
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
           "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
           "-I", str(ROOT / "include"), "-Xptxas", "-v", "-c", str(CSRC / src), "-o", "/dev/null"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out, name, spill = {}, None, 0
    for line in r.stderr.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            name = m.group(1)
            continue
        m = re.search(r"(\d+) bytes spill stores", line)
        if m and name:
            spill = int(m.group(1))
            continue
        m = re.search(r"Used (\d+) registers", line)
        if m and name:
            out[name] = (int(m.group(1)), spill)
            name, spill = None, 0
    return out


def _pick(res, pattern):
    hits = {k: v for k, v in res.items() if pattern in k}
    assert hits, f"no kernel matching {pattern}"
    return hits


def test_learned_step_kernel_fits_128_registers_without_spills():
    # learned_kernel<IDX 0, LG 4, OUT 0 (step), K 32, MINB 2>: the k = 32, g = 16 step
    hits = _pick(_resources("learned.cu"), "learned_kernelILi0ELi4ELi0ELi32ELi2E")
    for name, (regs, spill) in hits.items():
        assert regs <= 128 and spill == 0, (name, regs, spill)

