"""Build libmog.so (the sm_100a CUDA library behind include/mog.h) in-tree.

    python -m mog_solver_b200.build [--verbose-ptxas]

The library is compiled with nvcc for sm_100a only and placed next to this
file, where ``mog_solver_b200._lib`` loads it.  No JIT cache is involved, so
the built file travels with the source tree.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libmog.so"
SOURCES = ["mog_api.cu", "deposit.cu", "spectral.cu", "update.cu", "convolution.cu",
           "diagnostics.cu", "sort.cu", "learned.cu", "dft_tc.cu", "ics.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the MOG library needs the CUDA toolkit to build")
    return cand


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True) -> Path:
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    deps += [ROOT / "include" / "mog.h", Path(__file__)]
    if not force and not _stale(OUT, deps):
        return OUT
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-I", str(ROOT / "include")]
    if ptxas_verbose:
        common += ["-Xptxas", "-v"]
    objs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = common + ["-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if ptxas_verbose or not quiet:
            sys.stderr.write(r.stdout + r.stderr)
        objs.append(str(obj))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, OUT)
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    out = build(force=a.force, ptxas_verbose=a.verbose_ptxas, quiet=False)
    print(out)


if __name__ == "__main__":
    main()
