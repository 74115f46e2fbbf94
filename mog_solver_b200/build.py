"""Build libmog.so (the sm_100a CUDA library behind include/mog.h) in-tree.

    python -m mog_solver_b200.build [--force] [--verbose-ptxas] [--check]

The library is compiled with nvcc for sm_100a only and placed next to this
file, where ``mog_solver_b200._lib`` loads it.  No JIT cache is involved, so
the built file travels with the source tree.  The translation units compile
in parallel, one nvcc process each.

``--check`` builds libmog_check.so instead: the same kernels compiled with
-DMOG_CHECK, which bounds-check their scatter and gather indices, skip an
access outside its buffer and raise MOG_FLAG_BOUNDS in the status word.  Load
it with MOG_LIBRARY=<path to libmog_check.so>.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libmog.so"
OUT_CHECK = PKG / "libmog_check.so"
SOURCES = ["mog_api.cu", "deposit.cu", "spectral.cu", "update.cu", "convolution.cu",
           "diagnostics.cu", "sort.cu", "learned.cu", "dft_tc.cu", "ics.cu", "render.cu",
           "shard.cu"]
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


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = True,
          check: bool = False) -> Path:
    out = OUT_CHECK if check else OUT
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    deps += [ROOT / "include" / "mog.h", Path(__file__)]
    if not force and not _stale(out, deps):
        return out
    objdir = PKG / ("_build_check" if check else "_build")
    objdir.mkdir(exist_ok=True)
    common = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", str(ROOT / "include")]
    if check:
        common += ["-DMOG_CHECK"]
    if ptxas_verbose:
        common += ["-Xptxas", "-v"]

    def compile_one(src: str):
        obj = objdir / (Path(src).stem + ".o")
        r = subprocess.run(common + ["-c", str(CSRC / src), "-o", str(obj)], capture_output=True,
                           text=True)
        return src, obj, r

    objs = []
    with ThreadPoolExecutor(max_workers=max(1, min(len(SOURCES), os.cpu_count() or 1))) as pool:
        for src, obj, r in pool.map(compile_one, SOURCES):
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
            if ptxas_verbose or not quiet:
                sys.stderr.write(r.stdout + r.stderr)
            objs.append(str(obj))
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--check", action="store_true",
                    help="build libmog_check.so with the -DMOG_CHECK bounds checks")
    a = ap.parse_args()
    out = build(force=a.force, ptxas_verbose=a.verbose_ptxas, quiet=False, check=a.check)
    print(out)


if __name__ == "__main__":
    main()
