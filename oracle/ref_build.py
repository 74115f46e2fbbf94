"""Build oracle/_ref: the reference's own GLSL compute shaders compiled as C++.

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.  Reads the seven hot-path shaders
(shaders/{mass,complex,fft_batched,fourier,greens,pack,update}.glsl) and the
initial-condition sampler (shaders/init_particles.glsl) from a
reference checkout (default /root/reference, or $MOG_REFERENCE), rewrites
their GLSL-only declarations with a handful of regular expressions (SSBO
blocks -> SSBO<T>, image uniforms -> image references, layout qualifiers
dropped, float literals suffixed ``f`` so they stay binary32, swizzles
``.xyz``/``.xy`` -> accessor calls), wraps each shader in its own namespace
inside ``glsl`` and compiles them with glsl_compat.hpp and ref_harness.cpp:

    g++ -O2 -std=c++20 -ffp-contract=off -fopenmp -fPIC -shared

Output (git-ignored, never committed): oracle/_ref/gen/*.inc and
oracle/_ref/libmogref.so.  Nothing of the reference is copied into the
repository; the translation is regenerated from the checkout on each build.
"""
from __future__ import annotations

import os
import re
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
GEN = OUT / "gen"
LIB = OUT / "libmogref.so"
SHADERS = ["mass", "complex", "fft_batched", "fourier", "greens", "pack", "update", "init_particles"]


def reference_root() -> Path:
    return Path(os.environ.get("MOG_REFERENCE", "/root/reference"))


def translate(src: str, name: str) -> str:
    s = src.replace("#version 460", "")
    s = re.sub(r"layout\s*\(\s*local_size[^)]*\)\s*in\s*;", "", s)
    s = re.sub(
        r"layout\s*\([^)]*\)\s*(?:(?:readonly|writeonly|coherent|restrict)\s+)*buffer\s+\w+\s*"
        r"\{\s*(\w+)\s+(\w+)\s*\[\s*\]\s*;\s*\}\s*;",
        r"SSBO<\1> \2;", s)
    s = re.sub(r"layout\s*\([^)]*\)\s*(?:(?:readonly|writeonly)\s+)*uniform\s+image3D\s+(\w+)\s*;",
               r"image3D_ref \1;", s)
    s = re.sub(r"layout\s*\([^)]*\)\s*uniform\s+", "", s)
    s = re.sub(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])",
               r"\1f", s)
    s = re.sub(r"\.(xyz|xy)\b", r".\1_()", s)
    return ("namespace glsl {\nnamespace " + name + "_glsl {\n#define DIM 3\n" + s +
            "\n#undef DIM\n}  // namespace " + name + "_glsl\n}  // namespace glsl\n")


def sources_available() -> bool:
    root = reference_root() / "shaders"
    return all((root / f"{n}.glsl").exists() for n in SHADERS)


def build(force: bool = False) -> Path:
    root = reference_root() / "shaders"
    GEN.mkdir(parents=True, exist_ok=True)
    deps = [HERE / "glsl_compat.hpp", HERE / "ref_harness.cpp", Path(__file__)]
    deps += [root / f"{n}.glsl" for n in SHADERS]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    for n in SHADERS:
        (GEN / f"{n}.inc").write_text(translate((root / f"{n}.glsl").read_text(), n))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", "-I", str(HERE), "-I", str(GEN), "-o", str(tmp),
           str(HERE / "ref_harness.cpp")]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


def build_if_possible() -> Path | None:
    """Build when the reference checkout is present; otherwise keep whatever
    was built before (the .so travels with the source tree)."""
    if sources_available():
        return build()
    return LIB if LIB.exists() else None


if __name__ == "__main__":
    print(build(force=True))
