"""Build oracle/_ref: the reference's own GLSL compute shaders compiled as C++.

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.  Reads the seven hot-path shaders
(shaders/{mass,complex,fft_batched,fourier,greens,pack,update}.glsl) and the
initial-condition sampler (shaders/init_particles.glsl) from a
reference checkout ($MOG_REFERENCE, else ``reference`` beside this
repository's root), and the
particle vertex and fragment shaders embedded in main.py's init_render
(main.py:359-410), rewrites
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
    """$MOG_REFERENCE, else a checkout named ``reference`` beside the repository."""
    env = os.environ.get("MOG_REFERENCE")
    return Path(env) if env else HERE.parent.parent / "reference"


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


# stage-specific declarations of the particle draw's shaders (main.py:359-410)
POINT_STAGES = {"point_vs": "vec4 gl_Position;\nfloat gl_PointSize;\n",
                "point_fs": "vec2 gl_PointCoord;\nbool discarded;\n"}


def point_shader_sources() -> dict[str, str]:
    """The vertex and fragment shader strings of render_prog (main.py:359-410)."""
    text = (reference_root() / "main.py").read_text()
    m = re.search(r'self\.render_prog\s*=\s*self\.ctx\.program\(\s*vertex_shader\s*=\s*"""(.*?)"""'
                  r'\s*,\s*fragment_shader\s*=\s*"""(.*?)"""', text, re.S)
    if not m:
        raise RuntimeError("render_prog shaders not found in main.py")
    return {"point_vs": m.group(1), "point_fs": m.group(2)}


def translate_stage(src: str, name: str) -> str:
    """A vertex or fragment shader: attributes, varyings and plain uniforms
    become namespace variables the harness sets and reads; `discard` sets a
    flag and returns."""
    s = re.sub(r"layout\s*\([^)]*\)\s*in\s+", "", src)
    s = re.sub(r"^(\s*)(?:uniform|in|out)\s+", r"\1", s, flags=re.M)
    s = re.sub(r"\bdiscard\s*;", "{ discarded = true; return; }", s)
    body = translate(s, name)
    head = "namespace glsl {\nnamespace " + name + "_glsl {\n"
    return body.replace(head, head + POINT_STAGES[name], 1)


def sources_available() -> bool:
    root = reference_root() / "shaders"
    return (all((root / f"{n}.glsl").exists() for n in SHADERS) and
            (reference_root() / "main.py").exists())


def build(force: bool = False) -> Path:
    root = reference_root() / "shaders"
    GEN.mkdir(parents=True, exist_ok=True)
    deps = [HERE / "glsl_compat.hpp", HERE / "ref_harness.cpp", Path(__file__)]
    deps += [root / f"{n}.glsl" for n in SHADERS] + [reference_root() / "main.py"]
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    for n in SHADERS:
        (GEN / f"{n}.inc").write_text(translate((root / f"{n}.glsl").read_text(), n))
    for n, src in point_shader_sources().items():
        (GEN / f"{n}.inc").write_text(translate_stage(src, n))
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
