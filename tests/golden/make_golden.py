"""Generate the golden fixtures in tests/golden from the reference itself.

Run in a container that has the reference checkout ($MOG_REFERENCE, else
``reference`` beside this repository's root) and the built oracle/_ref
(python -m oracle.ref_build):

    python tests/golden/make_golden.py [transforms greens_kernel shaders two_galaxies init_particles camera
                                        point_shaders config]

* transforms.npz   — Simulation.compute_transforms (main.py:157-172) with
                     the reference's own RandomSE3Sampler (main.py:9-62),
                     seeded; main.py is imported with its GL modules stubbed.
* greens_kernel.npz — Simulation.init_greens_kernel (main.py:250-278).
* init_particles.npz — init_particles.glsl, the GPU Perlin/fBm rejection
                     sampler (compiled as C++ by oracle/_ref), two seeded cases.
* two_galaxies.npz — Simulation.init_particles2 (main.py:312-357) after
                     np.random.seed(seed), buffers captured from its writes.
* camera.npz       — the m_view and m_proj uniform bytes that on_render
                     (main.py:678-700) writes, for several orbit-camera
                     angles, distances and aspect ratios (on_render run on a
                     stand-in object that records the writes).
* point_shaders.npz — the particle vertex and fragment shaders of render_prog
                     (main.py:359-410, compiled as C++ by oracle/_ref) on
                     seeded vertices for three cameras and two speed
                     scales, and on seeded gl_PointCoord values.
* config.json      — Simulation.load_config (main.py:174-189) run by the
                     reference: the mapping it reads from its own config.yaml,
                     and its in-code defaults (the file made to look absent).
* shaders_g{8,16}.npz — the reference's compute shaders (compiled as C++ by
                     oracle/_ref) on small seeded particle sets: the mass
                     grid of mass.glsl, the gradient texture of the
                     complex..pack chain, and the particles after one
                     update.glsl pass (and after one whole step_fft).

The fixtures are committed so the tests never need the reference.
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
REF = Path(os.environ.get("MOG_REFERENCE") or ROOT.parent / "reference")


def import_reference_main():
    """main.py with moderngl / moderngl_window replaced by empty modules."""
    mgl = types.ModuleType("moderngl")
    mglw = types.ModuleType("moderngl_window")
    mglw.WindowConfig = object
    sys.modules.setdefault("moderngl", mgl)
    sys.modules.setdefault("moderngl_window", mglw)
    sys.path.insert(0, str(REF))
    import main as ref_main  # noqa: E402

    return ref_main


class _FakeBuffer:
    def __init__(self, data):
        self.data = data


class _FakeCtx:
    def buffer(self, data):
        return _FakeBuffer(data)


def transforms(ref_main):
    cases = [(16, 16, 100.0, 0), (3, 8, 100.0, 1), (240, 16, 100.0, 1), (32, 32, 2000.0, 7)]
    out = {}
    for k, g, L, seed in cases:
        orig = ref_main.RandomSE3Sampler

        def seeded(*a, _seed=seed, _orig=orig, **kw):
            kw["seed"] = _seed
            return _orig(*a, **kw)

        ref_main.RandomSE3Sampler = seeded
        try:
            fake = types.SimpleNamespace(n_grids=k, grid_size=g, world_size=L)
            off, rot = ref_main.Simulation.compute_transforms(fake)
        finally:
            ref_main.RandomSE3Sampler = orig
        key = f"k{k}_g{g}_L{int(L)}_s{seed}"
        out[f"{key}_offsets"] = off
        out[f"{key}_rotations"] = rot
    np.savez_compressed(HERE / "transforms.npz", **out)


def greens_kernel(ref_main):
    out = {}
    for g, L in [(8, 100.0), (16, 100.0)]:
        fake = types.SimpleNamespace(grid_size=g, voxel_size=L / g, ctx=_FakeCtx())
        import contextlib
        import io

        with contextlib.redirect_stdout(io.StringIO()):
            ref_main.Simulation.init_greens_kernel(fake)
        k = np.frombuffer(fake.green_kernel_buf.data, dtype=np.float32).reshape(g, g, g, 4)
        out[f"g{g}"] = k
    np.savez_compressed(HERE / "greens_kernel.npz", **out)


def shaders():
    from oracle import ref_harness as rh

    assert rh.available(), "build oracle/_ref first (python -m oracle.ref_build)"
    T = np.load(HERE / "transforms.npz")
    for g, k, n in [(8, 3, 1500), (16, 3, 1000)]:
        L, G, dt, damping = 100.0, 10.0, 1e-3, 0.999
        key = "k3_g8_L100_s1" if g == 8 else None
        rng = np.random.default_rng(100 + g)
        if key is None:
            from mog_solver_b200.transforms import compute_transforms

            off, rot = compute_transforms(k, g, L, seed=5)
        else:
            off, rot = T[f"{key}_offsets"], T[f"{key}_rotations"]
        pos = np.zeros((n, 4), dtype=np.float32)
        half = n // 2
        pos[:half, :3] = rng.normal(L / 2, L / 10, (half, 3))
        pos[half:, :3] = rng.uniform(0, L, (n - half, 3))
        pos[:, :3] = np.mod(pos[:, :3], np.float32(L)).astype(np.float32)
        pos[:, 3] = rng.choice(np.array([1.0, 0.5, 2.0], dtype=np.float32), n)
        vel = np.zeros_like(pos)
        vel[:, :3] = rng.normal(0, 2, (n, 3))
        mass = rh.deposit(pos, off, rot, g, L)
        grad = rh.solve(mass, L, G)
        p1, v1 = rh.update(pos, vel, off, rot, grad, g, L, dt, damping)
        p2, v2, m2 = rh.step(pos, vel, off, rot, g, L, G, dt, damping)
        assert np.array_equal(m2, mass) and np.array_equal(p2, p1) and np.array_equal(v2, v1)
        np.savez_compressed(HERE / f"shaders_g{g}.npz", pos=pos, vel=vel, offsets=off,
                            rotations=rot, mass=mass, grad=grad, pos1=p1, vel1=v1,
                            params=np.array([L, G, dt, damping], dtype=np.float64))


def initial_conditions(ref_main):
    """Simulation.init_particles2 (main.py:312-357) after np.random.seed(s)."""
    out = {}
    for n, L, m, seed in [(1001, 100.0, 0.5, 3), (64, 250.0, 1.0, 0)]:
        bufs = {}

        class _Buf:
            def __init__(self, name):
                self.name = name

            def write(self, data):
                bufs[self.name] = data

        fake = types.SimpleNamespace(num_particles=n, world_size=L, cfg={"particle_mass": m},
                                     pos_buf=_Buf("pos"), vel_buf=_Buf("vel"))
        np.random.seed(seed)
        ref_main.Simulation.init_particles2(fake)
        key = f"n{n}_L{int(L)}_s{seed}"
        out[f"{key}_pos"] = np.frombuffer(bufs["pos"], dtype=np.float32).reshape(n, 4)
        out[f"{key}_vel"] = np.frombuffer(bufs["vel"], dtype=np.float32).reshape(n, 4)
        out[f"{key}_params"] = np.array([n, L, m, seed], dtype=np.float64)
    np.savez_compressed(HERE / "two_galaxies.npz", **out)


def perlin_sampler(ref_main=None):
    """init_particles.glsl (compiled as C++ by oracle/_ref): the reference's
    default call (main.py:280-281: noise 4, contrast 2, seed 12345, sphere)
    and a cube-shaped variant."""
    from oracle import ref_harness as rh

    assert rh.available(), "build oracle/_ref first (python -m oracle.ref_build)"
    out = {}
    for n, L, noise, contrast, seed, m, buf, shape in [(4096, 100.0, 4.0, 2.0, 12345, 1.0, 0.1, 1),
                                                       (3000, 250.0, 2.5, 3.0, 7, 0.25, 0.05, 0)]:
        pos, vel = rh.init_particles(n, L, noise, contrast, seed, m, buf, shape)
        key = f"n{n}_shape{shape}"
        out[f"{key}_pos"] = pos
        out[f"{key}_vel"] = vel
        out[f"{key}_params"] = np.array([n, L, noise, contrast, seed, m, buf, shape], dtype=np.float64)
    np.savez_compressed(HERE / "init_particles.npz", **out)


class _Uniform:
    def __init__(self):
        self.data = None

    def write(self, data):
        self.data = bytes(data)


def camera(ref_main):
    """The matrix uniforms on_render writes (main.py:678-700), per camera."""
    for name in ("BLEND", "SRC_ALPHA", "ONE_MINUS_SRC_ALPHA", "POINTS", "LINES"):
        setattr(ref_main.moderngl, name, 0)
    out = {}
    cases = [(0.0, 0.0, 3.0, 2560 / 1440), (30.0, 20.0, 3.0, 2560 / 1440), (-135.5, 95.0, 1.7, 4 / 3),
             (250.0, -40.0, 6.25, 1.0), (12.0, -89.0, 0.1, 16 / 9)]
    for idx, (rx, ry, dist, aspect) in enumerate(cases):
        uniforms = {"m_view": _Uniform(), "m_proj": _Uniform()}
        ctx = types.SimpleNamespace(clear=lambda *a, **k: None, enable=lambda *a, **k: None,
                                    blend_func=None)
        fake = types.SimpleNamespace(paused=True, ctx=ctx, cam_rot_x=rx, cam_rot_y=ry,
                                     cam_dist=dist, aspect_ratio=aspect, render_prog=uniforms,
                                     show_particles=False, show_grid_debug=False)
        ref_main.Simulation.on_render(fake, 0.0, 0.0)
        out[f"c{idx}_params"] = np.array([rx, ry, dist, aspect], dtype=np.float64)
        out[f"c{idx}_m_view"] = np.frombuffer(uniforms["m_view"].data, np.float32)
        out[f"c{idx}_m_proj"] = np.frombuffer(uniforms["m_proj"].data, np.float32)
    np.savez_compressed(HERE / "camera.npz", **out)


def point_shaders(ref_main=None):
    """render_prog's vertex and fragment shaders (oracle/_ref) on seeded inputs."""
    from oracle import ref_harness as rh
    from mog_solver_b200.render import camera_matrices

    assert rh.available(), "build oracle/_ref first (python -m oracle.ref_build)"
    rng = np.random.default_rng(2024)
    n = 512
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.uniform(-20.0, 120.0, (n, 3))
    pos[:, 3] = 1.0
    vel = np.zeros((n, 4), np.float32)
    vel[:, :3] = rng.normal(0.0, 3.0, (n, 3)) * rng.uniform(0.0, 3.0, (n, 1))
    out = {"pos": pos, "vel": vel}
    for c, cam in enumerate([(0.0, 0.0, 3.0, 2560 / 1440), (30.0, 20.0, 2.0, 4 / 3),
                             (-135.5, 95.0, 1.7, 1.0)]):
        m_view, m_proj = camera_matrices(*cam)
        out[f"cam{c}_m_view"], out[f"cam{c}_m_proj"] = m_view, m_proj
        for s, scale in enumerate((0.13, 2.0)):
            clip, size, v_speed = rh.point_vertex(pos, vel, 100.0, scale, m_view, m_proj)
            out[f"cam{c}_s{s}_params"] = np.array([100.0, scale], np.float32)
            out[f"cam{c}_s{s}_clip"], out[f"cam{c}_s{s}_size"] = clip, size
            out[f"cam{c}_s{s}_v_speed"] = v_speed
    m = 4000
    pc = rng.uniform(-0.1, 1.1, (m, 2)).astype(np.float32)
    vs = rng.uniform(0.0, 1.0, m).astype(np.float32)
    vs[:8] = [0.0, 0.3, 0.7, 1.0, 0.29999998, 0.70000005, 0.5, 0.9]
    colour, kept = rh.point_fragment(pc, vs)
    out.update(frag_point_coord=pc, frag_v_speed=vs, frag_colour=colour, frag_kept=kept)
    np.savez_compressed(HERE / "point_shaders.npz", **out)


def config(ref_main):
    """The reference's load_config output, with and without its config.yaml."""
    import json
    from unittest import mock

    fake = types.SimpleNamespace()
    with_file = ref_main.Simulation.load_config(fake)
    with mock.patch.object(ref_main.Path, "exists", lambda self: False):
        defaults = ref_main.Simulation.load_config(fake)
    (HERE / "config.json").write_text(json.dumps({"config_yaml": with_file, "defaults": defaults},
                                                 indent=1, sort_keys=True) + "\n")


PARTS = {"transforms": transforms, "greens_kernel": greens_kernel, "shaders": None,
         "two_galaxies": initial_conditions, "init_particles": perlin_sampler, "camera": camera,
         "point_shaders": point_shaders, "config": config}


def main():
    """python tests/golden/make_golden.py [part ...]  (default: every part)"""
    ref_main = import_reference_main()
    names = sys.argv[1:] or list(PARTS)
    for name in names:
        if name == "shaders":
            shaders()
        else:
            PARTS[name](ref_main)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
