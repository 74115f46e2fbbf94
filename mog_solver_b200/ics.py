"""Seeded synthetic particle sets (host-side numpy, float32 (N, 4) records).

The reference initialises particles with a GPU Perlin/fBm rejection sampler
(init_particles.glsl, driven from main.py:280-310) or an unseeded two-galaxy
numpy routine (main.py:312-357).  The benchmark workloads of this library
use their own seeded distributions instead:

* ``uniform_cube``    positions U[0, L)^3, zero velocity;
* ``two_disks``       two exponential disks (scale radius R_d, sech^2 scale
                      height z0) with circular velocities from the enclosed
                      mass, centres ``sep`` apart along x, approaching with
                      relative speed ``v_rel``;
* ``plummer``         a Plummer sphere of scale radius a, at rest;
* ``clumps``          a Gaussian mixture (log-uniform widths) plus a uniform
                      background fraction;
* ``reference_two_galaxies`` the reference's own two-galaxy routine,
                      seeded (bit-identical to it after np.random.seed);
* ``perlin_host``     the reference's GPU Perlin/fBm rejection sampler
                      (init_particles.glsl) on the host through libmog;
                      ``Simulation.init_particles("perlin")`` runs it on the GPU.

Every record is (x, y, z, m) for positions and (vx, vy, vz, 0) for
velocities, the std430 vec4 layout of the reference's buffers
(main.py:192-193, update.glsl:3-4).  Masses are ``total_mass / N``.
"""
from __future__ import annotations

import numpy as np


def _records(xyz: np.ndarray, m: float, vel: np.ndarray | None = None):
    n = xyz.shape[0]
    pos = np.empty((n, 4), dtype=np.float32)
    pos[:, :3] = xyz
    pos[:, 3] = np.float32(m)
    v = np.zeros((n, 4), dtype=np.float32)
    if vel is not None:
        v[:, :3] = vel
    return pos, v


def wrap(xyz: np.ndarray, world: float) -> np.ndarray:
    return np.mod(xyz, world).astype(np.float32)


def uniform_cube(n: int, world: float = 100.0, seed: int = 0, total_mass: float = 1.0):
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(0.0, world, (n, 3)).astype(np.float32)
    xyz = np.minimum(xyz, np.nextafter(np.float32(world), np.float32(0)))
    return _records(xyz, total_mass / n if n else 0.0)


def _exp_disk(rng, n: int, r_d: float, z0: float, r_max: float):
    # Surface density ~ exp(-R/R_d): R ~ Gamma(2, R_d); truncated at r_max.
    r = rng.gamma(2.0, r_d, size=n)
    bad = r > r_max
    while bad.any():
        r[bad] = rng.gamma(2.0, r_d, size=int(bad.sum()))
        bad = r > r_max
    phi = rng.uniform(0.0, 2 * np.pi, n)
    # sech^2(z/z0) profile: CDF (1 + tanh(z/z0)) / 2
    u = rng.uniform(1e-7, 1 - 1e-7, n)
    z = z0 * np.arctanh(2 * u - 1)
    z = np.clip(z, -10 * z0, 10 * z0)
    return r, phi, z


def two_disks(n: int, world: float = 100.0, seed: int = 1, r_d: float = 8.0, z0: float = 0.5,
              sep: float = 40.0, v_rel: float = 5.0, g_eff: float = 1.0, total_mass: float = 1.0,
              r_max: float = 18.0):
    """Two colliding exponential disks.

    ``g_eff`` is the gravitational constant in the units of the solver's
    acceleration (for the reference's normalisation: G * h^3 / 2, see
    ``Simulation.effective_g``); circular speeds are sqrt(g_eff M(<R) / R)
    with M(<R) the disk mass inside cylindrical radius R.
    """
    rng = np.random.default_rng(seed)
    n_a = n // 2
    n_b = n - n_a
    c = world / 2.0
    centres = [np.array([c - sep / 2, c, c]), np.array([c + sep / 2, c, c])]
    bulk = [np.array([v_rel / 2, 0.0, 0.0]), np.array([-v_rel / 2, 0.0, 0.0])]
    # disk normals: the second disk is tilted 30 degrees about x
    t = np.radians(30.0)
    frames = [np.eye(3), np.array([[1, 0, 0], [0, np.cos(t), -np.sin(t)], [0, np.sin(t), np.cos(t)]])]
    m_disk = [total_mass * n_a / n, total_mass * n_b / n]
    xs, vs = [], []
    for count, centre, vb, frame, md in zip((n_a, n_b), centres, bulk, frames, m_disk):
        r, phi, z = _exp_disk(rng, count, r_d, z0, r_max)
        order = np.argsort(r)
        enclosed = np.empty(count)
        enclosed[order] = (np.arange(count) + 1) * (md / count)
        vc = np.sqrt(g_eff * enclosed / np.maximum(r, 1e-3))
        local = np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)
        lv = np.stack([-vc * np.sin(phi), vc * np.cos(phi), np.zeros(count)], axis=1)
        xs.append(local @ frame.T + centre)
        vs.append(lv @ frame.T + vb)
    xyz = wrap(np.concatenate(xs), world)
    vel = np.concatenate(vs).astype(np.float32)
    return _records(xyz, total_mass / n, vel)


def plummer(n: int, world: float = 100.0, seed: int = 0, a: float = 5.0,
            total_mass: float = 1.0, r_max: float | None = None):
    rng = np.random.default_rng(seed)
    r_max = world * 0.45 if r_max is None else r_max
    out = np.empty((0, 3))
    while out.shape[0] < n:
        m = n - out.shape[0]
        u = rng.uniform(1e-9, 1.0, m)
        r = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        d = rng.normal(size=(m, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        pts = d * r[:, None]
        out = np.concatenate([out, pts[r <= r_max]])
    xyz = wrap(out[:n] + world / 2.0, world)
    return _records(xyz, total_mass / n)


def rotated_disk_pair(n: int, world: float = 100.0, seed: int = 500):
    """Two exponential disks (two_disks) with a scale radius drawn from
    [5, 11], a sech^2 height log-uniform in [0.25, 1] and centres 25 to 55
    apart, the whole set turned by a random rotation about the box centre
    (periodic wrap).  Disk-like training data for the learned correction,
    drawn around (never at) the benchmark's parameters."""
    rng = np.random.default_rng(seed)
    pos, vel = two_disks(n, world, seed=seed, r_d=float(rng.uniform(5.0, 11.0)),
                         z0=float(np.exp(rng.uniform(np.log(0.25), np.log(1.0)))),
                         sep=float(rng.uniform(25.0, 55.0)))
    q = rng.normal(size=4)
    w, x, y, z = q / np.linalg.norm(q)
    R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    c = pos[:, :3].astype(np.float64) - world / 2.0
    pos[:, :3] = wrap(c @ R.T + world / 2.0, world)
    vel[:, :3] = (vel[:, :3].astype(np.float64) @ R.T).astype(np.float32)
    return pos, vel


def clumps(n: int, world: float = 100.0, seed: int = 100, n_clumps: int = 20,
           sigma_range: tuple[float, float] = (1.0, 8.0), background: float = 0.1,
           total_mass: float = 1.0):
    rng = np.random.default_rng(seed)
    n_bg = int(round(background * n))
    n_cl = n - n_bg
    centres = rng.uniform(0.15 * world, 0.85 * world, (n_clumps, 3))
    sig = np.exp(rng.uniform(np.log(sigma_range[0]), np.log(sigma_range[1]), n_clumps))
    which = rng.integers(0, n_clumps, n_cl)
    pts = centres[which] + rng.normal(size=(n_cl, 3)) * sig[which, None]
    bg = rng.uniform(0.0, world, (n_bg, 3))
    xyz = wrap(np.concatenate([pts, bg]), world)
    xyz = xyz[rng.permutation(n)]
    return _records(xyz, total_mass / n)


def reference_two_galaxies(n: int, world: float = 100.0, particle_mass: float = 1.0,
                           seed: int = 0):
    """The reference's numpy two-galaxy initialiser (main.py:312-357,
    ``Simulation.init_particles2``) with its global ``np.random`` made an
    explicit legacy ``RandomState(seed)``: the same draws in the same order,
    so ``np.random.seed(seed)`` followed by the reference's routine gives the
    same float32 buffers bit for bit.

    Two spherical exponential blobs (scale 0.08 L) at ±0.2 L along x with
    bulk velocities ±(0.3, 0.1, 0), each spinning about its own axis with
    v = 0.3 sqrt(r / L + 0.01).  Masses are ``particle_mass`` each (the
    reference's config value); with odd n the last record stays zero, as in
    the reference.
    """
    rs = np.random.RandomState(seed)
    pos = np.zeros((n, 4), dtype=np.float32)
    vel = np.zeros((n, 4), dtype=np.float32)
    centre = world / 2.0
    per = n // 2
    blobs = ((np.array([-0.2, 0.0, 0.0]), np.array([0.3, 0.1, 0.0]), np.array([0.3, 0.7, 0.5])),
             (np.array([0.2, 0.0, 0.0]), np.array([-0.3, -0.1, 0.0]), np.array([-0.5, 0.2, 0.8])))
    for i, (offset, v_bulk, axis) in enumerate(blobs):
        lo, hi = i * per, (i + 1) * per
        r = rs.exponential(scale=0.08, size=per) * world
        theta = rs.uniform(0, 2 * np.pi, per)
        phi = np.arccos(rs.uniform(-1, 1, per))
        x = r * np.sin(phi) * np.cos(theta)
        y = r * np.sin(phi) * np.sin(theta)
        z = r * np.cos(phi)
        for j, c in enumerate((x, y, z)):
            pos[lo:hi, j] = centre + offset[j] * world + c
        pos[lo:hi, 3] = particle_mass
        axis = axis / np.linalg.norm(axis)
        v_circ = 0.3 * np.sqrt(r / world + 0.01)
        v_dir = np.cross(axis, np.stack([x, y, z], axis=1))
        v_dir = v_dir / (np.linalg.norm(v_dir, axis=1, keepdims=True) + 1e-10)
        for j in range(3):
            vel[lo:hi, j] = v_circ * v_dir[:, j] + v_bulk[j]
    return pos, vel


def two_galaxies_host(n: int, world: float = 100.0, particle_mass: float = 1.0, seed: int = 0):
    """The two-galaxy initialiser of mog_init_two_galaxies evaluated on the
    host (mog_init_two_galaxies_host; no GPU needed): the reference's
    formulas (main.py:312-357) with counter-based draws keyed by ``seed``."""
    import ctypes

    from . import _lib

    pos = np.zeros((n, 4), dtype=np.float32)
    vel = np.zeros((n, 4), dtype=np.float32)
    _lib.check(_lib.lib().mog_init_two_galaxies_host(
        pos.ctypes.data_as(ctypes.c_void_p), vel.ctypes.data_as(ctypes.c_void_p), int(n),
        float(world), float(particle_mass), int(seed) & 0xFFFFFFFFFFFFFFFF),
        "mog_init_two_galaxies_host")
    return pos, vel


def two_galaxies_uniforms(n: int, seed: int = 0) -> np.ndarray:
    """The (n, 3) uniforms that mog_init_two_galaxies draws (SplitMix64 of a
    seed-derived key plus 4 i + j, top 53 bits), in NumPy."""
    M = np.uint64(0xFFFFFFFFFFFFFFFF)

    def mix(z):
        with np.errstate(over="ignore"):
            z = (z + np.uint64(0x9E3779B97F4A7C15)) & M
            z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M
            z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M
            return z ^ (z >> np.uint64(31))

    key = mix(np.array([int(seed) & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64))[0]
    i = np.arange(n, dtype=np.uint64)[:, None]
    j = np.arange(3, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        ctr = (key + (i << np.uint64(2)) + j) & M
    return (mix(ctr) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def perlin_args(n: int, world: float, mass: float, spawn_buffer: float = 0.1, seed: int = 12345,
                noise_scale: float = 4.0, density_contrast: float = 2.0, shape: str = "sphere"):
    """Arguments of mog_init_particles after the buffers (stream excluded).
    Defaults: the reference's call, init_particles_gpu(noise_scale=4.0,
    density_contrast=2.0, seed=12345) with spawnShape 1 (main.py:280-305)."""
    if shape not in ("sphere", "cube"):
        raise ValueError("shape must be 'sphere' or 'cube'")
    return (int(n), float(world), float(noise_scale), float(density_contrast),
            int(seed) & 0xFFFFFFFF, float(mass), float(spawn_buffer), 1 if shape == "sphere" else 0)


def perlin_host(n: int, world: float = 100.0, mass: float = 1.0, spawn_buffer: float = 0.1,
                seed: int = 12345, noise_scale: float = 4.0, density_contrast: float = 2.0,
                shape: str = "sphere"):
    """init_particles.glsl on the host (mog_init_particles_host; no GPU needed)."""
    import ctypes

    from . import _lib

    pos = np.zeros((n, 4), dtype=np.float32)
    vel = np.zeros((n, 4), dtype=np.float32)
    args = perlin_args(n, world, mass, spawn_buffer, seed, noise_scale, density_contrast, shape)
    _lib.check(_lib.lib().mog_init_particles_host(pos.ctypes.data_as(ctypes.c_void_p),
                                                  vel.ctypes.data_as(ctypes.c_void_p), *args),
               "mog_init_particles_host")
    return pos, vel
