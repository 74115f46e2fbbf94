"""The two-galaxy initialiser's formulas given its uniforms — TEST
INFRASTRUCTURE ONLY (the checker of mog_init_two_galaxies and its host twin).

Restates Simulation.init_particles2 (main.py:312-357) in NumPy FP64 with the
three uniforms of each particle passed in, instead of drawn from NumPy's
global generator:
  r = exponential(0.08) * L = -ln(1 - u0) * 0.08 L       (main.py:326)
  theta = uniform(0, 2 pi) = 2 pi u1                       (main.py:327)
  phi = arccos(uniform(-1, 1)) = arccos(-1 + 2 u2)         (main.py:328)
  position and spin velocity as main.py:330-355.
"""
from __future__ import annotations

import numpy as np

OFFSETS = (np.array([-0.2, 0.0, 0.0]), np.array([0.2, 0.0, 0.0]))      # main.py:320-321
BULK = (np.array([0.3, 0.1, 0.0]), np.array([-0.3, -0.1, 0.0]))
AXES = (np.array([0.3, 0.7, 0.5]), np.array([-0.5, 0.2, 0.8]))          # main.py:341-343


def two_galaxies_from_uniforms(U: np.ndarray, world: float, mass: float):
    """(pos, vel) float32 (n, 4) records for uniforms U (n, 3) float64."""
    n = U.shape[0]
    per = n // 2
    pos = np.zeros((n, 4), dtype=np.float32)
    vel = np.zeros((n, 4), dtype=np.float32)
    centre = world / 2.0
    for b in range(2):
        lo, hi = b * per, (b + 1) * per
        u = U[lo:hi]
        r = -np.log(1.0 - u[:, 0]) * 0.08 * world
        theta = 2.0 * np.pi * u[:, 1]
        phi = np.arccos(-1.0 + 2.0 * u[:, 2])
        x = r * np.sin(phi) * np.cos(theta)
        y = r * np.sin(phi) * np.sin(theta)
        z = r * np.cos(phi)
        for j, c in enumerate((x, y, z)):
            pos[lo:hi, j] = centre + OFFSETS[b][j] * world + c
        pos[lo:hi, 3] = mass
        axis = AXES[b] / np.linalg.norm(AXES[b])
        v_circ = 0.3 * np.sqrt(r / world + 0.01)
        d = np.cross(axis, np.stack([x, y, z], axis=1))
        d = d / (np.linalg.norm(d, axis=1, keepdims=True) + 1e-10)
        for j in range(3):
            vel[lo:hi, j] = v_circ * d[:, j] + BULK[b][j]
    return pos, vel
