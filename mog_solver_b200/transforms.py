"""Per-grid random rigid transforms (rotation + sub-voxel offset).

Restates ``RandomSE3Sampler`` (main.py:9-62) and the GPU packing of
``Simulation.compute_transforms`` (main.py:157-172):

* from one ``numpy.random.default_rng(seed)`` stream, draw ``u ~ U[0,1)^(k x 3)``
  first and then the offsets ``~ U[0, voxel)^(k x 3)`` (main.py:18-28);
* Shoemake's uniform quaternion (w, x, y, z) = (sqrt(1-u0) sin 2pi u1,
  sqrt(1-u0) cos 2pi u1, sqrt(u0) sin 2pi u2, sqrt(u0) cos 2pi u2), cast to
  float32 (main.py:21-26);
* the rotation matrix M of that quaternion evaluated in float32 with the
  same expression order as main.py:37-62, so the packed floats match the
  reference bit for bit;
* packing: ``rotations[i, 4j:4j+3] = M[j, :]`` (row j of M) and
  ``offsets[i, 0:3] = offset`` (main.py:166-170).  The shaders read the three
  float4 rows as the columns of their mat3, i.e. they rotate by M^T
  (mass.glsl:20-25, 43) and rotate forces back by M (update.glsl:77).

The same draw order and formulas are required for the transforms to be the
reference's own for a given seed; the code is this package's.
"""
from __future__ import annotations

import numpy as np


def _quat_to_matrix_f32(q: np.ndarray) -> np.ndarray:
    """Rotation matrices (k, 3, 3) float32 of quaternions q (k, 4) float32."""
    w, x, y, z = (q[:, i] for i in range(4))
    two = np.float32(2)
    one = np.float32(1)
    m = np.empty((q.shape[0], 3, 3), dtype=np.float32)
    m[:, 0, 0] = one - two * y * y - two * z * z
    m[:, 0, 1] = two * x * y - two * z * w
    m[:, 0, 2] = two * x * z + two * y * w
    m[:, 1, 0] = two * x * y + two * z * w
    m[:, 1, 1] = one - two * x * x - two * z * z
    m[:, 1, 2] = two * y * z - two * x * w
    m[:, 2, 0] = two * x * z - two * y * w
    m[:, 2, 1] = two * y * z + two * x * w
    m[:, 2, 2] = one - two * x * x - two * y * y
    return m


class RandomSE3Sampler:
    """Same constructor and methods as the reference's sampler (main.py:9-62).

    ``generate()`` returns ``(rotations, offsets)`` where ``rotations`` is
    (k, 3, 4) float32 laid out like the reference's ``_quat_to_matrix``
    output (``rotations[i][r][c] = M_i[c][r]`` for c < 3, last column 0)
    and ``offsets`` is (k, 3) float32.
    """

    def __init__(self, grid_size, world_size, n_grids, seed=None):
        self.grid_size = grid_size
        self.world_size = world_size
        self.voxel_size = world_size / grid_size
        self.n_grids = n_grids
        self.seed = seed

    def quaternions_and_offsets(self) -> tuple[np.ndarray, np.ndarray]:
        rng = np.random.default_rng(self.seed)
        n = self.n_grids
        u = rng.uniform(0, 1, (n, 3))
        a = np.sqrt(1 - u[:, 0])
        b = np.sqrt(u[:, 0])
        quats = np.stack(
            [a * np.sin(2 * np.pi * u[:, 1]), a * np.cos(2 * np.pi * u[:, 1]),
             b * np.sin(2 * np.pi * u[:, 2]), b * np.cos(2 * np.pi * u[:, 2])],
            axis=1,
        ).astype(np.float32)
        offsets = rng.uniform(0, self.voxel_size, (n, 3)).astype(np.float32)
        return quats, offsets

    def generate(self) -> tuple[np.ndarray, np.ndarray]:
        quats, offsets = self.quaternions_and_offsets()
        m = _quat_to_matrix_f32(quats)
        rot = np.zeros((self.n_grids, 3, 4), dtype=np.float32)
        rot[:, :, :3] = np.transpose(m, (0, 2, 1))
        return rot, offsets

    def get_transforms(self, verbose=False):
        if verbose:
            print(f"  Generating {self.n_grids} random SE(3) transforms...")
        return self.generate()

    def _quat_to_matrix(self, q):
        return self.generate_one(q)

    @staticmethod
    def generate_one(q) -> np.ndarray:
        m = _quat_to_matrix_f32(np.asarray(q, dtype=np.float32).reshape(1, 4))[0]
        out = np.zeros((3, 4), dtype=np.float32)
        out[:, :3] = m.T
        return out


def compute_transforms(n_grids: int, grid_size: int, world_size: float,
                       seed: int | None = None) -> tuple[np.ndarray, np.ndarray]:
    """(offsets (k, 4) float32, rotations (k, 12) float32) packed for the GPU.

    Note the return order (offsets, rotations), as in main.py:172.
    """
    sampler = RandomSE3Sampler(grid_size=grid_size, world_size=world_size, n_grids=n_grids,
                               seed=seed)
    rot_mats, offs = sampler.get_transforms()
    offsets = np.zeros((n_grids, 4), dtype=np.float32)
    rotations = np.zeros((n_grids, 12), dtype=np.float32)
    offsets[:, 0:3] = offs
    for j in range(3):
        rotations[:, 4 * j:4 * j + 3] = rot_mats[:, :, j]
    return offsets, rotations


def rotation_matrices(rotations: np.ndarray) -> np.ndarray:
    """Unpack (k, 12) GPU rotations to (k, 3, 3) matrices M (rows j)."""
    r = np.asarray(rotations, dtype=np.float32).reshape(-1, 3, 4)
    return r[:, :, :3].copy()
