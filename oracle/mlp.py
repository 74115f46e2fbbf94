"""FP64 NumPy oracle of the learned correction — TEST INFRASTRUCTURE ONLY.

* ``features``: the per-particle statistics of a k-grid ensemble, computed
  from the oracle's cell indices and an FP64 copy of the world-frame force
  grid and mass grid (same definitions as learned.cu).
* ``forward`` / ``backward``: the 12 -> 64 -> 64 -> 3 GELU (tanh form)
  network and the gradient of the mean squared error, in FP64.

Parameter layout: W1[64][12] b1[64] W2[64][64] b2[64] W3[3][64] b3[3].
"""
from __future__ import annotations

import numpy as np

N_IN, N_H, N_OUT = 12, 64, 3
SIZES = [("W1", (N_H, N_IN)), ("b1", (N_H,)), ("W2", (N_H, N_H)), ("b2", (N_H,)),
         ("W3", (N_OUT, N_H)), ("b3", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)
C = 0.7978845608028654


def unpack(params: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + n], dtype=np.float64).reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def init(seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    d = {"W1": rng.normal(0, 1 / np.sqrt(N_IN), (N_H, N_IN)), "b1": np.zeros(N_H),
         "W2": rng.normal(0, 1 / np.sqrt(N_H), (N_H, N_H)), "b2": np.zeros(N_H),
         "W3": rng.normal(0, 0.1 / np.sqrt(N_H), (N_OUT, N_H)), "b3": np.zeros(N_OUT)}
    return pack(d)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(C * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    t = np.tanh(C * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * C * (1 + 3 * 0.044715 * x * x)


def forward(params, x):
    p = unpack(params)
    a1 = x @ p["W1"].T + p["b1"]
    h1 = gelu(a1)
    a2 = h1 @ p["W2"].T + p["b2"]
    h2 = gelu(a2)
    y = h2 @ p["W3"].T + p["b3"]
    return y, (a1, h1, a2, h2)


def loss_and_grad(params, x, t):
    """Mean over samples of the summed squared error, and its gradient."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    p = unpack(params)
    y, (a1, h1, a2, h2) = forward(params, x)
    B = x.shape[0]
    d = y - t
    loss = float((d * d).sum() / B)
    dy = 2.0 * d / B
    g = {"W3": dy.T @ h2, "b3": dy.sum(0)}
    da2 = (dy @ p["W3"]) * gelu_grad(a2)
    g["W2"] = da2.T @ h1
    g["b2"] = da2.sum(0)
    da1 = (da2 @ p["W2"]) * gelu_grad(a1)
    g["W1"] = da1.T @ x
    g["b1"] = da1.sum(0)
    return loss, pack(g)


def features(cells, fgrid_world, mass_values, t, rot12, h, norm):
    """Per-particle features (n, 12), plain mean force (n, 3) and the
    least-squares correction (n, 3), FP64.

    cells: (n, k) cell indices; fgrid_world: (k, g^3, 3) world-frame forces;
    mass_values: (k, g^3) cell masses; t: (n, k, 3) scaled grid coordinates
    (cell = floor(t)); rot12: (k, 12) packed rotations; h: voxel size;
    norm: dict with force_scale, rho_ref, mu (12), inv_sigma (12).
    Definitions follow features_kernel in learned.cu.
    """
    k = cells.shape[1]
    gi = np.arange(k)[None, :]
    F = fgrid_world[gi, cells]                        # (n, k, 3)
    mean = F.mean(axis=1)
    var = np.maximum((F * F).mean(axis=1) - mean * mean, 0.0)
    M = np.asarray(rot12, dtype=np.float32).reshape(-1, 3, 4)[:, :, :3].astype(np.float64)
    dg = (t - np.floor(t) - 0.5) * h
    d = np.einsum("kab,nkb->nka", M, dg)              # world-frame offsets
    dbar = d.mean(axis=1)
    ridge = 1e-3 * h * h
    Cdd = np.einsum("nki,nkj->nij", d, d) / k - dbar[:, :, None] * dbar[:, None, :] + ridge * np.eye(3)
    CFd = np.einsum("nki,nkj->nij", F, d) / k - mean[:, :, None] * dbar[:, None, :]
    w = np.linalg.solve(Cdd, dbar[:, :, None])[:, :, 0]
    corr = -np.einsum("nij,nj->ni", CFd, w)
    rho = mass_values[gi, cells].mean(axis=1)
    s = norm["force_scale"]
    f = np.empty((cells.shape[0], 12))
    f[:, 0:3] = mean / s
    f[:, 3:6] = corr / s
    f[:, 6:9] = np.sqrt(var) / s
    f[:, 9] = np.log1p(rho / norm["rho_ref"])
    f[:, 10] = np.linalg.norm(mean, axis=1) / s
    f[:, 11] = np.sqrt(np.maximum(np.trace(Cdd, axis1=1, axis2=2) - 3 * ridge, 0.0)) / h
    return (f - norm["mu"]) * norm["inv_sigma"], mean, corr
