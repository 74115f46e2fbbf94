"""NumPy oracles of the MOG pipeline — TEST INFRASTRUCTURE ONLY.

* FP64 ideal pipeline: the reference's mathematics (main.py:592-669) with
  exact FFTs — forward transform of the cell masses, DC removed
  (fourier.glsl:16-18), phi^ = rho^ * (-2 pi G / k^2) where the reference's
  FP32 k^2 exceeds 1e-4 (greens.glsl:17-47), d^_j = i k_j phi^
  (greens.glsl:23, 53-60), F_j = Re(IFFT(d^_j)) / g^3 (pack.glsl:20-27),
  gather at each particle's NGP cell, rotate back by M and average
  (update.glsl:67-81).
* FP32 transcription of the shader chain including its quirks
  (uint x1000 mass, per-stage radix-2 passes with the |x| < 1e-6 flushes
  and twiddle snapping of fft_batched.glsl:19-34, 123-126).
* FP64 direct-sum yardstick: minimum-image Newtonian field scaled to the
  solver's units (G h^3 / 2).
"""
from __future__ import annotations

import numpy as np

TWO_PI_F32 = np.float32(2.0) * np.float32(3.14159265359)


def shift(g: int) -> np.ndarray:
    i = np.arange(g)
    return np.where(i <= g // 2, i, i - g)


def wavenumbers(g: int, world: float) -> np.ndarray:
    return shift(g) * (2.0 * np.pi / float(np.float32(world)))


def keep_mask(g: int, world: float) -> np.ndarray:
    """Bins the reference keeps: FP32 k^2 > 1e-4 (greens.glsl:17-21, 39, 45)."""
    step = np.float32(TWO_PI_F32 / np.float32(world))
    k = (shift(g).astype(np.float32) * step).astype(np.float32)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    k2 = (kx * kx + ky * ky) + kz * kz
    return k2 > np.float32(1e-4)


def green_fp64(g: int, world: float, G: float, softening: float = 0.0) -> np.ndarray:
    """-2 pi G / k^2 on [kz][ky][kx] (greens.glsl:39-47), or with softening a
    (in voxels) the variant commented out in greens.glsl:63-115,
    -4 pi G exp(-k^2 a^2) / k^2; zero where the reference drops the bin."""
    k = wavenumbers(g, world)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    out = np.zeros((g, g, g))
    keep = keep_mask(g, world)
    Gf = float(np.float32(G))
    if softening > 0:
        a = float(np.float32(softening)) * float(np.float32(world)) / g
        out[keep] = -4.0 * np.pi * Gf * np.exp(-k2[keep] * a * a) / k2[keep]
    else:
        out[keep] = -2.0 * np.pi * Gf / k2[keep]
    return out


def forces_grid_fp64(rho: np.ndarray, G: float, world: float, softening: float = 0.0) -> np.ndarray:
    """Grid-frame forces (k, g, g, g, 3) in FP64 from cell masses (k, g, g, g)."""
    rho = np.asarray(rho, dtype=np.float64)
    g = rho.shape[-1]
    k = wavenumbers(g, world)
    rho_hat = np.fft.fftn(rho, axes=(1, 2, 3))
    phi_hat = rho_hat * green_fp64(g, world, G, softening)[None]
    out = np.empty(rho.shape + (3,))
    # axis 3 is x, 2 is y, 1 is z ([z][y][x] layout, x fastest)
    shapes = {0: (1, 1, 1, g), 1: (1, 1, g, 1), 2: (1, g, 1, 1)}
    for comp in range(3):
        kj = k.reshape(shapes[comp])
        out[..., comp] = np.real(np.fft.ifftn(1j * kj * phi_hat, axes=(1, 2, 3)))
    return out


def rotations_fp64(rot12: np.ndarray) -> np.ndarray:
    r = np.asarray(rot12, dtype=np.float32).reshape(-1, 3, 4)
    return r[:, :, :3].astype(np.float64)


def gather_fp64(cells: np.ndarray, fgrid: np.ndarray, rot12: np.ndarray,
                chunk: int = 65536) -> np.ndarray:
    """Ensemble-averaged world-frame force (n, 3) in FP64.

    cells: (n, k) cell indices; fgrid: (k, g, g, g, 3) grid-frame forces.
    """
    k = fgrid.shape[0]
    flat = fgrid.reshape(k, -1, 3)
    M = rotations_fp64(rot12)
    n = cells.shape[0]
    out = np.empty((n, 3))
    gi = np.arange(k)[None, :]
    for a in range(0, n, chunk):
        c = cells[a:a + chunk].astype(np.int64)
        F = flat[gi, c]                      # (m, k, 3)
        W = np.einsum("kab,mkb->mka", M, F)  # M_i F_i
        out[a:a + chunk] = W.mean(axis=1)
    return out


def relative_l2(a: np.ndarray, b: np.ndarray) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


# ---------------------------------------------------------------------------
# FP32 transcription of the shader chain (the reference's CPU-side math).

def _bitrev(n_bits: int, size: int) -> np.ndarray:
    idx = np.arange(size)
    r = np.zeros(size, dtype=np.int64)
    for b in range(n_bits):
        r = (r << 1) | ((idx >> b) & 1)
    return r


def _twiddle_f32(kk: np.ndarray, stage_size: int, direction: int) -> tuple[np.ndarray, np.ndarray]:
    """compute_twiddle of fft_batched.glsl:19-34 in float32."""
    pi2 = TWO_PI_F32
    phase = (np.float32(-direction) * pi2 * kk.astype(np.float32)) / np.float32(stage_size)
    c = np.cos(phase.astype(np.float32)).astype(np.float32)
    s = np.sin(phase.astype(np.float32)).astype(np.float32)
    c = np.where(np.abs(c) < np.float32(1e-6), np.float32(0), c)
    s = np.where(np.abs(s) < np.float32(1e-6), np.float32(0), s)
    c = np.where(kk == 0, np.float32(1), c)
    s = np.where(kk == 0, np.float32(0), s)
    half = stage_size // 2
    c = np.where(kk == half, np.float32(-1), c)
    s = np.where(kk == half, np.float32(0), s)
    return c.astype(np.float32), s.astype(np.float32)


def fft_axis_f32(re: np.ndarray, im: np.ndarray, axis: int, direction: int):
    """One run_fft_3d_batched axis (main.py:573-588): bit reversal, then
    log2 g butterfly stages with the shader's flushes."""
    g = re.shape[axis]
    n_bits = int(np.log2(g))
    rev = _bitrev(n_bits, g)
    re = np.take(re, np.argsort(rev), axis=axis)
    im = np.take(im, np.argsort(rev), axis=axis)
    for stage in range(1, n_bits + 1):
        size = 1 << stage
        half = size >> 1
        t = np.arange(g // 2)
        i1 = (t // half) * size + (t % half)
        i2 = i1 + half
        kk = t % half
        c, s = _twiddle_f32(kk, size, direction)
        shape = [1] * re.ndim
        shape[axis] = g // 2
        c = c.reshape(shape)
        s = s.reshape(shape)
        pr, pi = np.take(re, i1, axis=axis), np.take(im, i1, axis=axis)
        qr, qi = np.take(re, i2, axis=axis), np.take(im, i2, axis=axis)
        tr = (qr * c - qi * s).astype(np.float32)
        ti = (qr * s + qi * c).astype(np.float32)
        tr = np.where(np.abs(tr) < np.float32(1e-6), np.float32(0), tr)
        ti = np.where(np.abs(ti) < np.float32(1e-6), np.float32(0), ti)
        nre = np.empty_like(re)
        nim = np.empty_like(im)
        idx1 = [slice(None)] * re.ndim
        idx2 = [slice(None)] * re.ndim
        idx1[axis] = i1
        idx2[axis] = i2
        nre[tuple(idx1)] = pr + tr
        nim[tuple(idx1)] = pi + ti
        nre[tuple(idx2)] = pr - tr
        nim[tuple(idx2)] = pi - ti
        re, im = nre, nim
    return re, im


def fft3_f32(re, im, direction: int):
    # axes 0,1,2 of the shader are x, y, z -> array axes 3, 2, 1
    for ax in (3, 2, 1):
        re, im = fft_axis_f32(re, im, ax, direction)
    return re, im


def texture_aliasing(g: int) -> bool:
    """True when run_fft_3d_batched's 3 (log2 g + 1) passes are odd, so the z
    inverse transform overwrites the x result (main.py:564-590, 638-646)."""
    return (3 * (int(np.log2(g)) + 1)) % 2 == 1


def forces_grid_f32(mass_u32: np.ndarray, G: float, world: float,
                    aliasing: bool = True) -> np.ndarray:
    """Shader chain in FP32 from a u32 x1000 mass grid -> (k, g, g, g, 4).

    With ``aliasing`` (the reference's behaviour) the x component is the
    z-gradient wherever ``texture_aliasing(g)``."""
    g = mass_u32.shape[-1]
    re = (mass_u32.astype(np.float32) / np.float32(1000.0)).astype(np.float32)  # complex.glsl:23
    im = np.zeros_like(re)
    re, im = fft3_f32(re, im, 1)
    re[:, 0, 0, 0] = 0
    im[:, 0, 0, 0] = 0                                                      # fourier.glsl
    step = np.float32(TWO_PI_F32 / np.float32(world))
    kv = (shift(g).astype(np.float32) * step).astype(np.float32)
    kz, ky, kx = np.meshgrid(kv, kv, kv, indexing="ij")
    k2 = ((kx * kx + ky * ky) + kz * kz).astype(np.float32)
    geo = np.float32(-2.0) * np.float32(3.14159265359)
    fac = np.where(k2 > np.float32(1e-4), (geo * np.float32(G)) / np.where(k2 > 0, k2, 1), 0)
    fac = fac.astype(np.float32)
    pr = np.where(k2 > np.float32(1e-4), re * fac, 0).astype(np.float32)
    pi = np.where(k2 > np.float32(1e-4), im * fac, 0).astype(np.float32)
    out = np.empty(mass_u32.shape + (4,), dtype=np.float32)
    scale = np.float32(1.0) / np.float32(g * g * g)
    for comp, kk in enumerate((kx, ky, kz)):
        gr = (-pi * kk).astype(np.float32)                                  # mult_ik
        gi = (pr * kk).astype(np.float32)
        rr, _ = fft3_f32(gr, gi, -1)
        out[..., comp] = rr * scale
    if aliasing and texture_aliasing(g):
        out[..., 0] = out[..., 2]
    f = out[..., :3]
    out[..., 3] = np.sqrt((f[..., 0] * f[..., 0] + f[..., 1] * f[..., 1]) + f[..., 2] * f[..., 2])
    return out


# ---------------------------------------------------------------------------
# FP64 direct-sum yardstick.

def direct_sum_fp64(targets: np.ndarray, sources: np.ndarray, masses: np.ndarray, world: float,
                    g_eff: float, soft: float = 0.0, chunk: int = 256) -> np.ndarray:
    """Minimum-image Newtonian gradient g_eff * sum_j m_j d / (|d|^2 + soft^2)^(3/2),
    d = x - x_j wrapped to [-L/2, L/2): the same sign and units as the
    solver's F (vel -= F dt attracts)."""
    targets = np.asarray(targets, dtype=np.float64)
    sources = np.asarray(sources, dtype=np.float64)
    masses = np.asarray(masses, dtype=np.float64)
    L = float(world)
    out = np.zeros((targets.shape[0], 3))
    for a in range(0, targets.shape[0], chunk):
        d = targets[a:a + chunk, None, :] - sources[None, :, :]
        d -= L * np.round(d / L)
        r2 = (d * d).sum(-1) + soft * soft
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = np.where(r2 > 0, r2 ** -1.5, 0.0)
        out[a:a + chunk] = g_eff * np.einsum("tj,tjc->tc", masses[None, :] * inv, d)
    return out
