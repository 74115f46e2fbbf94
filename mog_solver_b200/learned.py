"""Learned correction of a cheap MOG ensemble (no counterpart in the reference).

A cheap ensemble (k = 32 grids) is corrected towards an expensive one
(k = 240) by a 12 -> 64 -> 64 -> 3 GELU network that reads per-particle
statistics of the cheap ensemble.  Everything runs in libmog.so:

* ``mog_features``       deposit + solve + feature gather of the cheap ensemble;
* ``mog_model_train_step`` fused FP32 forward/backward + Adam (deterministic);
* ``mog_learned_step``   features + FP16 tensor-core inference + leapfrog, one fused kernel.

``generate_dataset`` builds training pairs from the method itself (features
of a k = 32 ensemble, targets = k = 240 force minus the k = 32 mean and
its per-particle least-squares correction);
``train`` fits the model; ``LearnedSimulation`` steps with the corrected
force and falls back to the plain expensive ensemble when a variance gate
fires (the particles' grid-to-grid force spread is far outside what the
model was trained on).
"""
from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from .simulation import Simulation, torch_device

FEATURES = ("Fx", "Fy", "Fz", "cFx", "cFy", "cFz", "sFx", "sFy", "sFz", "log_rho", "|F|",
            "offset_spread")
FORCE_COLS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 10]   # features proportional to 1/force_scale
SPREAD_COLS = slice(6, 9)


def _torch():
    import torch

    return torch


def norm_vector(mu, inv_sigma, force_scale: float, rho_ref: float, out_scale: float,
                base_mode: int = 0) -> np.ndarray:
    """The model's normalisation (MOG_MODEL_NORM floats).  base_mode 0: the
    residual is added to the plain mean force; 1: to the mean plus the
    least-squares correction (feature slots 12-14)."""
    v = np.zeros(_lib.MODEL_NORM, dtype=np.float32)
    v[0:12] = mu
    v[12:24] = inv_sigma
    v[24] = force_scale
    v[25] = rho_ref
    v[26] = out_scale
    v[27] = float(base_mode)
    return v


def init_params(seed: int = 0) -> np.ndarray:
    """Scaled-normal initialisation (the last layer starts small)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, 1 / np.sqrt(12), 64 * 12), np.zeros(64),
             rng.normal(0, 1 / np.sqrt(64), 64 * 64), np.zeros(64),
             rng.normal(0, 0.1 / np.sqrt(64), 3 * 64), np.zeros(3)]
    return np.concatenate(parts).astype(np.float32)


class Model:
    """A device-resident model (mog_model)."""

    def __init__(self, params: np.ndarray | None = None, norm: np.ndarray | None = None,
                 seed: int = 0):
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().mog_model_create(ctypes.byref(self._h)), "mog_model_create")
        if params is None:
            params = init_params(seed)
        if norm is None:
            norm = norm_vector(np.zeros(12), np.ones(12), 1.0, 1.0, 1.0)
        self.set(params, norm)

    @property
    def handle(self):
        return self._h

    def set(self, params: np.ndarray, norm: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        n = np.ascontiguousarray(norm, dtype=np.float32)
        if p.size != _lib.MODEL_PARAMS or n.size != _lib.MODEL_NORM:
            raise ValueError("params must have 5187 and norm 28 floats")
        _lib.check(_lib.lib().mog_model_set(self._h, p.ctypes.data_as(ctypes.c_void_p),
                                            n.ctypes.data_as(ctypes.c_void_p)), "mog_model_set")

    def get(self) -> tuple[np.ndarray, np.ndarray]:
        p = np.empty(_lib.MODEL_PARAMS, dtype=np.float32)
        n = np.empty(_lib.MODEL_NORM, dtype=np.float32)
        _lib.check(_lib.lib().mog_model_get(self._h, p.ctypes.data_as(ctypes.c_void_p),
                                            n.ctypes.data_as(ctypes.c_void_p)), "mog_model_get")
        return p, n

    def train_step(self, feat, target, idx, lr: float, want_loss: bool = False, grad_out=None):
        torch = _torch()
        loss = ctypes.c_float(0.0)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(_lib.lib().mog_model_train_step(
            self._h, feat.data_ptr(), target.data_ptr(), idx.data_ptr(), int(idx.numel()),
            float(lr), ctypes.byref(loss) if want_loss else None,
            grad_out.data_ptr() if grad_out is not None else None, stream), "mog_model_train_step")
        return float(loss.value) if want_loss else None

    def save(self, path: str | Path) -> None:
        p, n = self.get()
        np.savez(path, params=p, norm=n)

    @classmethod
    def load(cls, path: str | Path) -> "Model":
        d = np.load(path)
        return cls(d["params"], d["norm"])

    def close(self) -> None:
        if self._h:
            _lib.lib().mog_model_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


def features(sim: Simulation, model: Model, pos=None):
    """(mean force (n, 4), features (n, 16)) of sim's ensemble: columns 0-11
    standardised with model's norm, 12-14 the least-squares correction in
    force units, 15 zero."""
    torch = _torch()
    p = sim.pos if pos is None else pos
    n = int(p.shape[0])
    mean = torch.empty((n, 4), dtype=torch.float32, device=sim.device)
    feat = torch.empty((n, 16), dtype=torch.float32, device=sim.device)
    with torch_device(sim.device):
        _lib.check(_lib.lib().mog_features(sim.handle, model.handle, p.data_ptr(), n,
                                           mean.data_ptr(), feat.data_ptr(), sim._stream()),
                   "mog_features")
    return mean, feat


def learned_forces(sim: Simulation, model: Model, pos=None):
    torch = _torch()
    p = sim.pos if pos is None else pos
    out = torch.empty_like(p)
    with torch_device(sim.device):
        _lib.check(_lib.lib().mog_learned_forces(sim.handle, model.handle, p.data_ptr(),
                                                 out.data_ptr(), int(p.shape[0]), sim._stream()),
                   "mog_learned_forces")
    return out


@dataclass
class Dataset:
    feat: object            # torch (M, 16) standardised features
    target: object          # torch (M, 4) residual / out_scale
    norm: np.ndarray        # the model normalisation
    stats: dict = field(default_factory=dict)


def _cfg(k: int, g: int, L: float, G: float, n: int, seed: int, dt: float = 1e-5,
         damping: float = 0.999) -> dict:
    return {"n_grids": k, "grid_size": g, "world_size": L, "num_particles": n, "G": G, "dt": dt,
            "damping": damping, "seed": seed}


def training_sets(n_sets: int, n: int, world: float, seed0: int, disk_sets: int, disk_seed0: int):
    """The particle sets of the training data: n_sets Gaussian-clump sets
    (ics.clumps, seeds seed0...) and disk_sets randomly oriented disk pairs
    (ics.rotated_disk_pair, seeds disk_seed0...)."""
    from . import ics

    for i in range(n_sets):
        yield ics.clumps(n, world, seed=seed0 + i)[0]
    for i in range(disk_sets):
        yield ics.rotated_disk_pair(n, world, seed=disk_seed0 + i)[0]


def generate_dataset(n_sets: int = 64, n: int = 262144, k_small: int = 32, k_big: int = 240,
                     g: int = 16, world: float = 100.0, G: float = 100.0, seed0: int = 100,
                     small_seed: int = 1000, big_seed: int = 2000, disk_sets: int = 0,
                     disk_seed0: int = 500) -> Dataset:
    """Training pairs the method generates itself: for seeded clump sets
    (and disk_sets randomly oriented disk pairs), features of the k_small
    ensemble and the k_big force minus the k_small base force (mean +
    least-squares correction, base_mode 1).  Returns standardised tensors
    and the matching normalisation."""
    torch = _torch()
    small = Simulation(_cfg(k_small, g, world, G, n, small_seed))
    big = Simulation(_cfg(k_big, g, world, G, n, big_seed))
    rho_ref = 1.0 / g ** 3          # total mass 1 over g^3 cells
    raw = Model(norm=norm_vector(np.zeros(12), np.ones(12), 1.0, rho_ref, 1.0))
    feats, resid = [], []
    for pos in training_sets(n_sets, n, world, seed0, disk_sets, disk_seed0):
        small.set_particles(pos)
        big.set_particles(pos)
        mean, f = features(small, raw)
        fb = big.forces()
        feats.append(f[:, :12].clone())
        resid.append((fb[:, :3] - mean[:, :3] - f[:, 12:15]).clone())
    raw.close()
    small.close()
    big.close()
    F = torch.cat(feats)
    R = torch.cat(resid)
    # force scale: RMS of the cheap mean force; features then standardised
    s = float(torch.sqrt((F[:, 0:3].double() ** 2).sum(1).mean()).item())
    F[:, FORCE_COLS] /= s
    mu = F.double().mean(0)
    sd = F.double().std(0).clamp_min(1e-12)
    Fz = ((F.double() - mu) / sd).float()
    out_scale = float(torch.sqrt((R.double() ** 2).sum(1).mean()).item())
    T = torch.zeros((R.shape[0], 4), dtype=torch.float32, device=R.device)
    T[:, :3] = (R / out_scale).float()
    feat16 = torch.zeros((Fz.shape[0], 16), dtype=torch.float32, device=Fz.device)
    feat16[:, :12] = Fz
    norm = norm_vector(mu.cpu().numpy(), (1.0 / sd).cpu().numpy(), s, rho_ref, out_scale, base_mode=1)
    stats = {"force_scale": s, "out_scale": out_scale, "samples": int(Fz.shape[0]),
             "spread_mean": float(F[:, SPREAD_COLS].double().mean().item())}
    return Dataset(feat16, T, norm, stats)


def train(model: Model, data: Dataset, steps: int = 2000, batch: int = 8192, lr: float = 1e-3,
          seed: int = 0, log_every: int = 100) -> list[tuple[int, float]]:
    """Adam on the mean squared error of the standardised residual."""
    torch = _torch()
    params, _ = model.get()
    model.set(params, data.norm)
    g = torch.Generator(device=data.feat.device)
    g.manual_seed(seed)
    M = data.feat.shape[0]
    history = []
    for step in range(1, steps + 1):
        idx = torch.randint(0, M, (batch,), generator=g, device=data.feat.device, dtype=torch.int32)
        want = step == 1 or step % log_every == 0 or step == steps
        loss = model.train_step(data.feat, data.target, idx, lr, want_loss=want)
        if want:
            history.append((step, loss))
    return history


def residual_errors(model: Model, sets, k_small: int = 32, k_big: int = 240, g: int = 16,
                    world: float = 100.0, G: float = 100.0, alphas=(1.0,), small_seed: int = 1000,
                    big_seed: int = 2000) -> list[dict]:
    """For each particle set: the relative RMS distance to the k_big force of
    the k_small plain mean, of its least-squares correction alone ("ls") and
    of the learned force with the network's output scaled by each alpha
    (alpha 0 is the least-squares force)."""
    n = max(int(p.shape[0]) for p in sets)
    small = Simulation(_cfg(k_small, g, world, G, n, small_seed))
    big = Simulation(_cfg(k_big, g, world, G, n, big_seed))
    params, norm = model.get()
    rows = []
    try:
        for pos in sets:
            small.set_particles(pos)
            big.set_particles(pos)
            fb = big.forces()
            mean, feat = features(small, model)
            ls = mean.clone()
            ls[:, :3] += feat[:, 12:15]
            row = {"plain": rms_error(mean, fb), "ls": rms_error(ls, fb)}
            for a in alphas:
                scaled = norm.copy()
                scaled[26] = norm[26] * a
                model.set(params, scaled)
                row[f"net_x{a:g}"] = rms_error(learned_forces(small, model), fb)
            model.set(params, norm)
            rows.append(row)
    finally:
        model.set(params, norm)
        small.close()
        big.close()
    return rows


def select_output_scale(model: Model, val_sets, alphas=(0.25, 0.5, 0.75, 1.0), **kw) -> dict:
    """Scale the network's output (the norm's out_scale) by the alpha whose
    learned force is closest to the k_big force on held-out validation
    sets (mean relative RMS error); alpha 0, the least-squares force alone,
    is kept when no alpha beats it.  Returns the table it chose from."""
    rows = residual_errors(model, val_sets, alphas=alphas, **kw)
    score = {a: float(np.mean([r[f"net_x{a:g}"] for r in rows])) for a in alphas}
    score[0.0] = float(np.mean([r["ls"] for r in rows]))
    best = min(score, key=score.get)
    params, norm = model.get()
    norm[26] = norm[26] * best
    model.set(params, norm)
    return {"alpha": best, "validation_mean_error": score, "validation": rows}


def _gate_stats(feat, norm) -> tuple[float, float]:
    """(mean spread, mean |mean force|) over particles from a feature pass:
    features 6-8 and 10 before standardisation, in units of force_scale."""
    torch = _torch()
    sd = torch.from_numpy((1.0 / norm[12:24]).astype(np.float64)).to(feat.device)
    mu = torch.from_numpy(norm[0:12].astype(np.float64)).to(feat.device)
    raw = feat[:, :12].double() * sd + mu
    return float(raw[:, 6:9].mean(dim=1).mean().item()), float(raw[:, 10].mean().item())


class LearnedSimulation:
    """A cheap ensemble stepped with the learned correction, and the plain
    expensive ensemble as fallback when the variance gate fires.

    Gate: every ``gate_every`` steps, the relative grid-to-grid force spread
    of the particles -- their mean force spread over their mean force
    magnitude, both summed inside the last learned step's own kernel
    (mog_learned_spread) -- is compared with ``gate_factor`` times the same
    ratio on the training data (``train_ratio``; by default taken from the
    model's normalisation offsets of features 6-8 and 10).  When it is
    above, the fallback ensemble takes the next ``gate_every`` steps, after
    which a feature pass of the cheap ensemble decides again.
    """

    def __init__(self, cheap: Simulation, model: Model, fallback: Simulation | None = None,
                 train_ratio: float | None = None, gate_factor: float = 3.0,
                 gate_every: int = 10):
        self.cheap = cheap
        self.model = model
        self.fallback = fallback
        if train_ratio is None:
            _, norm = model.get()
            train_ratio = float(np.mean(norm[6:9]) / norm[10]) if norm[10] > 0 else 0.0
        self.train_ratio = train_ratio
        self.gate_factor = gate_factor
        self.gate_every = gate_every
        self.steps = 0
        self.fallback_steps = 0
        self.last_ratio = None
        self._use_fallback = False

    @property
    def pos(self):
        return self.cheap.pos

    @property
    def vel(self):
        return self.cheap.vel

    def step_stats(self) -> tuple[float, float]:
        """(mean spread, mean |mean force|) of the last learned step."""
        out = (ctypes.c_double * 2)()
        with torch_device(self.cheap.device):
            _lib.check(_lib.lib().mog_learned_spread(self.cheap.handle, out, self.cheap._stream()),
                       "mog_learned_spread")
        return float(out[0]), float(out[1])

    def feature_stats(self) -> tuple[float, float]:
        """The same statistics from a separate feature pass (mog_features)."""
        _, norm = self.model.get()
        _, feat = features(self.cheap, self.model)
        return _gate_stats(feat, norm)

    def gate_fires(self) -> bool:
        if self.fallback is None or not self.train_ratio:
            return False
        # after a learned step its kernel has summed the statistics already;
        # after fallback steps a feature pass measures them
        spread, fmag = self.feature_stats() if self._use_fallback else self.step_stats()
        self.last_ratio = spread / fmag if fmag > 0 else float("inf")
        return self.last_ratio > self.gate_factor * self.train_ratio

    def step(self, n_steps: int = 1) -> None:
        torch = _torch()
        lib = _lib.lib()
        for _ in range(n_steps):
            if self.gate_every and self.steps % self.gate_every == 0 and self.steps > 0:
                self._use_fallback = self.gate_fires()
            if self._use_fallback:
                fb = self.fallback
                fb.pos, fb.vel = self.cheap.pos, self.cheap.vel
                fb.step()
                self.fallback_steps += 1
            else:
                c = self.cheap
                dt = float(c.cfg.dt * c.timescale)
                with torch_device(c.device):
                    _lib.check(lib.mog_learned_step(c.handle, self.model.handle, c.pos.data_ptr(),
                                                    c.vel.data_ptr(), c.n_particles, dt,
                                                    c._stream()), "mog_learned_step")
            self.steps += 1

    def step_host(self, pos_host, vel_host, n_steps: int = 1, chunks: int = 8) -> None:
        """``step`` for particles held in host memory ((N, 4) float32 CPU
        tensors, page-locked): each step copies the records in, steps them
        and copies them back in overlapped chunks (mog_learned_step_host,
        or mog_step_host on the fallback ensemble when the gate has fired).
        The gate reads the last learned step's own statistics; after
        fallback steps a feature pass over the current records decides.
        Returns once the stepped records are in the host buffers."""
        from .simulation import _check_host_records

        torch = _torch()
        _check_host_records(pos_host, vel_host)
        lib = _lib.lib()
        n = int(pos_host.shape[0])
        c = self.cheap
        for _ in range(n_steps):
            if self.gate_every and self.steps % self.gate_every == 0 and self.steps > 0:
                if self._use_fallback:
                    c.pos.copy_(pos_host)
                self._use_fallback = self.gate_fires()
            with torch_device(c.device):
                stream = c._stream()
                if self._use_fallback:
                    fb = self.fallback
                    _lib.check(lib.mog_step_host(fb.handle, pos_host.data_ptr(), vel_host.data_ptr(),
                                                 n, float(fb.cfg.dt * fb.timescale), int(chunks),
                                                 stream), "mog_step_host")
                    self.fallback_steps += 1
                else:
                    _lib.check(lib.mog_learned_step_host(c.handle, self.model.handle,
                                                         pos_host.data_ptr(), vel_host.data_ptr(), n,
                                                         float(c.cfg.dt * c.timescale), int(chunks),
                                                         stream), "mog_learned_step_host")
            self.steps += 1
        torch.cuda.current_stream(c.device).synchronize()


def rms_error(F, D) -> float:
    """Relative RMS error ||F - D|| / ||D|| over the target particles."""
    torch = _torch()
    F = F[:, :3].double()
    D = D[:, :3].double()
    return float((torch.linalg.norm(F - D) / torch.linalg.norm(D)).item())


def direct_sum(targets, sources, world: float, g_eff: float, soft: float = 0.0):
    """FP64 direct-sum yardstick on the GPU (mog_direct_sum), (nt, 3) float64."""
    torch = _torch()
    out = torch.empty((targets.shape[0], 3), dtype=torch.float64, device=targets.device)
    _lib.check(_lib.lib().mog_direct_sum(targets.data_ptr(), int(targets.shape[0]),
                                         sources.data_ptr(), int(sources.shape[0]), float(world),
                                         float(g_eff), float(soft), out.data_ptr(),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
               "mog_direct_sum")
    return out


def save_report(path: str | Path, report: dict) -> None:
    Path(path).write_text(json.dumps(report, indent=2))
