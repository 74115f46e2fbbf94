"""``Simulation``: the reference's operator surface over the CUDA library.

The reference's ``Simulation`` (main.py:101-773) owns GL buffers and runs
``step()`` (main.py:671-672) once per frame.  This class keeps the same
surface for the force-and-step path:

* construction from a config mapping (or a config.yaml path) with the
  reference's parse rules and per-grid transforms drawn by
  ``RandomSE3Sampler`` (main.py:157-172);
* ``pos`` / ``vel``: device-resident (N, 4) float32 torch tensors, the
  std430 ``vec4`` records of ``pos_buf`` / ``vel_buf`` (main.py:192-193);
* ``step()`` advances one step with ``deltaTime = dt * timescale``
  (main.py:662), ``timescale`` playing the role of the reference's key
  controls (main.py:741-751);
* ``offsets`` / ``rotations``: the packed transforms (main.py:157-172).

All arithmetic runs in libmog.so on the GPU; this module only moves
pointers and sizes across the C ABI.  There is no CPU path.
"""
from __future__ import annotations

import ctypes
import json
import math
from pathlib import Path
from typing import Any, Mapping

import numpy as np

from . import _lib
from .config import MogConfig, load_config
from .transforms import compute_transforms

_MASS_MODE = {"u64": _lib.MASS_U64_FIXED, "u32x1000": _lib.MASS_U32_X1000}
_INDEX = {"fast": _lib.INDEX_FAST, "exact": _lib.INDEX_EXACT}
_SOLVER = {"fft": _lib.SOLVER_FFT, "convolution": _lib.SOLVER_CONVOLUTION}
_DFT = {"fp32": _lib.DFT_FFT32, "bf16x3": _lib.DFT_TC_BF16X3}


def _torch():
    import torch

    return torch


def _check_host_records(pos_host, vel_host) -> None:
    """Host-step buffers: (N, 4) contiguous float32 CPU tensors of one shape."""
    torch = _torch()
    for t in (pos_host, vel_host):
        if not torch.is_tensor(t) or t.is_cuda or t.dtype != torch.float32 or t.dim() != 2 \
                or t.shape[1] != 4 or not t.is_contiguous():
            raise ValueError("host records must be contiguous (N, 4) float32 CPU tensors")
    if pos_host.shape != vel_host.shape:
        raise ValueError("pos and vel must have the same shape")


def auto_scale_bits(total_mass: float) -> int:
    """u64 fixed-point scale 2^bits with bits = 52 - ceil(log2(total mass)).

    Every cell holds at most the total mass, so the largest cell value stays
    below 2^53 (and far below 2^64): no overflow, and with masses 1/N of a
    power-of-two N every particle's mass is represented exactly.
    """
    if not total_mass > 0 or not math.isfinite(total_mass):
        return 32
    return int(min(100, max(0, 52 - math.ceil(math.log2(total_mass)))))


class Simulation:
    """Mixture-of-Grids N-body simulation on one GPU."""

    def __init__(self, cfg: Mapping[str, Any] | MogConfig | str | Path | None = None, *,
                 seed: int | None = None, device: str | int | None = None,
                 offsets: np.ndarray | None = None, rotations: np.ndarray | None = None):
        torch = _torch()
        if cfg is None or isinstance(cfg, (str, Path)):
            cfg = load_config(cfg)
        self.cfg = cfg if isinstance(cfg, MogConfig) else MogConfig.from_dict(cfg)
        if seed is not None:
            self.cfg.seed = seed
        c = self.cfg
        self.timescale = 1.0
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   torch.device(device).index or 0)
        if offsets is None or rotations is None:
            self.offsets, self.rotations = compute_transforms(c.n_grids, c.grid_size, c.world_size,
                                                              seed=c.seed)
        else:
            self.offsets = np.ascontiguousarray(offsets, dtype=np.float32).reshape(c.n_grids, 4)
            self.rotations = np.ascontiguousarray(rotations, dtype=np.float32).reshape(c.n_grids, 12)
        n = c.num_particles
        self.pos = torch.zeros((n, 4), dtype=torch.float32, device=self.device)
        self.vel = torch.zeros((n, 4), dtype=torch.float32, device=self.device)
        self._handle = None
        self._handle_bits = None
        self._auto_bits = None
        self.steps_taken = 0

    # ------------------------------------------------------------------
    @property
    def voxel_size(self) -> float:
        return self.cfg.voxel_size

    @property
    def n_particles(self) -> int:
        return int(self.pos.shape[0])

    def effective_g(self) -> float:
        """Gravitational constant of the solver's force units, G * h^3 / 2.

        greens.glsl uses -2 pi G / k^2 on cell masses and pack.glsl divides
        by g^3, so the reference's field is h^3/2 times the Newtonian
        periodic gradient for G.
        """
        h = self.voxel_size
        return self.cfg.G * h ** 3 / 2.0

    def _stream(self):
        torch = _torch()
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _config_c(self, scale_bits: int) -> _lib.MogConfigC:
        c = self.cfg
        cc = _lib.MogConfigC()
        cc.n_grids = c.n_grids
        cc.grid_size = c.grid_size
        cc.world_size = c.world_size
        cc.G = c.G
        cc.dt = c.dt
        cc.damping = c.damping
        cc.solver = _SOLVER[c.solver]
        cc.mass_mode = _MASS_MODE[c.mass_mode]
        cc.scale_bits = scale_bits
        cc.index_mode = _INDEX[c.index_mode]
        cc.dft_prec = _DFT[c.dft_precision]
        cc.compat_flags = _lib.COMPAT_FFT_TEXTURE_ALIAS if c.reference_texture_aliasing else 0
        cc.num_particles = max(self.n_particles, c.num_particles)
        cc.softening = c.softening
        return cc

    def _scale_bits(self) -> int:
        """Configured scale, else one chosen from the total mass (computed once
        per particle set, so steps never synchronise the host)."""
        if self.cfg.scale_bits is not None:
            return self.cfg.scale_bits
        if self._auto_bits is None:
            torch = _torch()
            total = float(self.pos[:, 3].to(torch.float64).sum().item()) if self.n_particles else 1.0
            self._auto_bits = auto_scale_bits(total)
        return self._auto_bits

    @property
    def scale_bits(self) -> int:
        """u64 fixed-point scale 2^bits of the current handle (0 in u32 mode)."""
        self.handle
        return self._handle_bits

    def deposit_layout(self, bits: int) -> int:
        """The one-word deposit histogram that suits the masses at scale
        2^bits (u64 fixed-point mode): 1 (high words) when every particle
        has the same mass m and q = m 2^bits is a multiple of 2^32, 2
        (counts) when the masses are equal otherwise, 0 (the two-word
        histogram) for unequal masses."""
        if self.cfg.mass_mode != "u64" or not self.n_particles:
            return 0
        w = self.pos[:, 3]
        lo, hi = float(w.min().item()), float(w.max().item())
        if lo != hi or not (lo > 0 and math.isfinite(lo)):
            return 0
        q = lo * 2.0 ** bits  # exact: a float32 times a power of two
        if q < 2.0 ** 64 and q >= 2.0 ** 32 and math.fmod(q, 2.0 ** 32) == 0:
            return 1
        return 2

    def _apply_layout(self, h) -> None:
        """Deposit histogram layout unless the caller chose one (see
        deposit_layout): one word per cell, twice the grids per CTA, when
        the masses are equal.  Checked once per particle set (one host read
        of the masses' range)."""
        self._layout_checked = True
        if "deposit_split" in (getattr(self, "_tuning", None) or {}):
            return
        want = self.deposit_layout(self._handle_bits or 0)
        lib = _lib.lib()
        t = _lib.MogTuningC()
        _lib.check(lib.mog_get_tuning(h, ctypes.byref(t)), "mog_get_tuning")
        if t.deposit_split != want:
            t.deposit_split = want
            _lib.check(lib.mog_set_tuning(h, ctypes.byref(t)), "mog_set_tuning")

    @property
    def handle(self):
        """The libmog handle; (re)created when the fixed-point scale changes."""
        bits = self._scale_bits() if self.cfg.mass_mode == "u64" else 0
        if self._handle is not None and bits == self._handle_bits:
            if not getattr(self, "_layout_checked", False):
                self._apply_layout(self._handle)
            return self._handle
        self.close()
        lib = _lib.lib()
        h = ctypes.c_void_p()
        cc = self._config_c(bits)
        with torch_device(self.device):
            _lib.check(lib.mog_create(ctypes.byref(cc), self.rotations.ctypes.data_as(ctypes.c_void_p),
                                      self.offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(h)),
                       "mog_create")
        self._handle = h
        self._handle_bits = bits
        if getattr(self, "_tuning", None):
            t = _lib.MogTuningC()
            _lib.check(lib.mog_get_tuning(h, ctypes.byref(t)), "mog_get_tuning")
            for k, v in self._tuning.items():
                setattr(t, k, int(v))
            _lib.check(lib.mog_set_tuning(h, ctypes.byref(t)), "mog_set_tuning")
        self._apply_layout(h)
        return h

    def close(self) -> None:
        if self._handle is not None:
            _lib.lib().mog_destroy(self._handle)
            self._handle = None
            self._handle_bits = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order varies
        try:
            self.close()
        except Exception:
            pass

    def tuning(self) -> dict[str, int]:
        """Current launch shapes of the handle (mog_get_tuning)."""
        t = _lib.MogTuningC()
        _lib.check(_lib.lib().mog_get_tuning(self.handle, ctypes.byref(t)), "mog_get_tuning")
        return {name: getattr(t, name) for name, _ in t._fields_}

    def tune(self, **shapes: int) -> None:
        """Set launch shapes (mog_set_tuning); results never depend on them."""
        t = _lib.MogTuningC()
        lib = _lib.lib()
        _lib.check(lib.mog_get_tuning(self.handle, ctypes.byref(t)), "mog_get_tuning")
        for k, v in shapes.items():
            if k not in {name for name, _ in t._fields_}:
                raise KeyError(f"unknown tuning field {k!r}")
            setattr(t, k, int(v))
        _lib.check(lib.mog_set_tuning(self.handle, ctypes.byref(t)), "mog_set_tuning")
        self._tuning = {**(getattr(self, "_tuning", None) or {}), **shapes}

    # ------------------------------------------------------------------
    def set_particles(self, pos, vel=None) -> None:
        """Upload (N, 4) float32 records (numpy or torch)."""
        torch = _torch()
        p = torch.as_tensor(np.asarray(pos, dtype=np.float32) if not torch.is_tensor(pos) else pos)
        p = p.to(device=self.device, dtype=torch.float32).reshape(-1, 4).contiguous()
        if vel is None:
            v = torch.zeros_like(p)
        else:
            v = torch.as_tensor(np.asarray(vel, dtype=np.float32) if not torch.is_tensor(vel) else vel)
            v = v.to(device=self.device, dtype=torch.float32).reshape(-1, 4).contiguous()
        if v.shape != p.shape:
            raise ValueError("pos and vel must have the same shape")
        if p.shape[0] > self.cfg.num_particles:
            self.cfg.num_particles = int(p.shape[0])
            self.close()
        self.pos = p
        self.vel = v
        self._auto_bits = None  # the fixed-point scale depends on the masses
        self._layout_checked = False  # and so does the deposit's histogram layout

    def init_particles(self, kind: str = "uniform", seed: int | None = None, **kw) -> None:
        """Replace the particles with a named initial set: uniform, disks,
        plummer, clumps (seed default 0), two_galaxies (the reference's
        init_particles2, its exact NumPy draws), two_galaxies_gpu (the same
        initialiser as a CUDA kernel with counter-based draws) or perlin
        (the reference's GPU sampler,
        init_particles.glsl, seed default 12345 as in main.py:281)."""
        from . import ics

        n, L = self.cfg.num_particles, self.cfg.world_size
        if seed is None:
            seed = 12345 if kind == "perlin" else 0
        if kind == "uniform":
            pos, vel = ics.uniform_cube(n, L, seed=seed, **kw)
        elif kind == "disks":
            kw.setdefault("g_eff", self.effective_g())
            pos, vel = ics.two_disks(n, L, seed=seed, **kw)
        elif kind == "plummer":
            pos, vel = ics.plummer(n, L, seed=seed, **kw)
        elif kind == "clumps":
            pos, vel = ics.clumps(n, L, seed=seed, **kw)
        elif kind == "two_galaxies":  # the reference's init_particles2 (main.py:312-357)
            pos, vel = ics.reference_two_galaxies(n, L, self.cfg.particle_mass, seed=seed)
        elif kind == "two_galaxies_gpu":  # the same distribution drawn on this GPU
            torch = _torch()
            pos = torch.empty((n, 4), dtype=torch.float32, device=self.device)
            vel = torch.empty_like(pos)
            with torch_device(self.device):
                _lib.check(_lib.lib().mog_init_two_galaxies(
                    pos.data_ptr(), vel.data_ptr(), n, float(L), float(self.cfg.particle_mass),
                    int(seed) & 0xFFFFFFFFFFFFFFFF, self._stream()), "mog_init_two_galaxies")
        elif kind == "perlin":  # the reference's GPU sampler (main.py:280-310), on this GPU
            torch = _torch()
            pos = torch.empty((n, 4), dtype=torch.float32, device=self.device)
            vel = torch.empty_like(pos)
            args = ics.perlin_args(n, L, self.cfg.particle_mass, self.cfg.spawn_buffer,
                                   seed=seed, **kw)
            with torch_device(self.device):
                _lib.check(_lib.lib().mog_init_particles(pos.data_ptr(), vel.data_ptr(), *args,
                                                         self._stream()), "mog_init_particles")
        else:
            raise ValueError(f"unknown particle set {kind!r}")
        self.set_particles(pos, vel)

    # ------------------------------------------------------------------
    def step(self, n_steps: int = 1) -> None:
        """Advance ``n_steps`` steps (main.py:671-676)."""
        dt_eff = float(self.cfg.dt * self.timescale)
        h = self.handle
        lib = _lib.lib()
        with torch_device(self.device):
            if n_steps == 1:
                _lib.check(lib.mog_step(h, self.pos.data_ptr(), self.vel.data_ptr(), self.n_particles,
                                        dt_eff, self._stream()), "mog_step")
            else:
                _lib.check(lib.mog_step_n(h, self.pos.data_ptr(), self.vel.data_ptr(),
                                          self.n_particles, dt_eff, int(n_steps), self._stream()),
                           "mog_step_n")
        self.steps_taken += n_steps

    def step_host(self, pos_host, vel_host, n_steps: int = 1, chunks: int = 8) -> None:
        """Advance particles held in host memory (mog_step_host): (N, 4)
        float32 CPU tensors, page-locked for the copies to overlap the
        kernels.  The call returns once the stepped records are back in
        the host buffers.  ``self.pos`` / ``self.vel`` are not touched."""
        torch = _torch()
        _check_host_records(pos_host, vel_host)
        dt_eff = float(self.cfg.dt * self.timescale)
        n = int(pos_host.shape[0])
        lib = _lib.lib()
        with torch_device(self.device):
            stream = self._stream()
            for _ in range(n_steps):
                _lib.check(lib.mog_step_host(self.handle, pos_host.data_ptr(), vel_host.data_ptr(), n,
                                             dt_eff, int(chunks), stream), "mog_step_host")
            torch.cuda.current_stream(self.device).synchronize()
        self.steps_taken += n_steps

    def render(self, width: int = 2560, height: int = 1440, **kw):
        """The frame on_render draws (main.py:678-703), headless: an
        (height, width, 4) image on this GPU.  Keywords as
        mog_solver_b200.render.params (camera angles and distance,
        speed_scale, point_mode, fmt)."""
        from .render import render

        kw.setdefault("world_size", self.cfg.world_size)
        with torch_device(self.device):
            return render(self.pos, self.vel, width=width, height=height, **kw)

    def forces(self, pos=None):
        """Ensemble-averaged force at each particle, (N, 4) with w = 0."""
        torch = _torch()
        p = self.pos if pos is None else pos
        out = torch.empty_like(p)
        h = self.handle
        with torch_device(self.device):
            _lib.check(_lib.lib().mog_forces(h, p.data_ptr(), out.data_ptr(), int(p.shape[0]),
                                             self._stream()), "mog_forces")
        return out

    def mass_grid(self, pos=None):
        """Fixed-point mass grid (k, g, g, g): int64 view of u64 cells, or int64 of u32."""
        torch = _torch()
        p = self.pos if pos is None else pos
        c = self.cfg
        shape = (c.n_grids, c.grid_size, c.grid_size, c.grid_size)
        dt = torch.int64 if c.mass_mode == "u64" else torch.int32
        out = torch.empty(shape, dtype=dt, device=self.device)
        h = self.handle
        with torch_device(self.device):
            _lib.check(_lib.lib().mog_deposit(h, p.data_ptr(), int(p.shape[0]), out.data_ptr(),
                                              self._stream()), "mog_deposit")
        return out

    def solve_grid(self, mass):
        """Force grid (k, g, g, g, 4) = (fx, fy, fz, |f|) per cell, grid frame."""
        torch = _torch()
        c = self.cfg
        out = torch.empty((c.n_grids, c.grid_size, c.grid_size, c.grid_size, 4),
                          dtype=torch.float32, device=self.device)
        h = self.handle
        with torch_device(self.device):
            _lib.check(_lib.lib().mog_solve(h, mass.data_ptr(), out.data_ptr(), self._stream()),
                       "mog_solve")
        return out

    def update_from_grid(self, force_grid, dt_eff: float | None = None) -> None:
        """update.glsl from a caller force grid (k, g, g, g, 4), in place."""
        dt = float(self.cfg.dt * self.timescale) if dt_eff is None else float(dt_eff)
        h = self.handle
        with torch_device(self.device):
            _lib.check(_lib.lib().mog_update(h, self.pos.data_ptr(), self.vel.data_ptr(),
                                             self.n_particles, force_grid.data_ptr(), dt,
                                             self._stream()), "mog_update")

    def status(self) -> int:
        """Device status bits raised since the last call (synchronises)."""
        v = ctypes.c_uint32(0)
        with torch_device(self.device):
            _lib.check(_lib.lib().mog_get_status(self.handle, ctypes.byref(v), self._stream()),
                       "mog_get_status")
        return int(v.value)

    def check(self) -> None:
        """Raise MogError if a device flag was raised."""
        flags = self.status()
        if flags & _lib.FLAG_NONFINITE:
            raise _lib.MogError(_lib.MOG_ERR_NONFINITE, "step", "a particle position became NaN/Inf")
        if flags & _lib.FLAG_OVERFLOW:
            raise _lib.MogError(_lib.MOG_ERR_OVERFLOW, "deposit", "fixed-point mass total left the u64 range")
        if flags & _lib.FLAG_TIMEOUT:
            raise _lib.MogError(_lib.MOG_ERR_TIMEOUT, "update", "a bounded device wait timed out")
        if flags & _lib.FLAG_BADMASS:
            raise _lib.MogError(_lib.MOG_ERR_ARG, "deposit", "negative or NaN particle mass")

    def diagnostics(self) -> dict[str, Any]:
        """FP64 momentum, kinetic energy, total mass and centre of mass."""
        out = (ctypes.c_double * 8)()
        with torch_device(self.device):
            _lib.check(_lib.lib().mog_diagnostics(self.handle, self.pos.data_ptr(), self.vel.data_ptr(),
                                                  self.n_particles, out, self._stream()),
                       "mog_diagnostics")
        v = list(out)
        return {"momentum": v[0:3], "kinetic_energy": v[3], "mass": v[4], "com": v[5:8]}

    # ------------------------------------------------------------------
    def save(self, path: str | Path) -> None:
        """Checkpoint: particles, transforms, config and step count (.npz)."""
        header = {"cfg": self.cfg.to_dict(), "steps_taken": self.steps_taken,
                  "timescale": self.timescale, "format": "mog-b200-checkpoint-1"}
        np.savez(path, pos=self.pos.cpu().numpy(), vel=self.vel.cpu().numpy(),
                 offsets=self.offsets, rotations=self.rotations,
                 header=np.frombuffer(json.dumps(header).encode(), dtype=np.uint8))

    @classmethod
    def load(cls, path: str | Path, device=None) -> "Simulation":
        data = np.load(path)
        header = json.loads(bytes(data["header"]).decode())
        cfg = MogConfig(**header["cfg"])
        sim = cls(cfg, device=device, offsets=data["offsets"], rotations=data["rotations"])
        sim.set_particles(data["pos"], data["vel"])
        sim.steps_taken = int(header["steps_taken"])
        sim.timescale = float(header["timescale"])
        return sim


class torch_device:
    """Context manager making ``device`` current for the duration of a call."""

    def __init__(self, device):
        self.device = device

    def __enter__(self):
        torch = _torch()
        self._ctx = torch.cuda.device(self.device)
        return self._ctx.__enter__()

    def __exit__(self, *exc):
        return self._ctx.__exit__(*exc)
