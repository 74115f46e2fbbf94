"""Several independent simulations advanced together (one CUDA graph per
ensemble step; mog_batch_* in include/mog.h).

The reference runs one simulation per window; this is the batched uneven
ensemble of the benchmark configurations: simulations of different N, k and
g step in a single graph launch.  By default the graph holds one persistent
work-queue deposit over every simulation, each simulation's solve on its
own branch, and one persistent work-queue gather + update over every
simulation (CTAs pop (simulation, grid group, particle chunk) tiles, largest
first); ``tune(work_queue=0)`` runs each simulation's kernels on its own
branch instead.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .simulation import Simulation, torch_device


class Batch:
    def __init__(self, sims: list[Simulation]):
        if not sims:
            raise ValueError("a batch needs at least one simulation")
        self.sims = list(sims)
        self._h = ctypes.c_void_p()
        self._built_for = None
        self._tuning = {"work_queue": 1, "deposit_chunk": 0, "deposit_split": 0}
        self._split_chosen = False  # deposit_split set by the caller

    def _handles(self):
        hs = [s.handle for s in self.sims]  # creates / refreshes each handle
        key = tuple(h.value for h in hs)
        if self._built_for != key:
            self.close()
            arr = (ctypes.c_void_p * len(hs))(*[h.value for h in hs])
            _lib.check(_lib.lib().mog_batch_create(arr, len(hs), ctypes.byref(self._h)),
                       "mog_batch_create")
            self._built_for = key
            self._apply_tuning()
        return self._h

    def _apply_tuning(self) -> None:
        split = int(self._tuning["deposit_split"])
        if not self._split_chosen:
            # one word per cell when every simulation's masses are equal:
            # high words if every low half is zero, else counts (checked
            # when the batch is built or retuned)
            kinds = {s.deposit_layout(s.scale_bits) for s in self.sims}
            split = 0 if 0 in kinds else (1 if kinds == {1} else 2)
        t = _lib.MogBatchTuningC(work_queue=int(self._tuning["work_queue"]),
                                 deposit_chunk=int(self._tuning["deposit_chunk"]),
                                 deposit_split=split)
        _lib.check(_lib.lib().mog_batch_set_tuning(self._h, ctypes.byref(t)), "mog_batch_set_tuning")

    def tune(self, **kw) -> None:
        """Set launch shapes: work_queue (1 persistent work-queue launches,
        0 one branch per simulation), deposit_chunk (particles per deposit
        tile, 0 = library default), deposit_split (1: high-word histograms
        at every grid size, for masses whose fixed-point low halves are 0;
        2: count histograms, for equal masses; chosen from the masses
        unless set here)."""
        unknown = set(kw) - set(self._tuning)
        if unknown:
            raise ValueError(f"unknown batch tuning fields {sorted(unknown)}")
        self._tuning.update(kw)
        if "deposit_split" in kw:
            self._split_chosen = True
        if self._h:
            self._apply_tuning()

    def tuning(self) -> dict:
        """The batch's launch shapes, plus whether the work queue applies
        to these simulations (active_work_queue)."""
        t = _lib.MogBatchTuningC()
        _lib.check(_lib.lib().mog_batch_get_tuning(self._handles(), ctypes.byref(t)),
                   "mog_batch_get_tuning")
        return {name: int(getattr(t, name)) for name, _ in t._fields_}

    def step(self, n_steps: int = 1) -> None:
        import torch

        h = self._handles()
        k = len(self.sims)
        pos = (ctypes.c_void_p * k)(*[s.pos.data_ptr() for s in self.sims])
        vel = (ctypes.c_void_p * k)(*[s.vel.data_ptr() for s in self.sims])
        n = (ctypes.c_int64 * k)(*[s.n_particles for s in self.sims])
        dt = (ctypes.c_float * k)(*[float(s.cfg.dt * s.timescale) for s in self.sims])
        dev = self.sims[0].device
        with torch_device(dev):
            stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
            _lib.check(_lib.lib().mog_batch_step(h, pos, vel, n, dt, int(n_steps), stream),
                       "mog_batch_step")
        for s in self.sims:
            s.steps_taken += n_steps

    @property
    def n_particles(self) -> int:
        return sum(s.n_particles for s in self.sims)

    def close(self) -> None:
        if self._h:
            _lib.lib().mog_batch_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._built_for = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
