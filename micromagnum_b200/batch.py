"""Batched solves over the C ABI (`mm_batch_*`).

Many independent boxes of uneven size (each with its own mask, Ms, A, alpha and applied field)
advance in lock step: every round is one Runge-Kutta attempt (dp54, MicroMagneticsStepSizeController)
for every instance still running, issued as grouped launches replayed from CUDA graphs.  A relax
instance (t_end = 0) stops at the first accepted step, at a multiple of `check_every_nth_step`,
whose state has max |m x H_eff| / Ms below `max_torque`; a timed instance stops at t_end.  Instances
live in slots and can be added and removed between calls.  The reference has no batched form;
each instance follows the reference's single-world semantics.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import check, lib


@dataclass
class Instance:
    """A box of nx*ny*nz cells of size delta [m]; mask (optional, (N,) 0/1, x fastest) marks the
    material cells, which carry Ms [A/m], A [J/m] and alpha."""
    dims: tuple
    delta: tuple
    Ms: float
    A: float
    alpha: float
    mask: Optional[np.ndarray] = None
    H_ext: tuple = (0.0, 0.0, 0.0)
    H_pulse: tuple = (0.0, 0.0, 0.0)
    pulse_rise: float = 0.0
    t_end: float = 0.0

    def to_c(self) -> "_lib.mm_batch_instance":
        a = _lib.mm_batch_instance()
        a.nx, a.ny, a.nz = (int(v) for v in self.dims)
        a.dx, a.dy, a.dz = (float(v) for v in self.delta)
        a.Ms, a.A, a.alpha = float(self.Ms), float(self.A), float(self.alpha)
        for k in range(3):
            a.H_ext[k] = float(self.H_ext[k])
            a.H_pulse[k] = float(self.H_pulse[k])
        a.pulse_rise, a.t_end = float(self.pulse_rise), float(self.t_end)
        return a

    def mask_bytes(self) -> np.ndarray:
        m = np.ones(self.n, dtype=np.uint8) if self.mask is None else np.asarray(self.mask, dtype=np.uint8).reshape(-1)
        if m.size != self.n:
            raise ValueError(f"mask has {m.size} cells, expected {self.n}")
        return np.ascontiguousarray(m)

    def device_bytes(self, precision: str = "f32"):
        """(resident, transient) device bytes of this instance in a batch."""
        r, t = ctypes.c_size_t(), ctypes.c_size_t()
        a = self.to_c()
        check(lib().mm_batch_instance_bytes(ctypes.byref(a), _lib.MM_F32 if precision == "f32" else _lib.MM_F64,
                                            ctypes.byref(r), ctypes.byref(t)))
        return r.value, t.value

    @property
    def n(self) -> int:
        return int(np.prod(self.dims))


class Batch:
    def __init__(self, instances: Sequence[Instance] = (), precision: str = "f32", eps_abs: float = 1e-3,
                 eps_rel: float = 1e-4, h0: float = 1e-13, max_torque: float = 1e-4,
                 check_every_nth_step: int = 1):
        self.precision = precision
        cfg = _lib.mm_batch_config(_lib.MM_F32 if precision == "f32" else _lib.MM_F64, float(eps_abs),
                                   float(eps_rel), float(h0), float(max_torque), int(check_every_nth_step))
        h = ctypes.c_void_p()
        check(lib().mm_batch_create(ctypes.byref(h), ctypes.byref(cfg), 0, None, None, None))
        self._h = h
        self.instances = {}
        for q in instances:
            self.add(q)

    @property
    def count(self) -> int:
        return len(self.instances)

    def add(self, q: Instance, M=None) -> int:
        """Adds an instance in a free slot (returns the slot); with M it starts in the next round."""
        a = q.to_c()
        mask = q.mask_bytes()
        slot = ctypes.c_int(-1)
        check(lib().mm_batch_add(self._h, ctypes.byref(a), mask.ctypes.data_as(ctypes.c_void_p), ctypes.byref(slot),
                                 None))
        self.instances[slot.value] = q
        if M is not None:
            self.set_M(slot.value, M)
        return slot.value

    def remove(self, slot: int) -> None:
        check(lib().mm_batch_remove(self._h, int(slot)))
        del self.instances[slot]

    def stop(self, slot: int) -> None:
        check(lib().mm_batch_stop(self._h, int(slot), None))

    def set_M(self, index: int, M) -> None:
        """M of instance `index`, (3, N) or (3N,) in A/m (normalised to Ms in the material), or
        the bytes of an OMF file of the instance's mesh."""
        if isinstance(M, (bytes, bytearray, memoryview)):
            from . import omf
            h, v = omf.parse(bytes(M))
            if (h.xnodes, h.ynodes, h.znodes) != tuple(self.instances[index].dims):
                raise ValueError(f"OMF field of {(h.xnodes, h.ynodes, h.znodes)} cells for an instance of "
                                 f"{tuple(self.instances[index].dims)}")
            v = v.reshape(-1)
        else:
            v = torch.as_tensor(M, dtype=torch.float64).reshape(-1).cuda().contiguous()
        check(lib().mm_batch_set_M(self._h, int(index), ctypes.c_void_p(v.data_ptr()), None))
        torch.cuda.current_stream().synchronize()

    def get_M(self, index: int) -> torch.Tensor:
        out = torch.empty(3 * self.instances[index].n, dtype=torch.float64, device="cuda")
        check(lib().mm_batch_get_M(self._h, int(index), ctypes.c_void_p(out.data_ptr()), None))
        torch.cuda.current_stream().synchronize()
        return out.view(3, -1)

    def relax(self, max_rounds: int = 1_000_000, check_interval: int = 16) -> int:
        """Runs rounds until every instance stopped (or max_rounds); returns the rounds run."""
        rounds = ctypes.c_longlong(0)
        check(lib().mm_batch_relax(self._h, int(max_rounds), int(check_interval), ctypes.byref(rounds), None))
        return rounds.value

    def results(self) -> list:
        """One dict per slot (status -1 for a free slot)."""
        k = lib().mm_batch_slot_count(self._h)
        out = (_lib.mm_batch_result * max(k, 1))()
        check(lib().mm_batch_results(self._h, out, None))
        return [{f: getattr(r, f) for f, _ in _lib.mm_batch_result._fields_} for r in out[:k]]

    def launches_per_round(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        check(lib().mm_batch_launches_per_round(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().mm_batch_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
