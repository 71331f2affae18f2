"""Batched relaxations over the C ABI (`mm_batch_*`).

Many independent boxes of uneven size (each with its own mask, Ms, A and alpha) relax in lock
step: every round is one Runge-Kutta attempt (dp54, MicroMagneticsStepSizeController) for every
instance still running, issued as grouped launches replayed from CUDA graphs.  An instance stops
at the first accepted step, at a multiple of `check_every_nth_step`, whose state has
max |m x H_eff| / Ms below `max_torque`.  The reference has no batched form; each instance follows
the reference's single-world semantics (condition.py's relax criterion replaced by the torque).
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

    @property
    def n(self) -> int:
        return int(np.prod(self.dims))


class Batch:
    def __init__(self, instances: Sequence[Instance], precision: str = "f32", eps_abs: float = 1e-3,
                 eps_rel: float = 1e-4, h0: float = 1e-13, max_torque: float = 1e-4,
                 check_every_nth_step: int = 1):
        self.instances = list(instances)
        self.count = len(self.instances)
        arr = (_lib.mm_batch_instance * self.count)()
        masks = []
        for i, q in enumerate(self.instances):
            a = arr[i]
            a.nx, a.ny, a.nz = (int(v) for v in q.dims)
            a.dx, a.dy, a.dz = (float(v) for v in q.delta)
            a.Ms, a.A, a.alpha = float(q.Ms), float(q.A), float(q.alpha)
            m = np.ones(q.n, dtype=np.uint8) if q.mask is None else np.asarray(q.mask, dtype=np.uint8).reshape(-1)
            if m.size != q.n:
                raise ValueError(f"instance {i}: mask has {m.size} cells, expected {q.n}")
            masks.append(m)
        self._masks = np.ascontiguousarray(np.concatenate(masks))
        cfg = _lib.mm_batch_config(_lib.MM_F32 if precision == "f32" else _lib.MM_F64, float(eps_abs),
                                   float(eps_rel), float(h0), float(max_torque), int(check_every_nth_step))
        h = ctypes.c_void_p()
        check(lib().mm_batch_create(ctypes.byref(h), ctypes.byref(cfg), self.count, arr,
                                    self._masks.ctypes.data_as(ctypes.c_void_p), None))
        self._h = h

    def set_M(self, index: int, M) -> None:
        """M of instance `index`, (3, N) or (3N,) in A/m (normalised to Ms in the material)."""
        v = torch.as_tensor(M, dtype=torch.float64).reshape(-1).cuda().contiguous()
        check(lib().mm_batch_set_M(self._h, int(index), ctypes.c_void_p(v.data_ptr()), None))
        torch.cuda.synchronize()

    def get_M(self, index: int) -> torch.Tensor:
        out = torch.empty(3 * self.instances[index].n, dtype=torch.float64, device="cuda")
        check(lib().mm_batch_get_M(self._h, int(index), ctypes.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        return out.view(3, -1)

    def relax(self, max_rounds: int = 1_000_000, check_interval: int = 16) -> int:
        """Runs rounds until every instance stopped (or max_rounds); returns the rounds run."""
        rounds = ctypes.c_longlong(0)
        check(lib().mm_batch_relax(self._h, int(max_rounds), int(check_interval), ctypes.byref(rounds), None))
        return rounds.value

    def results(self) -> list:
        out = (_lib.mm_batch_result * self.count)()
        check(lib().mm_batch_results(self._h, out, None))
        return [{f: getattr(r, f) for f, _ in _lib.mm_batch_result._fields_} for r in out]

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
