"""The fused solver: the B200 replacement for MicroMagnum's per-stage Python/C++ loop.

``Solver`` plays the part of ``create_solver(world, [StrayField, ExchangeField, ...],
evolver="dp54", eps_abs=..., eps_rel=...)`` (magnum/micromagnetics/create_solver.py:27-64) and
of ``solver.step()`` / ``solver.solve(condition.Time(t))`` with an ``EveryNthSecond`` sampling
handler (magnum/solver/solver.py:76-139).  The state, the stage vectors, the demag spectra and
the step controller stay on the GPU; a call advances by whole Runge-Kutta steps with the
reference's semantics (runge_kutta.py:47-137, micro_magnetics_stepsize_controller.py:35-73).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Iterable, Optional, Sequence

import numpy as np
import torch

from . import _lib
from . import magneto as _magneto
from ._lib import check, lib

TERMS = {
    "demag": _lib.MM_TERM_DEMAG, "stray": _lib.MM_TERM_DEMAG, "exchange": _lib.MM_TERM_EXCHANGE,
    "uniaxial": _lib.MM_TERM_UNIAXIAL, "cubic": _lib.MM_TERM_CUBIC,
    "zhangli": _lib.MM_TERM_ZHANGLI, "zeeman": _lib.MM_TERM_ZEEMAN,
}
TABLEAUS = {"rkf45": _lib.MM_RK_RKF45, "cc45": _lib.MM_RK_CC45, "dp54": _lib.MM_RK_DP54,
            "rk23": _lib.MM_RK_RK23}


class RectangularMesh(_magneto.RectangularMesh):
    """magnum.mesh.RectangularMesh (src/magnum/mesh/rectangular_mesh.py:22-35): the mesh from
    the number of cells and the cell size, with periodic directions ("x", "xy", ...) and their
    repetitions."""

    def __init__(self, num_nodes, cell_size, periodic_bc: str = "", periodic_repeat=None):
        nx, ny, nz = (int(v) for v in num_nodes)
        dx, dy, dz = (float(v) for v in cell_size)
        super().__init__(nx, ny, nz, dx, dy, dz, periodic_bc, periodic_repeat or -1)


@dataclass
class Material:
    """Per-region parameters (the reference's Material / per-cell parameter fields)."""
    Ms: float = 0.0
    A: float = 0.0
    alpha: float = 0.0
    k_uniaxial: float = 0.0
    k_cubic: float = 0.0
    axis1: Sequence[float] = (0.0, 0.0, 0.0)
    axis2: Sequence[float] = (0.0, 0.0, 0.0)
    P: float = 0.0
    xi: float = 0.0
    j: Sequence[float] = (0.0, 0.0, 0.0)

    def to_c(self) -> _lib.mm_material:
        m = _lib.mm_material()
        m.Ms, m.A, m.alpha = self.Ms, self.A, self.alpha
        m.k_uniaxial, m.k_cubic, m.P, m.xi = self.k_uniaxial, self.k_cubic, self.P, self.xi
        for q in range(3):
            m.axis1[q], m.axis2[q], m.j[q] = self.axis1[q], self.axis2[q], self.j[q]
        return m


def _stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Solver:
    """Micromagnetic solver on one GPU.

    mesh       : RectangularMesh; its periodic directions make the exchange stencil wrap around
                 and the demag tensor periodic (repetitions from the mesh)
    materials  : list of Material (<= 256); regions selects one per cell
    regions    : None (all cells material 0) or uint8 array of nx*ny*nz region indices
    terms      : iterable of "demag", "exchange", "uniaxial", "cubic", "zhangli", "zeeman"
    precision  : "f64" (plain double, the reference's -G) or "f32" (float with compensated state)
    evolver    : "dp54", "rkf45", "cc45" or "rk23"
    tensor     : optional FP64 demag tensor (torch CUDA tensor or numpy, reference layout); by
                 default it is generated on the GPU
    """

    def __init__(self, mesh: RectangularMesh, materials: Sequence[Material], regions=None,
                 terms: Iterable[str] = ("demag", "exchange"), precision: str = "f64",
                 evolver: str = "dp54", eps_abs: float = 1e-3, eps_rel: float = 1e-4,
                 h0: float = 1e-13, do_precess: bool = True, zl_do_precess: bool = True,
                 H_ext=(0.0, 0.0, 0.0), H_pulse=(0.0, 0.0, 0.0), pulse_rise: float = 0.0,
                 padding: int = 2, tensor=None, fsal_reuse_after_reject: bool = True):
        if not torch.cuda.is_available():
            raise RuntimeError("Solver needs a CUDA device (there is no CPU implementation)")
        self.mesh = mesh
        nx, ny, nz = mesh.num_nodes
        self.n = nx * ny * nz
        cfg = _lib.mm_solver_config()
        cfg.nx, cfg.ny, cfg.nz = nx, ny, nz
        cfg.dx, cfg.dy, cfg.dz = mesh.delta
        cfg.precision = _lib.MM_F64 if precision == "f64" else _lib.MM_F32
        cfg.tableau = TABLEAUS[evolver]
        t = 0
        for name in terms:
            t |= TERMS[name]
        if any(H_ext) or any(H_pulse):
            t |= _lib.MM_TERM_ZEEMAN
        cfg.terms = t
        cfg.do_precess, cfg.zl_do_precess = int(do_precess), int(zl_do_precess)
        cfg.padding = padding
        cfg.eps_abs, cfg.eps_rel, cfg.h0 = eps_abs, eps_rel, h0
        for q in range(3):
            cfg.H_ext[q], cfg.H_pulse[q] = H_ext[q], H_pulse[q]
        cfg.pulse_rise = pulse_rise
        cfg.fsal_reuse_after_reject = int(fsal_reuse_after_reject)
        pbc, reps = mesh.periodic_bc
        for q, axis in enumerate("xyz"):
            cfg.pbc[q] = int(axis in pbc)
        cfg.pbc_repeat = int(reps) if pbc else 0
        self.cfg = cfg
        self.precision = precision
        mats = (_lib.mm_material * len(materials))(*[m.to_c() for m in materials])
        self._Ms = np.array([m.Ms for m in materials])
        reg_ptr = None
        self._regions = None
        if regions is not None:
            self._regions = np.ascontiguousarray(np.asarray(regions, dtype=np.uint8).reshape(-1))
            if self._regions.size != self.n:
                raise ValueError("regions must have nx*ny*nz entries")
            reg_ptr = self._regions.ctypes.data_as(ctypes.c_void_p)
        tptr = None
        if tensor is not None:
            tt = torch.as_tensor(tensor, dtype=torch.float64).reshape(-1).cuda().contiguous()
            self._tensor_keep = tt
            tptr = ctypes.c_void_p(tt.data_ptr())
        h = ctypes.c_void_p()
        check(lib().mm_solver_create(ctypes.byref(h), ctypes.byref(cfg), len(materials), mats,
                                     reg_ptr, tptr, _stream_ptr()))
        self._h = h
        self._tensor_keep = None

    # ---- state ---------------------------------------------------------------------------------
    @property
    def M(self) -> torch.Tensor:
        """Magnetisation [A/m] as a (3, N) float64 CUDA tensor (a copy)."""
        out = torch.empty(3 * self.n, dtype=torch.float64, device="cuda")
        check(lib().mm_solver_get_M(self._h, ctypes.c_void_p(out.data_ptr()), _stream_ptr()))
        return out.view(3, self.n)

    @M.setter
    def M(self, value) -> None:
        """Assign M (normalised to Ms per cell, like LandauLifshitzGilbert.update("M"));
        resets time and step counters."""
        v = torch.as_tensor(value, dtype=torch.float64).reshape(-1)
        if v.numel() == 3:
            v = v.view(3, 1).expand(3, self.n).reshape(-1)
        v = v.cuda().contiguous()
        check(lib().mm_solver_set_M(self._h, ctypes.c_void_p(v.data_ptr()), _stream_ptr()))
        torch.cuda.current_stream().synchronize()

    def load_M_device(self, M_device: torch.Tensor) -> None:
        """Replace the state by M (a 3N float64 CUDA tensor, A/m) without resetting time, step
        size or counters (stream-ordered)."""
        check(lib().mm_solver_load_M(self._h, ctypes.c_void_p(M_device.data_ptr()), _stream_ptr()))

    def read_M_device(self, out: torch.Tensor) -> None:
        """Write M (A/m) into a 3N float64 CUDA tensor (stream-ordered)."""
        check(lib().mm_solver_get_M(self._h, ctypes.c_void_p(out.data_ptr()), _stream_ptr()))

    def set_time(self, t: float, h_next: float) -> None:
        check(lib().mm_solver_set_time(self._h, t, h_next, _stream_ptr()))

    # ---- stepping ------------------------------------------------------------------------------
    def step(self, t_max: float = 1e100) -> None:
        """One accepted step (RungeKutta.evolve + finish_step)."""
        check(lib().mm_solver_step(self._h, float(t_max), _stream_ptr()))

    def solve(self, t_end: float, sample_dt: Optional[float] = None, max_samples: Optional[int] = None):
        """Advance until t >= t_end; with sample_dt, returns (times, <M>) sampled at every
        multiple of sample_dt (steps are clamped to those times, like EveryNthSecond)."""
        if sample_dt:
            cap = max_samples or int(t_end / sample_dt) + 4
            ts = np.zeros(cap)
            ms = np.zeros((cap, 3))
            cnt = ctypes.c_int(0)
            dp = ctypes.POINTER(ctypes.c_double)
            check(lib().mm_solver_run(self._h, float(t_end), float(sample_dt), ts.ctypes.data_as(dp),
                                      ms.ctypes.data_as(dp), cap, ctypes.byref(cnt), _stream_ptr()))
            return ts[:cnt.value], ms[:cnt.value]
        check(lib().mm_solver_run(self._h, float(t_end), 0.0, None, None, 0, None, _stream_ptr()))
        return None

    def attempt(self, h: float) -> None:
        """One Runge-Kutta attempt of size h without a state update (stream-ordered)."""
        check(lib().mm_solver_attempt(self._h, float(h), _stream_ptr()))

    # ---- observables ---------------------------------------------------------------------------
    def eval(self):
        """(H_eff, dM/dt, H_demag) at the current state, each (3, N) float64 CUDA tensors."""
        outs = [torch.empty(3 * self.n, dtype=torch.float64, device="cuda") for _ in range(3)]
        check(lib().mm_solver_eval(self._h, *[ctypes.c_void_p(o.data_ptr()) for o in outs], _stream_ptr()))
        return tuple(o.view(3, self.n) for o in outs)

    def average_M(self):
        out = (ctypes.c_double * 3)()
        check(lib().mm_solver_average_M(self._h, out, _stream_ptr()))
        return tuple(out)

    def relax_norms(self):
        """(max |dM/dt| [A/(m s)], max |M| [A/m], max |m x H_eff| / Ms) at the current state."""
        out = (ctypes.c_double * 3)()
        check(lib().mm_solver_relax_norms(self._h, out, _stream_ptr()))
        return tuple(out)

    def energies(self) -> dict:
        """E_stray, E_exch, E_aniso, E_ext and E_tot [J] at the current state (the reference's
        state.E_stray ... state.E_tot, landau_lifshitz_gilbert.py:103-106)."""
        out = (ctypes.c_double * 5)()
        check(lib().mm_solver_energies(self._h, out, _stream_ptr()))
        return dict(zip(("E_stray", "E_exch", "E_aniso", "E_ext", "E_tot"), out))

    @property
    def deg_per_ns(self) -> float:
        """LandauLifshitzGilbert.calculate_deg_per_ns (landau_lifshitz_gilbert.py:127-131) with the
        last step size."""
        dmdt, m, _ = self.relax_norms()
        h = self.stats["h"]
        return 1e-9 * math.degrees(math.atan2(dmdt * h, m)) / h

    def relax(self, max_degree_per_ns: float = 1.0, check_every_nth_step: int = 100,
              max_steps: Optional[int] = None) -> bool:
        """Solver.solve(condition.Relaxed(max_degree_per_ns, check_every_nth_step))
        (condition.py:169-200); returns True when relaxed (False when max_steps ran out)."""
        return self._relax(_lib.MM_RELAX_DEG_PER_NS, max_degree_per_ns, check_every_nth_step, max_steps)

    def relax_torque(self, max_torque: float = 1e-4, check_every_nth_step: int = 1,
                     max_steps: Optional[int] = None) -> bool:
        """Steps until max |m x H_eff| / Ms < max_torque (checked every nth step)."""
        return self._relax(_lib.MM_RELAX_TORQUE, max_torque, check_every_nth_step, max_steps)

    def _relax(self, criterion, threshold, every, max_steps):
        done = ctypes.c_int(0)
        last = ctypes.c_double(0.0)
        check(lib().mm_solver_relax(self._h, criterion, float(threshold), int(every),
                                    -1 if max_steps is None else int(max_steps), ctypes.byref(done),
                                    ctypes.byref(last), _stream_ptr()))
        self.last_relax_value = last.value
        return bool(done.value)

    @property
    def stats(self) -> dict:
        st = _lib.mm_solver_stats()
        check(lib().mm_solver_stats_get(self._h, ctypes.byref(st), _stream_ptr()))
        return {f: getattr(st, f) for f, _ in _lib.mm_solver_stats._fields_}

    @property
    def t(self) -> float:
        return self.stats["t"]

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().mm_solver_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
