"""Oracle — TEST INFRASTRUCTURE ONLY.

CPU checkers for the parity tests, smoke() and bench.py's CPU-baseline leg; never part of the
product (micromagnum_b200 does not import this package).

  Restatement : liboracle.so built from oracle.c (the project's C restatement of the reference
                algorithms, each function citing the reference file:line it follows).
  Reference   : _ref/libmmref.so, the reference's own CPU C++ (MicroMagnum 0.2rc3,
                src/magneto/...) compiled in place by oracle/Makefile, wrapped by ref_shim.cpp.

All arrays are numpy float64 in the reference layout: vector fields SoA with shape (3, N),
N = nx*ny*nz, x fastest; the demag tensor is flat (ez, ey, ex, 6) == Matrix(Shape(6,ex,ey,ez)).
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmmref.so")
# Root of a MicroMagnum checkout (the directory holding src/magneto and src/magnum): from the
# environment, else the checkout the last build compiled _ref/libmmref.so from (recorded in
# _ref/checkout by build()).  Only needed to compile _ref/libmmref.so and by the tests that run the
# reference's Python package; absent on machines without a checkout.
REF_RECORD = os.path.join(HERE, "_ref", "checkout")


def _checkout():
    root = os.environ.get("MMB200_REFERENCE")
    if not root and os.path.exists(REF_RECORD):
        with open(REF_RECORD) as f:
            root = f.read().strip()
    return root if root and os.path.isdir(os.path.join(root, "src")) else None


REF_ROOT = _checkout()
REF_SRC = os.path.join(REF_ROOT, "src", "magneto") if REF_ROOT else None

_dp = ctypes.POINTER(ctypes.c_double)
_D = ctypes.c_double


def build(with_ref: bool = True) -> None:
    """Compile liboracle.so, and _ref/libmmref.so when the reference tree is present."""
    if with_ref and REF_SRC and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True, stdout=subprocess.DEVNULL)
        with open(REF_RECORD, "w") as f:
            f.write(REF_ROOT + "\n")
    else:
        subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=subprocess.DEVNULL)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _f(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


_O = None
_R = None


def restated():
    global _O
    if _O is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        _O = ctypes.CDLL(ORACLE_SO)
        _O.or_exchange.restype = _D
        _O.or_uniaxial_anisotropy.restype = _D
        _O.or_cubic_anisotropy.restype = _D
        _O.or_scaled_abs_max.restype = _D
        _O.or_solver_create.restype = ctypes.c_void_p
        for name in ("or_solver_destroy", "or_solver_set_M", "or_solver_get_M", "or_solver_eval",
                     "or_solver_step", "or_solver_run", "or_solver_stats", "or_solver_attempt"):
            getattr(_O, name).argtypes = None
        _O.or_set_threads(os.cpu_count() or 1)
    return _O


def reference():
    """The reference's own CPU implementation (None if it could not be built)."""
    global _R
    if _R is None:
        if not os.path.exists(REF_SO):
            if REF_SRC and os.path.isdir(REF_SRC):
                build(with_ref=True)
            else:
                return None
        _R = ctypes.CDLL(REF_SO)
        for name in ("mmref_exchange", "mmref_uniaxial_anisotropy", "mmref_cubic_anisotropy",
                     "mmref_scaled_abs_max", "mmref_rk_adjust_stepsize"):
            getattr(_R, name).restype = _D
        _R.mmref_round_tensor_dimension.restype = ctypes.c_int
    return _R


def have_reference() -> bool:
    return reference() is not None


def set_threads(n: int) -> None:
    restated().or_set_threads(int(n))


# ---- thin numpy wrappers (impl: "oracle" restatement or "ref" compiled reference) ------------
def _lib(impl):
    return restated() if impl == "oracle" else reference()


def exchange(nx, ny, nz, dx, dy, dz, Ms, A, M, pbc=(0, 0, 0), impl="oracle"):
    H = np.zeros(3 * nx * ny * nz)
    Ms, A, M = _f(Ms), _f(A), _f(M).reshape(-1)
    fn = _lib(impl).or_exchange if impl == "oracle" else _lib(impl).mmref_exchange
    e = fn(nx, ny, nz, _D(dx), _D(dy), _D(dz), int(pbc[0]), int(pbc[1]), int(pbc[2]), _p(Ms), _p(A), _p(M), _p(H))
    return H.reshape(3, -1), e


def uniaxial_anisotropy(axis, k, Ms, M, impl="oracle"):
    axis, k, Ms, M = _f(axis).reshape(-1), _f(k), _f(Ms), _f(M).reshape(-1)
    n = Ms.size
    H = np.zeros(3 * n)
    if impl == "oracle":
        e = restated().or_uniaxial_anisotropy(ctypes.c_size_t(n), _p(axis), _p(k), _p(Ms), _p(M), _p(H))
    else:
        e = reference().mmref_uniaxial_anisotropy(n, 1, 1, _p(axis), _p(k), _p(Ms), _p(M), _p(H))
    return H.reshape(3, -1), e


def cubic_anisotropy(axis1, axis2, k, Ms, M, impl="oracle"):
    a1, a2, k, Ms, M = _f(axis1).reshape(-1), _f(axis2).reshape(-1), _f(k), _f(Ms), _f(M).reshape(-1)
    n = Ms.size
    H = np.zeros(3 * n)
    if impl == "oracle":
        e = restated().or_cubic_anisotropy(ctypes.c_size_t(n), _p(a1), _p(a2), _p(k), _p(Ms), _p(M), _p(H))
    else:
        e = reference().mmref_cubic_anisotropy(n, 1, 1, _p(a1), _p(a2), _p(k), _p(Ms), _p(M), _p(H))
    return H.reshape(3, -1), e


def llge(f1, f2, M, H, impl="oracle"):
    f1, f2, M, H = _f(f1), _f(f2), _f(M).reshape(-1), _f(H).reshape(-1)
    n = f1.size
    dM = np.zeros(3 * n)
    if impl == "oracle":
        restated().or_llge(ctypes.c_size_t(n), _p(f1), _p(f2), _p(M), _p(H), _p(dM))
    else:
        reference().mmref_llge(n, 1, 1, _p(f1), _p(f2), _p(M), _p(H), _p(dM))
    return dM.reshape(3, -1)


def fdm_zhangli(nx, ny, nz, dx, dy, dz, do_precess, P, xi, Ms, alpha, j, M, impl="oracle"):
    P, xi, Ms, alpha = _f(P), _f(xi), _f(Ms), _f(alpha)
    j, M = _f(j).reshape(-1), _f(M).reshape(-1)
    dM = np.zeros(3 * nx * ny * nz)
    fn = restated().or_fdm_zhangli if impl == "oracle" else reference().mmref_fdm_zhangli
    fn(nx, ny, nz, _D(dx), _D(dy), _D(dz), int(do_precess), _p(P), _p(xi), _p(Ms), _p(alpha), _p(j), _p(M), _p(dM))
    return dM.reshape(3, -1)


def scaled_abs_max(M, scale, impl="oracle"):
    M, scale = _f(M).reshape(-1), _f(scale)
    if impl == "oracle":
        return restated().or_scaled_abs_max(ctypes.c_size_t(scale.size), _p(M), _p(scale))
    return reference().mmref_scaled_abs_max(scale.size, 1, 1, _p(M), _p(scale))


def normalize(Ms, M, float_norm=True, impl="oracle"):
    Ms, M = _f(Ms), _f(M).reshape(-1).copy()
    if impl == "oracle":
        restated().or_normalize(ctypes.c_size_t(Ms.size), _p(Ms), _p(M), int(float_norm))
    else:
        reference().mmref_normalize(Ms.size, 1, 1, _p(Ms), _p(M))
    return M.reshape(3, -1)


def round_tensor_dimension(dim, periodic=False, padding=2):
    return int(restated().or_round_tensor_dimension(int(dim), int(periodic), int(padding)))


def padded(nx, ny, nz, padding=2):
    return tuple(round_tensor_dimension(d, False, padding) for d in (nx, ny, nz))


def demag_tensor(nx, ny, nz, dx, dy, dz, padding=2, impl="oracle", pbc=(0, 0, 0), repeat=1):
    """Negated Newell tensor; impl "oracle": exact (binary128) Newell, "ref": the reference's
    calculateDemagTensor (incl. its far-field series and periodic images)."""
    if impl == "ref":
        R = reference()
        ex, ey, ez = (R.mmref_round_tensor_dimension(d, int(p), padding) for d, p in zip((nx, ny, nz), pbc))
        N = np.zeros(6 * ex * ey * ez)
        R.mmref_demag_tensor(nx, ny, nz, _D(dx), _D(dy), _D(dz), int(pbc[0]), int(pbc[1]), int(pbc[2]),
                             int(repeat), ex, ey, ez, _p(N))
        return N, (ex, ey, ez)
    ex, ey, ez = padded(nx, ny, nz, padding)
    N = np.zeros(6 * ex * ey * ez)
    restated().or_demag_tensor(nx, ny, nz, _D(dx), _D(dy), _D(dz), ex, ey, ez, _p(N))
    return N, (ex, ey, ez)


def conv(N, dims, pdims, M, method="direct", impl="oracle"):
    nx, ny, nz = dims
    ex, ey, ez = pdims
    N, M = _f(N).reshape(-1), _f(M).reshape(-1)
    H = np.zeros_like(M)
    if impl == "ref":
        reference().mmref_conv_simple(_p(N), nx, ny, nz, ex, ey, ez, _p(M), _p(H))
    elif method == "direct":
        restated().or_conv_direct(_p(N), nx, ny, nz, ex, ey, ez, _p(M), _p(H))
    else:
        restated().or_conv_fft(_p(N), nx, ny, nz, ex, ey, ez, _p(M), _p(H))
    return H.reshape(3, -1)


class Solver:
    """The reference's Runge-Kutta solve loop restated in C (oracle.c or_solver_*)."""

    TABLEAUS = {"rkf45": 0, "cc45": 1, "dp54": 2, "rk23": 3}
    TERMS = {"demag": 1, "exchange": 2, "uniaxial": 4, "cubic": 8, "zhangli": 16, "zeeman": 32}

    class _Cfg(ctypes.Structure):
        _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                    ("dx", _D), ("dy", _D), ("dz", _D), ("tableau", ctypes.c_int), ("terms", ctypes.c_int),
                    ("do_precess", ctypes.c_int), ("zl_do_precess", ctypes.c_int),
                    ("eps_abs", _D), ("eps_rel", _D), ("h0", _D),
                    ("H_ext", _D * 3), ("H_pulse", _D * 3), ("pulse_rise", _D),
                    ("fsal_reuse_after_reject", ctypes.c_int), ("float_norm", ctypes.c_int),
                    ("use_fft", ctypes.c_int), ("pbc", ctypes.c_int * 3)]

    def __init__(self, dims, delta, Ms, A=0.0, alpha=0.0, k_uniaxial=0.0, k_cubic=0.0,
                 axis1=(0, 0, 0), axis2=(0, 0, 0), P=0.0, xi=0.0, j=(0, 0, 0),
                 terms=("demag", "exchange"), evolver="dp54", eps_abs=1e-3, eps_rel=1e-4, h0=1e-13,
                 do_precess=True, zl_do_precess=True, H_ext=(0, 0, 0), H_pulse=(0, 0, 0),
                 pulse_rise=0.0, fsal_reuse_after_reject=True, float_norm=True, use_fft=None,
                 tensor=None, padding=2, pbc=(0, 0, 0)):
        self.L = restated()
        nx, ny, nz = dims
        n = nx * ny * nz
        self.n = n
        c = self._Cfg()
        c.nx, c.ny, c.nz = nx, ny, nz
        c.dx, c.dy, c.dz = delta
        c.tableau = self.TABLEAUS[evolver]
        t = 0
        for name in terms:
            t |= self.TERMS[name]
        if any(H_ext) or any(H_pulse):
            t |= 32
        c.terms = t
        c.do_precess, c.zl_do_precess = int(do_precess), int(zl_do_precess)
        c.eps_abs, c.eps_rel, c.h0 = eps_abs, eps_rel, h0
        for q in range(3):
            c.H_ext[q], c.H_pulse[q] = H_ext[q], H_pulse[q]
        c.pulse_rise = pulse_rise
        c.fsal_reuse_after_reject = int(fsal_reuse_after_reject)
        c.float_norm = int(float_norm)
        c.use_fft = int(use_fft if use_fft is not None else n > 8192)
        for q in range(3):
            c.pbc[q] = int(bool(pbc[q]))
        self.cfg = c

        def cell(v):
            return np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), (n,)))

        def vec(v):
            v = np.asarray(v, dtype=np.float64)
            if v.size == 3:
                v = np.repeat(v.reshape(3, 1), n, axis=1)
            return np.ascontiguousarray(v.reshape(3, n))

        self._keep = [cell(Ms), cell(A), cell(alpha), cell(k_uniaxial), cell(k_cubic), vec(axis1),
                      vec(axis2), cell(P), cell(xi), vec(j)]
        if "demag" in terms:
            if tensor is None:
                tensor, pd = demag_tensor(nx, ny, nz, *delta, padding=padding)
            else:
                tensor, pd = tensor
            self._keep.append(_f(tensor))
            tp, (ex, ey, ez) = _p(self._keep[-1]), pd
        else:
            tp, ex, ey, ez = None, 1, 1, 1
        self.h = self.L.or_solver_create(ctypes.byref(c), *[_p(a) for a in self._keep[:10]], tp, ex, ey, ez)

    @property
    def M(self):
        out = np.zeros(3 * self.n)
        self.L.or_solver_get_M(ctypes.c_void_p(self.h), _p(out))
        return out.reshape(3, -1)

    @M.setter
    def M(self, v):
        v = np.asarray(v, dtype=np.float64)
        if v.size == 3:
            v = np.repeat(v.reshape(3, 1), self.n, axis=1)
        v = _f(v).reshape(-1)
        self.L.or_solver_set_M(ctypes.c_void_p(self.h), _p(v))

    def step(self, t_max=1e100):
        self.L.or_solver_step(ctypes.c_void_p(self.h), _D(t_max))

    def solve(self, t_end, sample_dt=None):
        if sample_dt:
            cap = int(t_end / sample_dt) + 4
            ts, ms = np.zeros(cap), np.zeros((cap, 3))
            cnt = self.L.or_solver_run(ctypes.c_void_p(self.h), _D(t_end), _D(sample_dt), _p(ts), _p(ms), cap)
            return ts[:cnt], ms[:cnt]
        self.L.or_solver_run(ctypes.c_void_p(self.h), _D(t_end), _D(0.0), None, None, 0)
        return None

    def attempt(self, h):
        self.L.or_solver_attempt(ctypes.c_void_p(self.h), _D(h))

    def eval(self):
        H, dM, Hd = np.zeros(3 * self.n), np.zeros(3 * self.n), np.zeros(3 * self.n)
        self.L.or_solver_eval(ctypes.c_void_p(self.h), _p(H), _p(dM), _p(Hd))
        return H.reshape(3, -1), dM.reshape(3, -1), Hd.reshape(3, -1)

    @property
    def stats(self):
        o = np.zeros(6)
        self.L.or_solver_stats(ctypes.c_void_p(self.h), _p(o))
        return dict(t=o[0], h=o[1], h_next=o[2], steps=int(o[3]), attempts=int(o[4]), rejected=int(o[5]))

    def relax_norms(self):
        """(state.dMdt.absMax(), state.M.absMax(), max |m x H| / Ms) at the current state."""
        H, dM, _ = self.eval()
        M = self.M
        Ms = np.sqrt((M ** 2).sum(0))
        m = np.divide(M, Ms, out=np.zeros_like(M), where=Ms > 0)
        tq = np.sqrt((np.cross(m.T, H.T) ** 2).sum(1))
        tq = np.divide(tq, Ms, out=np.zeros_like(tq), where=Ms > 0)
        return float(np.sqrt((dM ** 2).sum(0)).max()), float(Ms.max()), float(tq.max())

    def relax(self, max_degree_per_ns=1.0, check_every_nth_step=100, max_steps=None):
        """Solver.solve(condition.Relaxed(...)) restated: condition.py:169-200 checks every nth
        step (state.step % n == 0) and calls the state relaxed when deg/ns (from
        landau_lifshitz_gilbert.py:127-131, with the last step size state.h) is <= the limit and
        below its value at the previous check; solver.py:117-122 checks before each step.
        Returns (relaxed, last deg/ns)."""
        last, taken = None, 0
        while True:
            st = self.stats
            if st["steps"] % check_every_nth_step == 0:
                dmdt, mmax, _ = self.relax_norms()
                deg = 1e-9 * math.degrees(math.atan2(dmdt * st["h"], mmax)) / st["h"]
                done = last is not None and deg < last and deg <= max_degree_per_ns
                last = deg
                if done:
                    return True, deg
            if max_steps is not None and taken >= max_steps:
                return False, last
            self.step()
            taken += 1

    def __del__(self):
        if getattr(self, "h", None):
            self.L.or_solver_destroy(ctypes.c_void_p(self.h))
            self.h = None
