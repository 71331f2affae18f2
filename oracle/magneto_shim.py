"""A CPU ``magneto`` module for the unchanged MicroMagnum Python package — TEST INFRASTRUCTURE ONLY.

The reference's SWIG module ``magneto_cpu`` cannot be built here (SWIG and FFTW are absent).  This
module stands in for it so that the reference's own Python layer (``magnum``: the Runge-Kutta
evolver, the step-size controllers, the module system, the state caches) runs unchanged on the
CPU, with the arithmetic done by the reference's own compiled C++ wherever that builds
(oracle/_ref/libmmref.so: exchange, anisotropy, LLG, Zhang-Li, demag tensor, scaled_abs_max,
normalize, the direct convolution) and by the oracle's restated FFT convolution for
SymmetricMatrixVectorConvolution_FFT (the reference's needs FFTW).  The containers follow matty's
CPU semantics (src/magneto/matrix/matty.inc.i): SoA double arrays, x fastest, a uniform state
with one value until a single cell is written.

Used by tests/test_oracle.py to run magnum's RungeKutta.evolve/apply (runge_kutta.py:47-137) and
MicroMagneticsStepSizeController (micro_magnetics_stepsize_controller.py:35-73) over the
reference's kernels and compare them with the oracle's C restatement of the same loop
(oracle.Solver); the product never imports this module.
"""
from __future__ import annotations

import ctypes
import itertools
import math

import numpy as np

from . import _D, _f, _p, conv, reference

CUDA_DISABLED, CUDA_32, CUDA_64 = 0, 1, 2
PADDING_DISABLE, PADDING_ROUND_2, PADDING_ROUND_4 = 0, 1, 2
PADDING_ROUND_8, PADDING_ROUND_POT, PADDING_SMALL_PRIME_FACTORS = 3, 4, 5
INFINITY_NONE = 0
OMF_FORMAT_ASCII, OMF_FORMAT_BINARY_4, OMF_FORMAT_BINARY_8 = 0, 1, 2
CALLS = {}  # name -> number of calls (the tests check which reference kernels ran)


def _count(name):
    CALLS[name] = CALLS.get(name, 0) + 1


def initialize(cache_dir=""):
    pass


def deinitialize(cache_dir=""):
    pass


def enableCuda(mode=CUDA_DISABLED, device=-1):
    if mode != CUDA_DISABLED:
        raise RuntimeError("the CPU stand-in has no CUDA")


def isCudaEnabled():
    return False


def isCuda64Enabled():
    return False


def haveCudaSupport():
    return False


def enableProfiling(yes=True):
    pass


def isProfilingEnabled():
    return False


def printProfilingReport():
    pass


def haveFFTWThreads():
    return False


def setFFTWThreads(n):
    pass


def setDebugCallback(cb):
    pass


class Shape(tuple):
    def __new__(cls, *dims):
        if len(dims) == 1 and isinstance(dims[0], (tuple, list)):
            dims = tuple(dims[0])
        return super().__new__(cls, tuple(int(d) for d in dims))

    def getNumEl(self):
        return int(math.prod(self)) if len(self) else 0

    def getDim(self, d):
        return self[d]

    def getRank(self):
        return len(self)


class _Base:
    NCOMP = 1

    def __init__(self, shape):
        if isinstance(shape, _Base):
            self._shape, self._n, self._u = shape._shape, shape._n, shape._u
            self._a = None if shape._a is None else shape._a.copy()
            return
        self._shape = Shape(shape)
        self._n = self._shape.getNumEl()
        self._u = 0.0 if self.NCOMP == 1 else (0.0, 0.0, 0.0)
        self._a = None

    @property
    def arr(self):
        """The SoA double array (materialised from the uniform value on first use)."""
        if self._a is None:
            if self.NCOMP == 1:
                self._a = np.full(self._n, float(self._u))
            else:
                self._a = np.repeat(np.asarray(self._u, dtype=np.float64), self._n)
        return self._a

    def isUniform(self):
        return self._a is None

    def size(self):
        return self._n

    def dimX(self):
        return self._shape[0]

    def dimY(self):
        return self._shape[1] if len(self._shape) > 1 else 1

    def dimZ(self):
        return self._shape[2] if len(self._shape) > 2 else 1

    shape = property(lambda self: tuple(self._shape))

    def getShape(self):
        return self._shape

    @property
    def uniform_value(self):
        if not self.isUniform():
            raise ValueError("not uniform")
        return self._u

    def getUniformValue(self):
        return self.uniform_value

    def clear(self):
        self.fill(0.0 if self.NCOMP == 1 else (0.0, 0.0, 0.0))

    def assign(self, other):
        if other.isUniform():
            self._u, self._a = other._u, None
        else:
            self._a = other.arr.copy()

    def add(self, other, scale=1.0):
        # CPUDevice add: a[i] += b[i] * scale (uniform operands added as values)
        if self.isUniform() and other.isUniform():
            if self.NCOMP == 1:
                self._u = self._u + other._u * scale
            else:
                self._u = tuple(a + b * scale for a, b in zip(self._u, other._u))
        else:
            self.arr[:] = self.arr + other.arr * scale

    def scale(self, f):
        if self.isUniform():
            self._u = self._u * f if self.NCOMP == 1 else tuple(u * f for u in self._u)
        else:
            self.arr[:] = self.arr * f

    def _lin(self, idx):
        if len(idx) == 1:
            return int(idx[0])
        x, y, z = idx
        return int(x) + self.dimX() * (int(y) + self.dimY() * int(z))


class Matrix(_Base):
    def fill(self, v):
        self._u, self._a = float(v), None

    def get(self, *idx):
        return float(self._u) if self.isUniform() else float(self.arr[self._lin(idx)])

    def set(self, *args):
        *idx, v = args
        if self.isUniform() and float(v) == self._u:
            return
        self.arr[self._lin(idx)] = float(v)

    def average(self):
        return float(self._u) if self.isUniform() else float(self.arr.mean())

    def sum(self):
        return float(self._u) * self._n if self.isUniform() else float(self.arr.sum())


class VectorMatrix(_Base):
    NCOMP = 3

    def fill(self, v):
        self._u, self._a = tuple(float(x) for x in v), None

    def get(self, *idx):
        if self.isUniform():
            return self._u
        i = self._lin(idx)
        return tuple(float(self.arr[i + c * self._n]) for c in range(3))

    def set(self, *args):
        *idx, v = args
        v = tuple(float(x) for x in v)
        if self.isUniform() and v == self._u:
            return
        i = self._lin(idx)
        for c in range(3):
            self.arr[i + c * self._n] = v[c]

    def from_numpy(self, a):
        self._a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1)).copy()

    def normalize(self, length):
        _count("normalize")
        ms = length.arr if isinstance(length, Matrix) else np.full(self._n, float(length))
        reference().mmref_normalize(self._n, 1, 1, _p(_f(ms)), _p(self.arr))

    def absMax(self):
        v = self.arr.reshape(3, -1)
        return float(np.sqrt((v * v).sum(0)).max())

    def dotSum(self, other):
        return float((self.arr * other.arr).sum())

    def average(self):
        return tuple(self.arr.reshape(3, -1).mean(1).tolist())


class RectangularMesh:
    def __init__(self, nx, ny, nz, dx, dy, dz, pbc="", pbc_reps=-1):
        self.nx, self.ny, self.nz, self.dx, self.dy, self.dz = int(nx), int(ny), int(nz), dx, dy, dz
        self.pbc = pbc or ""
        if pbc_reps is None or pbc_reps == -1:
            pbc_reps = (1, 15, 3, 2)[sum(1 for s in "xyz" if s in self.pbc)]
        self.pbc_reps = int(pbc_reps)

    num_nodes = property(lambda self: (self.nx, self.ny, self.nz))
    delta = property(lambda self: (self.dx, self.dy, self.dz))
    total_nodes = property(lambda self: self.nx * self.ny * self.nz)
    cell_volume = property(lambda self: self.dx * self.dy * self.dz)
    volume = property(lambda self: self.cell_volume * self.total_nodes)
    size = property(lambda self: (self.nx * self.dx, self.ny * self.dy, self.nz * self.dz))
    periodic_bc = property(lambda self: (self.pbc, self.pbc_reps))

    def getPosition(self, i):
        x, y, z = i % self.nx, (i // self.nx) % self.ny, i // (self.nx * self.ny)
        return (x + 0.5) * self.dx, (y + 0.5) * self.dy, (z + 0.5) * self.dz

    def iterateCellIndices(self):
        return itertools.product(*map(range, self.num_nodes))

    def isCompatible(self, other):
        return self.num_nodes == other.num_nodes and self.delta == other.delta


class Field(Matrix):
    def __init__(self, mesh):
        super().__init__(Shape(*mesh.num_nodes))
        self.mesh = mesh


class VectorField(VectorMatrix):
    def __init__(self, mesh):
        super().__init__(Shape(*mesh.num_nodes))
        self.mesh = mesh

    def initFromFunction(self, fn):
        for i in range(self.mesh.total_nodes):
            self.set(i, fn(self.mesh, self.mesh.getPosition(i)))


def _dims(f):
    return f.dimX(), f.dimY(), f.dimZ()


# ---- field terms: the reference's compiled CPU kernels ------------------------------------------
def exchange(*args):
    _count("exchange")
    if len(args) == 4:
        Ms, A, M, H = args
        m = M.mesh
        (nx, ny, nz), (dx, dy, dz), pbc = m.num_nodes, m.delta, m.periodic_bc[0]
        px, py, pz = "x" in pbc, "y" in pbc, "z" in pbc
    else:
        nx, ny, nz, dx, dy, dz, px, py, pz, Ms, A, M, H = args
    return reference().mmref_exchange(nx, ny, nz, _D(dx), _D(dy), _D(dz), int(px), int(py), int(pz), _p(Ms.arr),
                                      _p(A.arr), _p(M.arr), _p(H.arr))


def uniaxial_anisotropy(axis, k, Ms, M, H):
    _count("uniaxial_anisotropy")
    return reference().mmref_uniaxial_anisotropy(*_dims(M), _p(axis.arr), _p(k.arr), _p(Ms.arr), _p(M.arr), _p(H.arr))


def cubic_anisotropy(axis1, axis2, k, Ms, M, H):
    _count("cubic_anisotropy")
    return reference().mmref_cubic_anisotropy(*_dims(M), _p(axis1.arr), _p(axis2.arr), _p(k.arr), _p(Ms.arr),
                                              _p(M.arr), _p(H.arr))


def llge(f1, f2, M, H, dM):
    _count("llge")
    reference().mmref_llge(*_dims(M), _p(f1.arr), _p(f2.arr), _p(M.arr), _p(H.arr), _p(dM.arr))


def fdm_zhangli(nx, ny, nz, dx, dy, dz, do_precess, P, xi, Ms, alpha, j, M, dM):
    _count("fdm_zhangli")
    reference().mmref_fdm_zhangli(nx, ny, nz, _D(dx), _D(dy), _D(dz), int(bool(do_precess)), _p(P.arr), _p(xi.arr),
                                  _p(Ms.arr), _p(alpha.arr), _p(j.arr), _p(M.arr), _p(dM.arr))


def scaled_abs_max(M, scale):
    _count("scaled_abs_max")
    return reference().mmref_scaled_abs_max(*_dims(M), _p(M.arr), _p(scale.arr))


# ---- demag ---------------------------------------------------------------------------------------
def round_tensor_dimension(dim, periodic, padding):
    return int(reference().mmref_round_tensor_dimension(int(dim), int(bool(periodic)), int(padding)))


def GenerateDemagTensor(nx, ny, nz, dx, dy, dz, px, py, pz, repeat, padding, cache_dir=None):
    _count("GenerateDemagTensor")
    ex, ey, ez = (round_tensor_dimension(d, p, padding) for d, p in zip((nx, ny, nz), (px, py, pz)))
    N = Matrix(Shape(6, ex, ey, ez))
    reference().mmref_demag_tensor(nx, ny, nz, _D(dx), _D(dy), _D(dz), int(px), int(py), int(pz), int(repeat), ex, ey,
                                   ez, _p(N.arr))
    return N


class SymmetricMatrixVectorConvolution_FFT:
    """The oracle's FFT convolution (restated; the reference's needs FFTW)."""

    def __init__(self, lhs, nx, ny, nz):
        self.N, self.dims, self.pd = lhs.arr, (nx, ny, nz), tuple(lhs.getShape()[1:])

    def execute(self, M, H):
        _count("conv_fft")
        H.arr[:] = conv(self.N, self.dims, self.pd, M.arr, method="fft").reshape(-1)


class SymmetricMatrixVectorConvolution_Simple:
    """SymmetricMatrixVectorConvolution_Simple.cpp:36-80 (the reference's direct sum)."""

    def __init__(self, lhs, nx, ny, nz):
        self.N, self.dims, self.pd = lhs.arr, (nx, ny, nz), tuple(lhs.getShape()[1:])

    def execute(self, M, H):
        _count("conv_simple")
        H.arr[:] = conv(self.N, self.dims, self.pd, M.arr, impl="ref").reshape(-1)


# ---- evolver --------------------------------------------------------------------------------------
class ButcherTableau:
    def __init__(self, num_steps):
        self.num_steps = int(num_steps)
        self.a = [0.0] * num_steps
        self.b = [[0.0] * num_steps for _ in range(num_steps)]
        self.c = [0.0] * num_steps
        self.ec = [0.0] * num_steps

    def setA(self, i, v): self.a[i] = float(v)
    def getA(self, i): return self.a[i]
    def setB(self, i, j, v): self.b[i][j] = float(v)
    def getB(self, i, j): return self.b[i][j]
    def setC(self, i, v): self.c[i] = float(v)
    def getC(self, i): return self.c[i]
    def setEC(self, i, v): self.ec[i] = float(v)
    def getEC(self, i): return self.ec[i]
    def getNumSteps(self): return self.num_steps


def _tab_arrays(tab):
    s = tab.num_steps
    b = np.array([[tab.getB(i, j) for j in range(s)] for i in range(s)], dtype=np.float64).reshape(-1)
    return s, [_f(tab.a), _f(b), _f(tab.c), _f(tab.ec)]


def _kptrs(ks):
    arr = (ctypes.POINTER(ctypes.c_double) * len(ks))()
    for i, k in enumerate(ks):
        arr[i] = _p(k.arr)
    return arr


def rk_prepare_step(step, h, tab, k0, k1, k2, k3, k4, k5, y, ytmp):
    """runge_kutta.cpp:32-48 (the reference's compiled CPU path)."""
    _count("rk_prepare_step")
    s, t = _tab_arrays(tab)
    out = np.zeros(3 * y.size())
    reference().mmref_rk_prepare_step(*_dims(y), int(step), _D(h), s, *[_p(a) for a in t],
                                      _kptrs([k0, k1, k2, k3, k4, k5]), _p(y.arr), _p(out))
    ytmp.from_numpy(out)


def rk_combine_result(h, tab, k0, k1, k2, k3, k4, k5, y, y_err):
    """runge_kutta.cpp:68-96, the six-vector form."""
    _count("rk_combine_result")
    s, t = _tab_arrays(tab)
    err = np.zeros(3 * y.size())
    reference().mmref_rk_combine_result(*_dims(y), _D(h), s, *[_p(a) for a in t], _kptrs([k0, k1, k2, k3, k4, k5]),
                                        _p(y.arr), _p(err))
    y_err.from_numpy(err)


def rk_adjust_stepsize(order, h, eps_abs, eps_rel, y, y_error):
    """runge_kutta.cpp:98-130 (the NR controller's rule)."""
    _count("rk_adjust_stepsize")
    return reference().mmref_rk_adjust_stepsize(*_dims(y), int(order), _D(h), _D(eps_abs), _D(eps_rel), _p(y.arr),
                                                _p(y_error.arr))
