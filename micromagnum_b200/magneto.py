"""Drop-in mirror of the reference's ``magneto`` extension module for the hot path.

MicroMagnum's Python layer (``magnum``) reaches its native code through one module,
``magnum.magneto`` = the SWIG module ``magneto_cuda`` / ``magneto_cpu`` (src/magnum/magneto.py:18-21).
This module offers the names, argument order and results that ``magnum`` uses, backed by
libmmb200.so (include/mmb200.h):

  field terms  exchange, uniaxial_anisotropy, cubic_anisotropy, llge, fdm_zhangli, scaled_abs_max
  demag        GenerateDemagTensor (with the reference's tensor cache), round_tensor_dimension,
               SymmetricMatrixVectorConvolution_FFT, PADDING_*
  evolver      ButcherTableau, rk_prepare_step, rk_combine_result, rk_adjust_stepsize
  containers   Shape, Matrix, VectorMatrix, Field, VectorField, RectangularMesh
               (src/magneto/matrix/matty.inc.i:61-305, mesh/Field.i, mesh/VectorField.i,
               mesh/RectangularMesh.i)
  io           OMFHeader, readOMF, writeOMF, OMF_FORMAT_* (bindings/mmm/io.i)
  set-up       initialize, deinitialize, enableCuda, isCudaEnabled, isCuda64Enabled,
               haveCudaSupport, cudaSync, enableProfiling, isProfilingEnabled,
               printProfilingReport, haveFFTWThreads, setFFTWThreads, setDebugCallback, CUDA_*

Containers follow the reference's matrices: a freshly created or filled matrix is *uniform* (one
value, no storage, AbstractMatrix.h state UNIFORM) and gets device storage only when its data is
needed on the GPU or a single element is written.  Storage follows the precision mode: float64 in
CUDA_64 (the reference's ``-G``), float32 in CUDA_32 (``-g``), so the per-term calls pass the
arrays as they are.  Nothing here computes on the CPU: with CUDA_DISABLED (``magnum`` without
``-g``/``-G``) every call that needs the device raises RuntimeError.  Errors raise RuntimeError,
as the reference's SWIG %exception handler does (bindings/magneto.i:31-42).
"""
from __future__ import annotations

import ctypes
import itertools
import math
import os
import time
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, lib

__all__ = [
    "CUDA_DISABLED", "CUDA_32", "CUDA_64", "PADDING_DISABLE", "PADDING_ROUND_2", "PADDING_ROUND_4",
    "PADDING_ROUND_8", "PADDING_ROUND_POT", "PADDING_SMALL_PRIME_FACTORS", "OMF_FORMAT_ASCII",
    "OMF_FORMAT_BINARY_4", "OMF_FORMAT_BINARY_8",
    "initialize", "deinitialize", "enableCuda", "isCudaEnabled", "isCuda64Enabled", "haveCudaSupport", "cudaSync",
    "flush", "enableProfiling", "isProfilingEnabled", "printProfilingReport", "haveFFTWThreads", "setFFTWThreads",
    "setDebugCallback",
    "Shape", "Matrix", "VectorMatrix", "RectangularMesh", "Field", "VectorField",
    "exchange", "uniaxial_anisotropy", "cubic_anisotropy", "llge", "fdm_zhangli", "scaled_abs_max",
    "round_tensor_dimension", "GenerateDemagTensor", "SymmetricMatrixVectorConvolution_FFT",
    "ButcherTableau", "rk_prepare_step", "rk_combine_result", "rk_adjust_stepsize",
    "OMFHeader", "readOMF", "writeOMF", "parseOMF", "formatOMF",
]

CUDA_DISABLED, CUDA_32, CUDA_64 = 0, 1, 2
PADDING_DISABLE, PADDING_ROUND_2, PADDING_ROUND_4 = 0, 1, 2
PADDING_ROUND_8, PADDING_ROUND_POT, PADDING_SMALL_PRIME_FACTORS = 3, 4, 5
OMF_FORMAT_ASCII, OMF_FORMAT_BINARY_4, OMF_FORMAT_BINARY_8 = 0, 1, 2

_mode = CUDA_64
_device: Optional[torch.device] = None
_cache_dir: Optional[str] = None
_debug_callback = None
CACHE_AFTER_S = 30.0  # tensors that took longer to generate are stored in the cache directory


# ------------------------------------------------------------------------------------------------
# set-up (bindings/magneto.i:77-101, Magneto.cpp)
# ------------------------------------------------------------------------------------------------
def initialize(cache_dir: str = "") -> None:
    """Magneto.cpp initialize(): remembers the cache directory (the demag tensor cache)."""
    global _cache_dir
    _cache_dir = cache_dir or None


def deinitialize(cache_dir: str = "") -> None:
    pass


def enableCuda(mode: int = CUDA_64, gpu_id: int = -1) -> None:
    """Magneto.cpp:56-73.  CUDA_64: plain FP64 kernels; CUDA_32: float storage and kernels.
    CUDA_DISABLED leaves the module without a compute device: this library has no CPU path, so a
    call that computes then raises RuntimeError."""
    global _mode, _device
    if mode == CUDA_DISABLED:
        _mode = CUDA_DISABLED
        return
    if mode not in (CUDA_32, CUDA_64):
        raise RuntimeError(f"enableCuda: unknown mode {mode}")
    if not torch.cuda.is_available():
        raise RuntimeError("enableCuda: no CUDA device")
    _mode = mode
    _device = torch.device("cuda", gpu_id if gpu_id >= 0 else torch.cuda.current_device())
    torch.cuda.set_device(_device)


def isCudaEnabled() -> bool:
    return _mode != CUDA_DISABLED


def isCuda64Enabled() -> bool:
    return _mode == CUDA_64


def haveCudaSupport() -> bool:
    return torch.cuda.is_available()


def cudaSync() -> None:
    torch.cuda.synchronize()


def flush() -> None:
    pass


def enableProfiling(yes: bool = True) -> None:
    """Per-kernel device timing of the library's launches (CUDA events), read by
    printProfilingReport()."""
    _lib.profile_enable(bool(yes))
    _prof["on"] = bool(yes)


_prof = {"on": False}


def isProfilingEnabled() -> bool:
    return _prof["on"]


def printProfilingReport() -> None:
    rows = sorted(_lib.profile_read().items(), key=lambda kv: -kv[1][1])
    total = sum(v[1] for _, v in rows) or 1.0
    print(f"{'kernel':40s} {'launches':>9s} {'ms':>12s} {'share':>7s} {'GB/s':>9s}")
    for name, (cnt, ms, by) in rows:
        gbs = by / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        print(f"{name:40s} {cnt:9d} {ms:12.3f} {ms / total:7.1%} {gbs:9.1f}")


def haveFFTWThreads() -> bool:
    """The convolution runs on the GPU; there are no FFTW threads to configure."""
    return False


def setFFTWThreads(num_threads: int) -> None:
    pass


def setDebugCallback(callback) -> None:
    global _debug_callback
    _debug_callback = callback


def _require_device():
    global _device
    if _mode == CUDA_DISABLED:
        raise RuntimeError("magneto: CUDA is disabled (enableCuda(CUDA_32 or CUDA_64), magnum's -g/-G); this "
                           "library has no CPU implementation")
    if _device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("micromagnum_b200.magneto needs a CUDA device")
        _device = torch.device("cuda", torch.cuda.current_device())
    return _device


def _dtype():
    return torch.float64 if _mode != CUDA_32 else torch.float32


def _prec() -> int:
    _require_device()
    return _lib.MM_F64 if _mode != CUDA_32 else _lib.MM_F32


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


# ------------------------------------------------------------------------------------------------
# containers
# ------------------------------------------------------------------------------------------------
class Shape(tuple):
    """matrix/Shape.h: dimensions, first index fastest."""

    def __new__(cls, *dims):
        if len(dims) == 1 and isinstance(dims[0], (tuple, list)):
            dims = tuple(dims[0])
        return super().__new__(cls, tuple(int(d) for d in dims))

    def getNumEl(self) -> int:
        return int(math.prod(self)) if len(self) else 0

    def getDim(self, d: int) -> int:
        return self[d]

    def getDims(self):
        return list(self)

    def getRank(self) -> int:
        return len(self)

    def getStride(self, d: int) -> int:
        return int(math.prod(self[:d]))

    def getStrides(self):
        return [self.getStride(d) for d in range(len(self))]

    def getLinIdx(self, *idx) -> int:
        return sum(int(i) * self.getStride(d) for d, i in enumerate(idx))

    def sameDims(self, other) -> bool:
        return tuple(self) == tuple(other)


class _Base:
    """Storage shared by Matrix and VectorMatrix: either a uniform value (no storage) or a flat
    device tensor of ncomp * size elements (SoA for vector fields, x fastest)."""
    NCOMP = 1

    def __init__(self, shape, *, _fixed_dtype=None):
        if isinstance(shape, _Base):  # copy constructor
            other = shape
            self._shape = Shape(other._shape)
            self._n = other._n
            self._fixed = other._fixed
            self._u = other._u
            self._t = None if other._t is None else other._t.clone()
            return
        self._shape = Shape(shape)
        self._n = self._shape.getNumEl()
        self._fixed = _fixed_dtype
        self._u = self._zero()
        self._t = None

    # -- storage ----------------------------------------------------------------------------------
    def _zero(self):
        return 0.0 if self.NCOMP == 1 else (0.0, 0.0, 0.0)

    def _want(self):
        return self._fixed or _dtype()

    @property
    def data(self) -> torch.Tensor:
        """The device tensor (created from the uniform value on first use; converted once when the
        precision mode changed since)."""
        dev = _require_device()
        want = self._want()
        if self._t is None:
            t = torch.empty(self.NCOMP * self._n, dtype=want, device=dev)
            if self.NCOMP == 1:
                t.fill_(float(self._u))
            else:
                for c in range(3):
                    t[c * self._n:(c + 1) * self._n].fill_(float(self._u[c]))
            self._t = t
        elif self._t.dtype != want or self._t.device != dev:
            self._t = self._t.to(device=dev, dtype=want)
        return self._t

    def _set_uniform(self, value):
        self._u = value
        self._t = None

    # -- AbstractMatrix ---------------------------------------------------------------------------
    def getShape(self) -> Shape:
        return self._shape

    shape = property(lambda self: tuple(self._shape) if len(self._shape) != 3 else
                     (self._shape[0], self._shape[1], self._shape[2]))
    rank = property(lambda self: len(self._shape))
    element_size = property(lambda self: self.NCOMP)

    def isUniform(self) -> bool:
        return self._t is None

    def isWriteLocked(self) -> bool:
        return False

    def isLocked(self) -> bool:
        return False

    def inspect(self) -> None:
        print(f"{type(self).__name__}{tuple(self._shape)}: "
              f"{'uniform ' + repr(self._u) if self._t is None else str(self._t.dtype) + ' on ' + str(self._t.device)}")

    def flush(self) -> None:
        pass

    def markUninitialized(self) -> None:
        pass

    def size(self) -> int:
        return self._n

    def dimX(self) -> int:
        return self._shape[0] if len(self._shape) > 0 else 1

    def dimY(self) -> int:
        return self._shape[1] if len(self._shape) > 1 else 1

    def dimZ(self) -> int:
        return self._shape[2] if len(self._shape) > 2 else 1

    def _lin(self, idx) -> int:
        if len(idx) == 1:
            return int(idx[0])
        return self._shape.getLinIdx(*idx)

    @property
    def uniform_value(self):
        if not self.isUniform():
            raise ValueError(f"{type(self).__name__} must be uniform in order to access the uniform_value property!")
        return self._u

    def getUniformValue(self):
        if not self.isUniform():
            raise RuntimeError("Cant get uniform value because matrix is not uniform")
        return self._u

    def swap(self, other) -> None:
        for a in ("_shape", "_n", "_fixed", "_u", "_t"):
            va, vb = getattr(self, a), getattr(other, a)
            setattr(self, a, vb)
            setattr(other, a, va)

    def clear(self) -> None:
        self._set_uniform(self._zero())

    def __repr__(self):
        return f"{type(self).__name__}({self.shape!r})"


class Matrix(_Base):
    """Scalar field (matrix/matrix/scalar/Matrix.h)."""

    def fill(self, value) -> None:
        self._set_uniform(float(value))

    def assign(self, other: "Matrix") -> None:
        if other.isUniform():
            self._set_uniform(other._u)
        else:
            self.data.copy_(other.data)

    def scale(self, factor) -> None:
        f = float(factor)
        if f == 0.0:
            self.fill(0.0)
        elif self.isUniform():
            self._set_uniform(self._u * f)
        else:
            self.data.mul_(f)

    def add(self, op: "Matrix", scale: float = 1.0) -> None:
        if self.isUniform() and op.isUniform():
            self._set_uniform(self._u + float(scale) * op._u)
        else:
            self.data.add_(op.data, alpha=float(scale))

    def multiply(self, rhs: "Matrix") -> None:
        if self.isUniform() and rhs.isUniform():
            self._set_uniform(self._u * rhs._u)
        else:
            self.data.mul_(rhs.data)

    def divide(self, rhs: "Matrix") -> None:
        if self.isUniform() and rhs.isUniform():
            self._set_uniform(self._u / rhs._u)
        else:
            self.data.div_(rhs.data)

    def randomize(self) -> None:
        """CPUDevice.cpp:164-170: every element uniform in [0, 1] (seed it with torch.manual_seed)."""
        self.data.uniform_(0.0, 1.0)

    def maximum(self) -> float:
        return float(self._u) if self.isUniform() else float(self.data.max().item())

    def sum(self) -> float:
        return float(self._u) * self._n if self.isUniform() else float(self.data.double().sum().item())

    def average(self) -> float:
        return self.sum() / self._n

    def absMax(self) -> float:
        return abs(float(self._u)) if self.isUniform() else float(self.data.abs().max().item())

    def get(self, *idx) -> float:
        if self.isUniform():
            return float(self._u)
        return float(self.data[self._lin(idx)].item())

    def set(self, *args) -> None:
        *idx, v = args
        if self.isUniform() and float(v) == self._u:
            return
        self.data[self._lin(idx)] = float(v)

    def to_numpy(self) -> np.ndarray:
        """(dimX, dimY, dimZ) array indexed [x, y, z] (matty.inc.i matrix_to_numpy)."""
        nx, ny, nz = self.dimX(), self.dimY(), self.dimZ()
        if self.isUniform():
            return np.full((nx, ny, nz), float(self._u))
        return self.data.view(nz, ny, nx).permute(2, 1, 0).double().cpu().numpy()

    def from_numpy(self, arr) -> None:
        """From a [x, y, z] array (to_numpy's layout) or a flat array of size() values."""
        a = np.asarray(arr, dtype=np.float64)
        if a.ndim == 3:
            a = np.transpose(a, (2, 1, 0))
        self.data.copy_(torch.as_tensor(np.ascontiguousarray(a).reshape(-1)))


class VectorMatrix(_Base):
    """3-vector field, SoA (matrix/matrix/vector/VectorMatrix.h)."""
    NCOMP = 3

    def comp(self, c: int) -> torch.Tensor:
        return self.data[c * self._n:(c + 1) * self._n]

    def fill(self, value) -> None:
        v = tuple(float(x) for x in value)
        if len(v) != 3:
            raise RuntimeError("VectorMatrix.fill: needs a 3-vector")
        self._set_uniform(v)

    def assign(self, other: "VectorMatrix") -> None:
        if other.isUniform():
            self._set_uniform(other._u)
        else:
            self.data.copy_(other.data)

    def scale(self, factor) -> None:
        f = float(factor)
        if f == 0.0:
            self.clear()
        elif self.isUniform():
            self._set_uniform(tuple(u * f for u in self._u))
        else:
            self.data.mul_(f)

    def scale_by_vector(self, factors) -> None:
        f = tuple(float(x) for x in factors)
        if self.isUniform():
            self._set_uniform(tuple(u * g for u, g in zip(self._u, f)))
        else:
            for c in range(3):
                self.comp(c).mul_(f[c])

    def add(self, op: "VectorMatrix", scale: float = 1.0) -> None:
        if self.isUniform() and op.isUniform():
            self._set_uniform(tuple(a + float(scale) * b for a, b in zip(self._u, op._u)))
        else:
            self.data.add_(op.data, alpha=float(scale))

    def randomize(self) -> None:
        """CPUDevice.cpp:164-170: every component uniform in [0, 1] (not uniform on the sphere)."""
        self.data.uniform_(0.0, 1.0)

    def normalize(self, length) -> None:
        """VectorMatrix::normalize(double) / normalize(Matrix) (VectorMatrix.cpp:205-230), with the
        reference's GPU semantics (zero vectors stay zero)."""
        if self.isUniform() and (not isinstance(length, Matrix) or length.isUniform()):
            ln = float(length._u if isinstance(length, Matrix) else length)
            r = math.sqrt(sum(u * u for u in self._u))
            self._set_uniform(tuple(u * ln / r for u in self._u) if r > 0 else (0.0, 0.0, 0.0))
            return
        if isinstance(length, Matrix):
            ms = length.data
            if ms.dtype != self.data.dtype:
                ms = ms.to(self.data.dtype)
        else:
            ms = torch.full((self._n,), float(length), dtype=self.data.dtype, device=self.data.device)
        check(lib().mm_normalize(_prec(), self._n, _ptr(ms), _ptr(self.data), _stream()))

    def absMax(self) -> float:
        if self.isUniform():
            return math.sqrt(sum(u * u for u in self._u))
        v = self.data.view(3, self._n).double()
        return float(torch.sqrt((v * v).sum(0).max()).item())

    def dotSum(self, other: "VectorMatrix") -> float:
        if self.isUniform() and other.isUniform():
            return self._n * sum(a * b for a, b in zip(self._u, other._u))
        return float((self.data.double() * other.data.double()).sum().item())

    def maximum(self):
        if self.isUniform():
            return self._u
        return tuple(self.data.view(3, self._n).max(1).values.double().tolist())

    def sum(self):
        if self.isUniform():
            return tuple(u * self._n for u in self._u)
        return tuple(self.data.view(3, self._n).double().sum(1).tolist())

    def average(self):
        return tuple(s / self._n for s in self.sum())

    def get(self, *idx):
        if self.isUniform():
            return self._u
        i = self._lin(idx)
        return tuple(float(v) for v in self.data.view(3, self._n)[:, i].tolist())

    def set(self, *args) -> None:
        *idx, v = args
        v = tuple(float(x) for x in v)
        if self.isUniform() and v == self._u:
            return
        i = self._lin(idx)
        t = self.data.view(3, self._n)
        t[:, i] = torch.tensor(v, dtype=t.dtype, device=t.device)

    def to_numpy(self) -> np.ndarray:
        """(dimX, dimY, dimZ, 3) array indexed [x, y, z, component] (matty.inc.i
        vector_matrix_to_numpy)."""
        nx, ny, nz = self.dimX(), self.dimY(), self.dimZ()
        if self.isUniform():
            return np.broadcast_to(np.asarray(self._u), (nx, ny, nz, 3)).copy()
        return self.data.view(3, nz, ny, nx).permute(3, 2, 1, 0).double().cpu().numpy()

    def from_numpy(self, arr) -> None:
        """From a [x, y, z, component] array (to_numpy's layout) or SoA data of 3 * size() values."""
        a = np.asarray(arr, dtype=np.float64)
        if a.ndim == 4:
            a = np.transpose(a, (3, 2, 1, 0))
        self.data.copy_(torch.as_tensor(np.ascontiguousarray(a).reshape(-1)))


class RectangularMesh:
    """mesh/RectangularMesh.h:7-66: nx x ny x nz cells of dx x dy x dz, periodic directions as a
    string of "x", "y", "z" with the number of periodic repetitions (defaults 1, 15, 3, 2 for 0-3
    periodic directions)."""

    def __init__(self, nx, ny, nz, dx, dy, dz, pbc: str = "", pbc_reps: int = -1):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)
        self.pbc = str(pbc or "")
        if pbc_reps is None or int(pbc_reps) == -1:
            ndirs = sum(1 for s in "xyz" if s in self.pbc)
            pbc_reps = (1, 15, 3, 2)[ndirs]
        self.pbc_reps = int(pbc_reps)

    def isCompatible(self, other) -> bool:
        return self.num_nodes == other.num_nodes and self.delta == other.delta

    def getCellVolume(self) -> float:
        return self.dx * self.dy * self.dz

    def getTotalNodes(self) -> int:
        return self.nx * self.ny * self.nz

    def getVolume(self) -> float:
        return self.getCellVolume() * self.getTotalNodes()

    def getNumNodes(self):
        return self.nx, self.ny, self.nz

    def getDelta(self):
        return self.dx, self.dy, self.dz

    def getSize(self):
        return self.nx * self.dx, self.ny * self.dy, self.nz * self.dz

    def getPeriodicBC(self):
        return self.pbc, self.pbc_reps

    def getPosition(self, linidx: int):
        """The middle point of the cell with linear index linidx."""
        i = int(linidx)
        x, y, z = i % self.nx, (i // self.nx) % self.ny, i // (self.nx * self.ny)
        return (x + 0.5) * self.dx, (y + 0.5) * self.dy, (z + 0.5) * self.dz

    def iterateCellIndices(self):
        return itertools.product(*map(range, self.num_nodes))

    volume = property(getVolume)
    cell_volume = property(getCellVolume)
    total_nodes = property(getTotalNodes)
    num_nodes = property(lambda self: (self.nx, self.ny, self.nz))
    delta = property(lambda self: (self.dx, self.dy, self.dz))
    size = property(getSize)
    periodic_bc = property(getPeriodicBC)

    def __repr__(self):
        return (f"RectangularMesh({self.num_nodes!r}, {self.delta!r}, periodic_bc={self.pbc!r}, "
                f"periodic_repeat={self.pbc_reps!r})")


def _mesh_shape(mesh):
    return Shape(*mesh.num_nodes)


class Field(Matrix):
    """Scalar field on a mesh (mesh/Field.h, mesh/Field.i)."""

    def __init__(self, mesh):
        if isinstance(mesh, Field):
            super().__init__(mesh)
            self._mesh = mesh._mesh
            return
        super().__init__(_mesh_shape(mesh))
        self._mesh = mesh

    def getMesh(self):
        return self._mesh

    mesh = property(getMesh)

    def __repr__(self):
        return f"Field({self._mesh!r})"


class VectorField(VectorMatrix):
    """Vector field on a mesh (mesh/VectorField.h, mesh/VectorField.i)."""

    def __init__(self, mesh):
        if isinstance(mesh, VectorField):
            super().__init__(mesh)
            self._mesh = mesh._mesh
            return
        super().__init__(_mesh_shape(mesh))
        self._mesh = mesh

    def getMesh(self):
        return self._mesh

    mesh = property(getMesh)

    def initFromFunction(self, init_fn) -> None:
        """VectorField.i initFromFunction: value of every cell from init_fn(mesh, position); the
        values are gathered on the host and uploaded once."""
        mesh = self._mesh
        vals = np.array([init_fn(mesh, mesh.getPosition(i)) for i in range(mesh.total_nodes)], dtype=np.float64)
        self.data.copy_(torch.as_tensor(np.ascontiguousarray(vals.T).reshape(-1)))

    def __repr__(self):
        return f"VectorField({self._mesh!r})"


def _mesh_of(f):
    mesh = getattr(f, "mesh", None)
    if mesh is None:
        raise RuntimeError("field has no mesh")
    return mesh


# ------------------------------------------------------------------------------------------------
# field terms (every array in the mode's precision, on the device)
# ------------------------------------------------------------------------------------------------
def exchange(*args) -> float:
    """exchange(nx, ny, nz, dx, dy, dz, px, py, pz, Ms, A, M, H) or exchange(Ms, A, M, H)
    (bindings/mmm/exchange.i:24-39).  Returns -mu0/2 V sum M.H."""
    if len(args) == 4:
        Ms, A, M, H = args
        mesh = _mesh_of(M)
        (nx, ny, nz), (dx, dy, dz) = mesh.num_nodes, mesh.delta
        pbc = mesh.periodic_bc[0]
        px, py, pz = "x" in pbc, "y" in pbc, "z" in pbc
    else:
        nx, ny, nz, dx, dy, dz, px, py, pz, Ms, A, M, H = args
    e = ctypes.c_double(0.0)
    p = _prec()
    check(lib().mm_exchange(p, nx, ny, nz, dx, dy, dz, int(px), int(py), int(pz), _ptr(Ms.data), _ptr(A.data),
                            _ptr(M.data), _ptr(H.data), ctypes.byref(e), _stream()))
    return e.value


def uniaxial_anisotropy(axis, k, Ms, M, H) -> float:
    """bindings/mmm/anisotropy.i:24-31; returns sum_i k |a x m|^2 (CPU path's value)."""
    e = ctypes.c_double(0.0)
    p = _prec()
    check(lib().mm_uniaxial_anisotropy(p, M.size(), *[_ptr(f.data) for f in (axis, k, Ms, M, H)],
                                       ctypes.byref(e), _stream()))
    return e.value


def cubic_anisotropy(axis1, axis2, k, Ms, M, H) -> float:
    """bindings/mmm/anisotropy.i:32-39."""
    e = ctypes.c_double(0.0)
    p = _prec()
    check(lib().mm_cubic_anisotropy(p, M.size(), *[_ptr(f.data) for f in (axis1, axis2, k, Ms, M, H)],
                                    ctypes.byref(e), _stream()))
    return e.value


def llge(f1, f2, M, H, dM) -> None:
    """bindings/mmm/llge.i:24-29: dM = f1 M x H + f2 M x (M x H)."""
    p = _prec()
    check(lib().mm_llge(p, M.size(), *[_ptr(f.data) for f in (f1, f2, M, H, dM)], _stream()))


def fdm_zhangli(nx, ny, nz, dx, dy, dz, do_precess, P, xi, Ms, alpha, j, M, dM) -> None:
    """bindings/mmm/zhangli.i:24-32."""
    p = _prec()
    check(lib().mm_fdm_zhangli(p, nx, ny, nz, dx, dy, dz, int(bool(do_precess)),
                               *[_ptr(f.data) for f in (P, xi, Ms, alpha, j, M, dM)], _stream()))


def scaled_abs_max(M, scale) -> float:
    """bindings/math.i:66 (math/ScaledAbsMax.cpp:52-68)."""
    if scale.isUniform():
        return M.absMax() / scale.getUniformValue()
    r = ctypes.c_double(0.0)
    p = _prec()
    check(lib().mm_scaled_abs_max(p, M.size(), _ptr(M.data), _ptr(scale.data), ctypes.byref(r), _stream()))
    return r.value


# ------------------------------------------------------------------------------------------------
# demag
# ------------------------------------------------------------------------------------------------
def round_tensor_dimension(dim: int, periodic: bool, padding: int) -> int:
    return int(lib().mm_round_tensor_dimension(int(dim), int(bool(periodic)), int(padding)))


def GenerateDemagTensor(nx, ny, nz, dx, dy, dz, px, py, pz, repeat, padding, cache_dir=None) -> Matrix:
    """bindings/mmm/demag.i:27-42 (mmm/demag/demag_tensor.cpp:116-186), computed on the GPU in FP64.
    Returns Matrix(Shape(6, ex, ey, ez)) holding the negated tensor (float64 in either mode); along
    periodic axes (px, py, pz) no padding and `repeat` periodic images plus the images beyond them
    (mm_demag_tensor_periodic).  With a cache directory, a tensor stored there under the
    reference's file name (demag_tensor.cpp:52-73) is loaded instead, and a computed one is stored
    when its generation took longer than 30 s, the reference's rule (demag_tensor.cpp:178-181); the
    file is the raw float64 array, as the reference writes it."""
    ex = round_tensor_dimension(nx, px, padding)
    ey = round_tensor_dimension(ny, py, padding)
    ez = round_tensor_dimension(nz, pz, padding)
    N = Matrix(Shape(6, ex, ey, ez), _fixed_dtype=torch.float64)
    path = demag_cache_file(nx, ny, nz, ex, ey, ez, dx, dy, dz, px, py, pz, repeat, cache_dir) if cache_dir else None
    if path and os.path.exists(path) and os.path.getsize(path) == 8 * N.size():
        N.data.copy_(torch.from_numpy(np.fromfile(path, dtype=np.float64)))
        return N
    t0 = time.perf_counter()
    check(lib().mm_demag_tensor_periodic(nx, ny, nz, dx, dy, dz, int(bool(px)), int(bool(py)), int(bool(pz)),
                                         int(repeat), ex, ey, ez, _ptr(N.data), _stream()))
    torch.cuda.current_stream().synchronize()
    if path and time.perf_counter() - t0 > CACHE_AFTER_S and not os.path.exists(path):
        tmp = f"{path}.{os.getpid()}.tmp"
        N.data.cpu().numpy().tofile(tmp)
        os.replace(tmp, path)
    return N


def demag_cache_file(nx, ny, nz, ex, ey, ez, dx, dy, dz, px, py, pz, repeat, cache_dir) -> str:
    """The reference's cache file name (demag_tensor.cpp:52-73): sizes, padded sizes and the cell
    size truncated to whole picometres (so cell sizes that differ below 1 pm share a file), plus
    the periodic directions and repetitions."""
    name = f"Demag--{nx}-{ny}-{nz}--{ex}-{ey}-{ez}--{int(dx * 1e12)}-{int(dy * 1e12)}-{int(dz * 1e12)}"
    if px or py or pz:
        name += "--p-" + ("x" if px else "") + ("y" if py else "") + ("z" if pz else "") + f"-{repeat}"
    return os.path.join(cache_dir, name + ".dat")


class SymmetricMatrixVectorConvolution_FFT:
    """bindings/math.i:27-33: H = N * M for a tensor field N of shape (6, ex, ey, ez)."""

    def __init__(self, lhs: Matrix, nx: int, ny: int, nz: int):
        _, ex, ey, ez = lhs.getShape()
        self.dims = (nx, ny, nz)
        self._prec = _prec()
        t = lhs.data if lhs.data.dtype == torch.float64 else lhs.data.double()
        h = ctypes.c_void_p()
        check(lib().mm_conv_create(ctypes.byref(h), self._prec, nx, ny, nz, ex, ey, ez, _ptr(t), _stream()))
        self._h = h

    def execute(self, rhs: VectorMatrix, res: VectorMatrix) -> None:
        want = torch.float64 if self._prec == _lib.MM_F64 else torch.float32
        m, out = rhs.data, res.data
        if m.dtype != want or out.dtype != want:
            raise RuntimeError("SymmetricMatrixVectorConvolution_FFT.execute: the precision mode changed "
                               "since the convolution was created")
        check(lib().mm_conv_execute(self._h, _ptr(m), _ptr(out), _stream()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().mm_conv_destroy(h)
            self._h = None


# ------------------------------------------------------------------------------------------------
# Runge-Kutta helpers (bindings/evolver.i:34-95)
# ------------------------------------------------------------------------------------------------
class ButcherTableau:
    def __init__(self, num_steps: int):
        self.num_steps = int(num_steps)
        self._a = [0.0] * num_steps
        self._b = [[0.0] * num_steps for _ in range(num_steps)]
        self._c = [0.0] * num_steps
        self._ec = [0.0] * num_steps
        self.fsal = False
        self.order = 0

    def setA(self, i, v): self._a[i] = float(v)
    def getA(self, i): return self._a[i]
    def setB(self, i, j, v): self._b[i][j] = float(v)
    def getB(self, i, j): return self._b[i][j]
    def setC(self, i, v): self._c[i] = float(v)
    def getC(self, i): return self._c[i]
    def setEC(self, i, v): self._ec[i] = float(v)
    def getEC(self, i): return self._ec[i]
    def getNumSteps(self): return self.num_steps


def _kptrs(ks):
    arr = (ctypes.c_void_p * len(ks))()
    for i, k in enumerate(ks):
        arr[i] = k.data.data_ptr()
    return arr


def rk_prepare_step(step, h, tab, k0, k1, k2, k3, k4, k5, y, ytmp) -> None:
    """ytmp = y + h sum_{j<step} b[step][j] k_j (evolver/runge_kutta.cpp:32-48)."""
    ks = [k0, k1, k2, k3, k4, k5][:step]
    b = (ctypes.c_double * max(step, 1))(*[tab.getB(step, j) for j in range(step)])
    p = _prec()
    check(lib().mm_rk_prepare_step(p, y.size(), int(step), float(h), b, _kptrs(ks), _ptr(y.data), _ptr(ytmp.data),
                                   _stream()))


def rk_combine_result(h, tab, *args) -> None:
    """y += h sum c_j k_j, y_error = h sum ec_j k_j (runge_kutta.cpp:72-96); k's then y, y_error."""
    *ks, y, y_err = args
    nk = len(ks)
    c = (ctypes.c_double * nk)(*[tab.getC(j) for j in range(nk)])
    ec = (ctypes.c_double * nk)(*[tab.getEC(j) for j in range(nk)])
    p = _prec()
    check(lib().mm_rk_combine_result(p, y.size(), nk, float(h), c, ec, _kptrs(ks), _ptr(y.data), _ptr(y_err.data),
                                     _stream()))


def rk_adjust_stepsize(order, h, eps_abs, eps_rel, y, y_error) -> float:
    """The NR step-size rule (evolver/runge_kutta.cpp:98-130) on the device's scaled error norm
    (runge_kutta_cpu.cpp:196-252): shrink by S / norm^(1/order) (at most 5x) above 1.1, grow by
    S / norm^(1/(order+1)) (between 1x and 5x) below 0.5, S = 0.9."""
    norm = ctypes.c_double(0.0)
    p = _prec()
    check(lib().mm_rk_scaled_error_norm(p, y.size(), float(eps_abs), float(eps_rel), _ptr(y.data),
                                        _ptr(y_error.data), ctypes.byref(norm), _stream()))
    return adjust_from_norm(order, h, norm.value)


def adjust_from_norm(order, h, norm) -> float:
    S = 0.9
    if norm > 1.1:
        r = S / norm ** (1.0 / order)
        return h * max(r, 0.2)
    if norm < 0.5:
        r = S / norm ** (1.0 / (order + 1.0)) if norm > 0 else 5.0
        return h * min(max(r, 1.0), 5.0)
    return h


# ------------------------------------------------------------------------------------------------
# OMF files (bindings/mmm/io.i)
# ------------------------------------------------------------------------------------------------
_OMF_STR = ("Title", "meshunit", "valueunit", "meshtype")
_OMF_NUM = ("valuemultiplier", "xmin", "ymin", "zmin", "xmax", "ymax", "zmax", "ValueRangeMaxMag",
            "ValueRangeMinMag", "xbase", "ybase", "zbase", "xstepsize", "ystepsize", "zstepsize")
_OMF_INT = ("xnodes", "ynodes", "znodes")


class OMFHeader:
    """mmm/io/OMFHeader.h: the header fields of an OMF 1.0 file (Desc is a list of lines)."""

    def __init__(self):
        for k in _OMF_STR:
            setattr(self, k, "")
        for k in _OMF_NUM:
            setattr(self, k, 0.0)
        for k in _OMF_INT:
            setattr(self, k, 0)
        self.Desc = []

    def _to_c(self) -> _lib.mm_omf_header:
        h = _lib.mm_omf_header()
        h.title = self.Title.encode()[:255]
        h.desc = "\n".join(str(d) for d in self.Desc).encode()[:4095]
        h.meshunit, h.valueunit, h.meshtype = (getattr(self, k).encode()[:63] for k in ("meshunit", "valueunit",
                                                                                        "meshtype"))
        for k in _OMF_NUM + _OMF_INT:
            setattr(h, k, getattr(self, k))
        return h

    def _from_c(self, h: _lib.mm_omf_header) -> None:
        self.Title = h.title.decode()
        self.Desc = h.desc.decode().split("\n") if h.desc else []
        self.meshunit, self.valueunit, self.meshtype = h.meshunit.decode(), h.valueunit.decode(), h.meshtype.decode()
        for k in _OMF_NUM + _OMF_INT:
            setattr(self, k, getattr(h, k))


def readOMF(path: str, header: OMFHeader) -> VectorMatrix:
    """bindings/mmm/io.i readOMF(path, header): the file's field (times valuemultiplier) as a
    VectorMatrix of Shape(xnodes, ynodes, znodes); fills `header`."""
    h = _lib.mm_omf_header()
    check(lib().mm_omf_read(str(path).encode(), ctypes.byref(h), 0, None, None))
    M = VectorMatrix(Shape(h.xnodes, h.ynodes, h.znodes))
    check(lib().mm_omf_read(str(path).encode(), ctypes.byref(h), _prec(), _ptr(M.data), _stream()))
    header._from_c(h)
    return M


def parseOMF(data: bytes, header: OMFHeader) -> VectorMatrix:
    """readOMF of an OMF file held in memory (request payloads)."""
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    h = _lib.mm_omf_header()
    check(lib().mm_omf_parse(buf, len(data), ctypes.byref(h), 0, None, None))
    M = VectorMatrix(Shape(h.xnodes, h.ynodes, h.znodes))
    check(lib().mm_omf_parse(buf, len(data), ctypes.byref(h), _prec(), _ptr(M.data), _stream()))
    header._from_c(h)
    return M


def writeOMF(path: str, header: OMFHeader, field: VectorMatrix, format: int = OMF_FORMAT_ASCII) -> None:
    """bindings/mmm/io.i writeOMF(path, header, field, format); updates the header's
    valuemultiplier and value range like the reference (OMFExport.cpp:61-79)."""
    h = header._to_c()
    check(lib().mm_omf_write(str(path).encode(), ctypes.byref(h), _prec(), _ptr(field.data), int(format), _stream()))
    header._from_c(h)


def formatOMF(header: OMFHeader, field: VectorMatrix, format: int = OMF_FORMAT_ASCII) -> bytes:
    """writeOMF into memory (response payloads)."""
    h = header._to_c()
    out, n = ctypes.c_void_p(), ctypes.c_size_t(0)
    check(lib().mm_omf_format(ctypes.byref(h), _prec(), _ptr(field.data), int(format), ctypes.byref(out),
                              ctypes.byref(n), _stream()))
    try:
        data = ctypes.string_at(out.value, n.value)
    finally:
        lib().mm_omf_free(out)
    header._from_c(h)
    return data
