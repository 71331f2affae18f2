"""Drop-in mirror of the reference's ``magneto`` extension module for the hot path.

MicroMagnum's Python layer (``magnum``) calls one C++ function per physical term through the SWIG
module ``magneto_cuda`` / ``magneto_cpu`` (src/magnum/magneto.py:18-21).  This module offers the
same names, argument order and results, backed by libmmb200.so (include/mmb200.h):

  exchange, uniaxial_anisotropy, cubic_anisotropy, llge, fdm_zhangli, scaled_abs_max,
  GenerateDemagTensor, SymmetricMatrixVectorConvolution_FFT, ButcherTableau, rk_prepare_step,
  rk_combine_result, enableCuda / isCudaEnabled / isCuda64Enabled, PADDING_*, CUDA_*,
  plus the containers Shape, Matrix, VectorMatrix (src/magneto/matrix/matty.inc.i:61-305).

Containers keep their data on the GPU (a torch CUDA tensor: float64, SoA for vector fields,
x fastest).  The global precision mode follows the reference's ``-G`` / ``-g`` switch:
CUDA_64 runs every kernel in double, CUDA_32 in float (arguments converted per call).  Errors
raise RuntimeError, as the reference's SWIG %exception handler does (bindings/magneto.i:31-42).
"""
from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from ._lib import check, lib

CUDA_DISABLED, CUDA_32, CUDA_64 = 0, 1, 2
PADDING_DISABLE, PADDING_ROUND_2, PADDING_ROUND_4 = 0, 1, 2
PADDING_ROUND_8, PADDING_ROUND_POT, PADDING_SMALL_PRIME_FACTORS = 3, 4, 5

_mode = CUDA_64
_device = None


def enableCuda(mode: int = CUDA_64, gpu_id: int = -1) -> None:
    """Magneto.cpp:56-73.  CUDA_DISABLED is rejected: this library has no CPU path."""
    global _mode, _device
    if mode not in (CUDA_32, CUDA_64):
        raise RuntimeError("enableCuda: only CUDA_32 and CUDA_64 exist in this library (no CPU path)")
    if not torch.cuda.is_available():
        raise RuntimeError("enableCuda: no CUDA device")
    _mode = mode
    _device = torch.device("cuda", gpu_id if gpu_id >= 0 else torch.cuda.current_device())


def isCudaEnabled() -> bool:
    return True


def isCuda64Enabled() -> bool:
    return _mode == CUDA_64


def haveCudaSupport() -> bool:
    return torch.cuda.is_available()


def cudaSync() -> None:
    torch.cuda.synchronize()


def _dev():
    global _device
    if _device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("micromagnum_b200.magneto needs a CUDA device")
        _device = torch.device("cuda", torch.cuda.current_device())
    return _device


def _prec() -> int:
    return _lib.MM_F64 if _mode == CUDA_64 else _lib.MM_F32


def _work(t: torch.Tensor) -> torch.Tensor:
    """Tensor in the working precision of the current mode (contiguous)."""
    return t.contiguous() if _mode == CUDA_64 else t.to(torch.float32).contiguous()


def _works(*fields):
    """Working-precision tensors of the given containers; the caller keeps the returned list
    alive until the library call has been issued (a temporary that is released early would let
    the allocator hand its memory to the next temporary)."""
    return [_work(f.data) for f in fields]


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


class _Base:
    def __init__(self, shape, ncomp: int):
        self.shape = Shape(shape)
        self._n = self.shape.getNumEl()
        self.data = torch.zeros(ncomp * self._n, dtype=torch.float64, device=_dev())

    def size(self) -> int:
        return self._n

    def dimX(self):
        return self.shape[0]

    def dimY(self):
        return self.shape[1] if len(self.shape) > 1 else 1

    def dimZ(self):
        return self.shape[2] if len(self.shape) > 2 else 1

    def clear(self):
        self.data.zero_()

    def scale(self, f):
        self.data.mul_(float(f))


class Matrix(_Base):
    """Scalar field on the GPU (matrix/matrix/scalar/Matrix.h)."""

    def __init__(self, shape):
        super().__init__(shape, 1)

    def fill(self, v):
        self.data.fill_(float(v))

    def assign(self, other: "Matrix"):
        self.data.copy_(other.data)

    def add(self, other: "Matrix", scale: float = 1.0):
        self.data.add_(other.data, alpha=float(scale))

    def get(self, *idx) -> float:
        return float(self.data[self._lin(idx)].item())

    def set(self, *args):
        *idx, v = args
        self.data[self._lin(idx)] = float(v)

    def _lin(self, idx):
        if len(idx) == 1:
            return int(idx[0])
        i = 0
        stride = 1
        for k, d in zip(idx, self.shape):
            i += int(k) * stride
            stride *= d
        return i

    def isUniform(self) -> bool:
        return bool((self.data == self.data[0]).all().item()) if self._n else True

    def getUniformValue(self) -> float:
        return float(self.data[0].item())

    uniform_value = property(getUniformValue)

    def absMax(self) -> float:
        return float(self.data.abs().max().item())

    def sum(self) -> float:
        return float(self.data.sum().item())

    def average(self) -> float:
        return self.sum() / self._n

    def to_numpy(self):
        return self.data.view(*reversed(self.shape)).cpu().numpy()


class VectorMatrix(_Base):
    """3-vector field on the GPU, SoA (matrix/matrix/vector/VectorMatrix.h)."""

    def __init__(self, shape):
        super().__init__(shape, 3)

    def comp(self, c: int) -> torch.Tensor:
        return self.data[c * self._n:(c + 1) * self._n]

    def fill(self, v):
        for c in range(3):
            self.comp(c).fill_(float(v[c]))

    def assign(self, other: "VectorMatrix"):
        self.data.copy_(other.data)

    def add(self, other: "VectorMatrix", scale: float = 1.0):
        self.data.add_(other.data, alpha=float(scale))

    def get(self, *idx):
        i = Matrix._lin(self, idx)
        return tuple(float(self.data[c * self._n + i].item()) for c in range(3))

    def set(self, *args):
        *idx, v = args
        i = Matrix._lin(self, idx)
        for c in range(3):
            self.data[c * self._n + i] = float(v[c])

    def normalize(self, length):
        """VectorMatrix::normalize(double) / normalize(Matrix) (VectorMatrix.cpp:205-230)."""
        if isinstance(length, Matrix):
            ms = length.data
        else:
            ms = torch.full((self._n,), float(length), dtype=torch.float64, device=self.data.device)
        if _mode == CUDA_64:
            check(lib().mm_normalize(_lib.MM_F64, self._n, _ptr(ms), _ptr(self.data), _stream()))
        else:
            w = _work(self.data)
            msw = _work(ms)
            check(lib().mm_normalize(_lib.MM_F32, self._n, _ptr(msw), _ptr(w), _stream()))
            self.data.copy_(w)

    def absMax(self) -> float:
        v = self.data.view(3, self._n)
        return float(torch.sqrt((v * v).sum(0).max()).item())

    def dotSum(self, other: "VectorMatrix") -> float:
        return float((self.data * other.data).sum().item())

    def average(self):
        return tuple((self.data.view(3, self._n).sum(1) / self._n).tolist())

    def sum(self):
        return tuple(self.data.view(3, self._n).sum(1).tolist())

    def to_numpy(self):
        return self.data.view(3, *reversed(self.shape)).cpu().numpy()

    def from_numpy(self, arr):
        self.data.copy_(torch.as_tensor(arr, dtype=torch.float64).reshape(-1))


def _mesh_of(f):
    mesh = getattr(f, "mesh", None)
    if mesh is None:
        raise RuntimeError("field has no mesh")
    return mesh


# ------------------------------------------------------------------------------------------------
# field terms
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
    out = _work(H.data) if _mode == CUDA_32 else H.data
    ms, a, m = _works(Ms, A, M)  # working-precision copies live until the call returns
    check(lib().mm_exchange(_prec(), nx, ny, nz, dx, dy, dz, int(px), int(py), int(pz),
                            _ptr(ms), _ptr(a), _ptr(m), _ptr(out), ctypes.byref(e), _stream()))
    if out is not H.data:
        H.data.copy_(out)
    return e.value


def uniaxial_anisotropy(axis, k, Ms, M, H) -> float:
    """bindings/mmm/anisotropy.i:24-31; returns sum_i k |a x m|^2 (CPU path's value)."""
    e = ctypes.c_double(0.0)
    out = _work(H.data) if _mode == CUDA_32 else H.data
    w = _works(axis, k, Ms, M)
    check(lib().mm_uniaxial_anisotropy(_prec(), M.size(), *[_ptr(t) for t in w], _ptr(out),
                                       ctypes.byref(e), _stream()))
    if out is not H.data:
        H.data.copy_(out)
    return e.value


def cubic_anisotropy(axis1, axis2, k, Ms, M, H) -> float:
    """bindings/mmm/anisotropy.i:32-39."""
    e = ctypes.c_double(0.0)
    out = _work(H.data) if _mode == CUDA_32 else H.data
    w = _works(axis1, axis2, k, Ms, M)
    check(lib().mm_cubic_anisotropy(_prec(), M.size(), *[_ptr(t) for t in w], _ptr(out),
                                    ctypes.byref(e), _stream()))
    if out is not H.data:
        H.data.copy_(out)
    return e.value


def llge(f1, f2, M, H, dM) -> None:
    """bindings/mmm/llge.i:24-29: dM = f1 M x H + f2 M x (M x H)."""
    out = _work(dM.data) if _mode == CUDA_32 else dM.data
    w = _works(f1, f2, M, H)
    check(lib().mm_llge(_prec(), M.size(), *[_ptr(t) for t in w], _ptr(out), _stream()))
    if out is not dM.data:
        dM.data.copy_(out)


def fdm_zhangli(nx, ny, nz, dx, dy, dz, do_precess, P, xi, Ms, alpha, j, M, dM) -> None:
    """bindings/mmm/zhangli.i:24-32."""
    out = _work(dM.data) if _mode == CUDA_32 else dM.data
    w = _works(P, xi, Ms, alpha, j, M)
    check(lib().mm_fdm_zhangli(_prec(), nx, ny, nz, dx, dy, dz, int(bool(do_precess)),
                               *[_ptr(t) for t in w], _ptr(out), _stream()))
    if out is not dM.data:
        dM.data.copy_(out)


def scaled_abs_max(M, scale) -> float:
    """bindings/math.i:66 (math/ScaledAbsMax.cpp:52-68)."""
    if scale.isUniform():
        return M.absMax() / scale.getUniformValue()
    r = ctypes.c_double(0.0)
    m, sc = _works(M, scale)
    check(lib().mm_scaled_abs_max(_prec(), M.size(), _ptr(m), _ptr(sc), ctypes.byref(r), _stream()))
    return r.value


# ------------------------------------------------------------------------------------------------
# demag
# ------------------------------------------------------------------------------------------------
def round_tensor_dimension(dim: int, periodic: bool, padding: int) -> int:
    return int(lib().mm_round_tensor_dimension(int(dim), int(bool(periodic)), int(padding)))


def GenerateDemagTensor(nx, ny, nz, dx, dy, dz, px, py, pz, repeat, padding, cache_dir=None) -> Matrix:
    """bindings/mmm/demag.i:27-42 (mmm/demag/demag_tensor.cpp:116-186), computed on the GPU.
    Returns Matrix(Shape(6, ex, ey, ez)) holding the negated tensor; periodic meshes are not
    supported by the GPU generator (RuntimeError)."""
    ex = round_tensor_dimension(nx, px, padding)
    ey = round_tensor_dimension(ny, py, padding)
    ez = round_tensor_dimension(nz, pz, padding)
    N = Matrix(Shape(6, ex, ey, ez))
    if px or py or pz:
        raise RuntimeError("GenerateDemagTensor: periodic boundaries are not supported on the GPU; "
                           "pass a tensor to SymmetricMatrixVectorConvolution_FFT instead")
    check(lib().mm_demag_tensor(nx, ny, nz, dx, dy, dz, ex, ey, ez, _ptr(N.data), _stream()))
    return N


class SymmetricMatrixVectorConvolution_FFT:
    """bindings/math.i:27-33: H = N * M for a tensor field N of shape (6, ex, ey, ez)."""

    def __init__(self, lhs: Matrix, nx: int, ny: int, nz: int):
        _, ex, ey, ez = lhs.shape
        self.dims = (nx, ny, nz)
        self._prec = _prec()
        h = ctypes.c_void_p()
        check(lib().mm_conv_create(ctypes.byref(h), self._prec, nx, ny, nz, ex, ey, ez,
                                   _ptr(lhs.data), _stream()))
        self._h = h

    def execute(self, rhs: VectorMatrix, res: VectorMatrix) -> None:
        if self._prec == _lib.MM_F64:
            check(lib().mm_conv_execute(self._h, _ptr(rhs.data), _ptr(res.data), _stream()))
        else:
            m = rhs.data.to(torch.float32)
            out = torch.empty_like(m)
            check(lib().mm_conv_execute(self._h, _ptr(m), _ptr(out), _stream()))
            res.data.copy_(out)

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
    keep = []
    for i, k in enumerate(ks):
        w = _work(k.data)
        keep.append(w)
        arr[i] = w.data_ptr()
    return arr, keep


def rk_prepare_step(step, h, tab, k0, k1, k2, k3, k4, k5, y, ytmp) -> None:
    """ytmp = y + h sum_{j<step} b[step][j] k_j (evolver/runge_kutta.cpp:32-48)."""
    ks = [k0, k1, k2, k3, k4, k5][:step]
    b = (ctypes.c_double * max(step, 1))(*[tab.getB(step, j) for j in range(step)])
    arr, keep = _kptrs(ks)
    out = _work(ytmp.data) if _mode == CUDA_32 else ytmp.data
    yw = _work(y.data)
    check(lib().mm_rk_prepare_step(_prec(), y.size(), int(step), float(h), b, arr,
                                   _ptr(yw), _ptr(out), _stream()))
    if out is not ytmp.data:
        ytmp.data.copy_(out)


def rk_combine_result(h, tab, *args) -> None:
    """y += h sum c_j k_j, y_error = h sum ec_j k_j (runge_kutta.cpp:72-96); k's then y, y_error."""
    *ks, y, y_err = args
    nk = len(ks)
    c = (ctypes.c_double * nk)(*[tab.getC(j) for j in range(nk)])
    ec = (ctypes.c_double * nk)(*[tab.getEC(j) for j in range(nk)])
    arr, keep = _kptrs(ks)
    yw = _work(y.data) if _mode == CUDA_32 else y.data
    ew = _work(y_err.data) if _mode == CUDA_32 else y_err.data
    check(lib().mm_rk_combine_result(_prec(), y.size(), nk, float(h), c, ec, arr, _ptr(yw), _ptr(ew),
                                     _stream()))
    if yw is not y.data:
        y.data.copy_(yw)
        y_err.data.copy_(ew)
