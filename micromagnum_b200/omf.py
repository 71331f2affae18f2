"""OMF 1.0 files of device fields: the wire format of served requests and results.

Thin wrappers of the library's mm_omf_parse / mm_omf_format (csrc/omf.cu), which replace the
reference's readOMF / writeOMF (src/magneto/mmm/io/OMFImport.cpp, OMFExport.cpp) for fields that
live on the GPU: binary payloads are byte-swapped and de-interleaved by a kernel, text payloads are
parsed by host threads.  Fields are (3, N) SoA tensors, x fastest, in A/m.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import torch

from . import _lib
from ._lib import check, lib

TEXT, BINARY_4, BINARY_8 = _lib.MM_OMF_TEXT, _lib.MM_OMF_BINARY_4, _lib.MM_OMF_BINARY_8


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def header_of(data: bytes) -> _lib.mm_omf_header:
    """The header of an OMF file held in memory (host only)."""
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    h = _lib.mm_omf_header()
    check(lib().mm_omf_parse(buf, len(data), ctypes.byref(h), 0, None, None))
    return h


def parse(data: bytes, dtype=torch.float64):
    """(header, field): the field of an OMF file held in memory as a (3, N) CUDA tensor of
    `dtype`, scaled by the header's valuemultiplier."""
    buf = ctypes.create_string_buffer(bytes(data), len(data))
    h = _lib.mm_omf_header()
    check(lib().mm_omf_parse(buf, len(data), ctypes.byref(h), 0, None, None))
    n = h.xnodes * h.ynodes * h.znodes
    out = torch.empty(3 * n, dtype=dtype, device="cuda")
    prec = _lib.MM_F64 if dtype == torch.float64 else _lib.MM_F32
    check(lib().mm_omf_parse(buf, len(data), ctypes.byref(h), prec, ctypes.c_void_p(out.data_ptr()), _stream()))
    return h, out.view(3, n)


def format(M: torch.Tensor, dims: Sequence[int], delta: Sequence[float], fmt: int = BINARY_8, title: str = "",
           desc: Sequence[str] = (), valueunit: str = "A/m") -> bytes:
    """The OMF file of a (3, N) or (3N,) CUDA field on an nx x ny x nz mesh, with the header the
    reference's writeOMF helper fills in (src/magnum/micromagnetics/io/write_omf.py:25-52)."""
    nx, ny, nz = (int(v) for v in dims)
    dx, dy, dz = (float(v) for v in delta)
    M = M.reshape(-1).contiguous()
    if M.numel() != 3 * nx * ny * nz:
        raise ValueError("the field does not match the mesh")
    h = _lib.mm_omf_header()
    h.title = title.encode()[:255]
    h.desc = "\n".join(desc).encode()[:4095]
    h.meshunit, h.valueunit, h.meshtype = b"m", valueunit.encode()[:63], b"rectangular"
    h.valuemultiplier = 1.0
    h.xmax, h.ymax, h.zmax = nx * dx, ny * dy, nz * dz
    h.xbase, h.ybase, h.zbase = dx / 2, dy / 2, dz / 2
    h.xstepsize, h.ystepsize, h.zstepsize = dx, dy, dz
    h.xnodes, h.ynodes, h.znodes = nx, ny, nz
    prec = _lib.MM_F64 if M.dtype == torch.float64 else _lib.MM_F32
    out, length = ctypes.c_void_p(), ctypes.c_size_t(0)
    check(lib().mm_omf_format(ctypes.byref(h), prec, ctypes.c_void_p(M.data_ptr()), int(fmt), ctypes.byref(out),
                              ctypes.byref(length), _stream()))
    try:
        return ctypes.string_at(out.value, length.value)
    finally:
        lib().mm_omf_free(out)
