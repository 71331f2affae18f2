"""ctypes binding of libmmb200.so, the C ABI declared in include/mmb200.h.

The library is built in-tree (``micromagnum_b200/libmmb200.so``, see ``build()``).  Loading
fails loudly when it is missing: there is no CPU implementation behind this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmmb200.so")

MM_OK = 0
STATUS_NAMES = {
    0: "MM_OK", 1: "MM_ERR_INVALID_ARGUMENT", 2: "MM_ERR_CUDA", 3: "MM_ERR_OUT_OF_MEMORY",
    4: "MM_ERR_UNSUPPORTED", 5: "MM_ERR_NOT_FINITE", 6: "MM_ERR_TIMEOUT",
}
MM_F64, MM_F32 = 0, 1
MM_RK_RKF45, MM_RK_CC45, MM_RK_DP54, MM_RK_RK23 = 0, 1, 2, 3
MM_TERM_DEMAG, MM_TERM_EXCHANGE, MM_TERM_UNIAXIAL = 1, 2, 4
MM_TERM_CUBIC, MM_TERM_ZHANGLI, MM_TERM_ZEEMAN = 8, 16, 32
MM_RELAX_DEG_PER_NS, MM_RELAX_TORQUE = 0, 1


class MMError(RuntimeError):
    """A failed mmb200 call (the reference raises RuntimeError from its SWIG layer)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class mm_material(ctypes.Structure):
    _fields_ = [
        ("Ms", ctypes.c_double), ("A", ctypes.c_double), ("alpha", ctypes.c_double),
        ("k_uniaxial", ctypes.c_double), ("k_cubic", ctypes.c_double),
        ("axis1", ctypes.c_double * 3), ("axis2", ctypes.c_double * 3),
        ("P", ctypes.c_double), ("xi", ctypes.c_double), ("j", ctypes.c_double * 3),
    ]


class mm_solver_config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("precision", ctypes.c_int), ("tableau", ctypes.c_int), ("terms", ctypes.c_int),
        ("do_precess", ctypes.c_int), ("zl_do_precess", ctypes.c_int), ("padding", ctypes.c_int),
        ("eps_abs", ctypes.c_double), ("eps_rel", ctypes.c_double), ("h0", ctypes.c_double),
        ("H_ext", ctypes.c_double * 3), ("H_pulse", ctypes.c_double * 3),
        ("pulse_rise", ctypes.c_double), ("fsal_reuse_after_reject", ctypes.c_int),
        ("pbc", ctypes.c_int * 3), ("pbc_repeat", ctypes.c_int),
    ]


class mm_batch_instance(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("Ms", ctypes.c_double), ("A", ctypes.c_double), ("alpha", ctypes.c_double),
        ("H_ext", ctypes.c_double * 3), ("H_pulse", ctypes.c_double * 3), ("pulse_rise", ctypes.c_double),
        ("t_end", ctypes.c_double),
    ]


class mm_batch_config(ctypes.Structure):
    _fields_ = [
        ("precision", ctypes.c_int), ("eps_abs", ctypes.c_double), ("eps_rel", ctypes.c_double),
        ("h0", ctypes.c_double), ("max_torque", ctypes.c_double), ("check_every_nth_step", ctypes.c_int),
    ]


class mm_batch_result(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int), ("steps", ctypes.c_int), ("attempts", ctypes.c_int), ("rejected", ctypes.c_int),
        ("t", ctypes.c_double), ("h", ctypes.c_double),
    ]


class mm_solver_stats(ctypes.Structure):
    _fields_ = [
        ("t", ctypes.c_double), ("h", ctypes.c_double), ("h_next", ctypes.c_double),
        ("steps", ctypes.c_int64), ("attempts", ctypes.c_int64), ("rejected", ctypes.c_int64),
        ("last_error", ctypes.c_double), ("last_max_dmdt", ctypes.c_double),
        ("not_finite", ctypes.c_int), ("stage_kernel", ctypes.c_int),
    ]


# (name, restype, argtypes) for every entry point of include/mmb200.h
class mm_omf_header(ctypes.Structure):
    _fields_ = [
        ("title", ctypes.c_char * 256), ("desc", ctypes.c_char * 4096), ("meshunit", ctypes.c_char * 64),
        ("valueunit", ctypes.c_char * 64), ("meshtype", ctypes.c_char * 64), ("valuemultiplier", ctypes.c_double),
        ("xmin", ctypes.c_double), ("ymin", ctypes.c_double), ("zmin", ctypes.c_double),
        ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
        ("ValueRangeMaxMag", ctypes.c_double), ("ValueRangeMinMag", ctypes.c_double),
        ("xbase", ctypes.c_double), ("ybase", ctypes.c_double), ("zbase", ctypes.c_double),
        ("xstepsize", ctypes.c_double), ("ystepsize", ctypes.c_double), ("zstepsize", ctypes.c_double),
        ("xnodes", ctypes.c_int), ("ynodes", ctypes.c_int), ("znodes", ctypes.c_int), ("format", ctypes.c_int),
    ]


MM_OMF_TEXT, MM_OMF_BINARY_4, MM_OMF_BINARY_8 = 0, 1, 2

_VP, _D, _I, _SZ = ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_size_t
_DP = ctypes.POINTER(ctypes.c_double)
_PROTOS = [
    ("mm_last_error", ctypes.c_char_p, []),
    ("mm_abi_version", _I, []),
    ("mm_kernel_launch_count", ctypes.c_uint64, []),
    ("mm_profile_enable", _I, [_I]),
    ("mm_profile_reset", _I, []),
    ("mm_profile_count", _I, []),
    ("mm_profile_get", _I, [_I, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int64), _DP, _DP]),
    ("mm_exchange", _I, [_I, _I, _I, _I, _D, _D, _D, _I, _I, _I, _VP, _VP, _VP, _VP, _DP, _VP]),
    ("mm_uniaxial_anisotropy", _I, [_I, _SZ, _VP, _VP, _VP, _VP, _VP, _DP, _VP]),
    ("mm_cubic_anisotropy", _I, [_I, _SZ, _VP, _VP, _VP, _VP, _VP, _VP, _DP, _VP]),
    ("mm_llge", _I, [_I, _SZ, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("mm_fdm_zhangli", _I, [_I, _I, _I, _I, _D, _D, _D, _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    ("mm_scaled_abs_max", _I, [_I, _SZ, _VP, _VP, _DP, _VP]),
    ("mm_scaled_abs_max_noalloc", _I, [_I, _SZ, _VP, _VP, _DP, _VP]),
    ("mm_rk_scaled_error_norm", _I, [_I, _SZ, _D, _D, _VP, _VP, _DP, _VP]),
    ("mm_normalize", _I, [_I, _SZ, _VP, _VP, _VP]),
    ("mm_rk_prepare_step", _I, [_I, _SZ, _I, _D, _DP, ctypes.POINTER(_VP), _VP, _VP, _VP]),
    ("mm_rk_combine_result", _I, [_I, _SZ, _I, _D, _DP, _DP, ctypes.POINTER(_VP), _VP, _VP, _VP]),
    ("mm_round_tensor_dimension", _I, [_I, _I, _I]),
    ("mm_demag_tensor", _I, [_I, _I, _I, _D, _D, _D, _I, _I, _I, _VP, _VP]),
    ("mm_demag_tensor_periodic", _I, [_I, _I, _I, _D, _D, _D, _I, _I, _I, _I, _I, _I, _I, _VP, _VP]),
    ("mm_conv_create", _I, [ctypes.POINTER(_VP), _I, _I, _I, _I, _I, _I, _I, _VP, _VP]),
    ("mm_conv_execute", _I, [_VP, _VP, _VP, _VP]),
    ("mm_conv_destroy", _I, [_VP]),
    ("mm_solver_create", _I, [ctypes.POINTER(_VP), ctypes.POINTER(mm_solver_config), _I,
                              ctypes.POINTER(mm_material), _VP, _VP, _VP]),
    ("mm_solver_destroy", _I, [_VP]),
    ("mm_solver_set_M", _I, [_VP, _VP, _VP]),
    ("mm_solver_get_M", _I, [_VP, _VP, _VP]),
    ("mm_solver_load_M", _I, [_VP, _VP, _VP]),
    ("mm_solver_set_time", _I, [_VP, _D, _D, _VP]),
    ("mm_solver_step", _I, [_VP, _D, _VP]),
    ("mm_solver_run", _I, [_VP, _D, _D, _DP, _DP, _I, ctypes.POINTER(_I), _VP]),
    ("mm_solver_attempt", _I, [_VP, _D, _VP]),
    ("mm_solver_eval", _I, [_VP, _VP, _VP, _VP, _VP]),
    ("mm_solver_stats_get", _I, [_VP, ctypes.POINTER(mm_solver_stats), _VP]),
    ("mm_solver_average_M", _I, [_VP, _DP, _VP]),
    ("mm_solver_relax_norms", _I, [_VP, _DP, _VP]),
    ("mm_solver_energies", _I, [_VP, _DP, _VP]),
    ("mm_batch_instance_bytes", _I, [ctypes.POINTER(mm_batch_instance), _I, ctypes.POINTER(_SZ),
                                     ctypes.POINTER(_SZ)]),
    ("mm_batch_add", _I, [_VP, ctypes.POINTER(mm_batch_instance), _VP, ctypes.POINTER(_I), _VP]),
    ("mm_batch_remove", _I, [_VP, _I]),
    ("mm_batch_slot_count", _I, [_VP]),
    ("mm_batch_stop", _I, [_VP, _I, _VP]),
    ("mm_batch_create", _I, [ctypes.POINTER(_VP), ctypes.POINTER(mm_batch_config), _I,
                             ctypes.POINTER(mm_batch_instance), _VP, _VP]),
    ("mm_batch_destroy", _I, [_VP]),
    ("mm_batch_set_M", _I, [_VP, _I, _VP, _VP]),
    ("mm_batch_get_M", _I, [_VP, _I, _VP, _VP]),
    ("mm_batch_relax", _I, [_VP, ctypes.c_longlong, _I, ctypes.POINTER(ctypes.c_longlong), _VP]),
    ("mm_batch_results", _I, [_VP, ctypes.POINTER(mm_batch_result), _VP]),
    ("mm_batch_launches_per_round", _I, [_VP, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("mm_solver_relax", _I, [_VP, _I, _D, _I, ctypes.c_longlong, ctypes.POINTER(ctypes.c_int), _DP, _VP]),
    ("mm_omf_parse", _I, [_VP, _SZ, ctypes.POINTER(mm_omf_header), _I, _VP, _VP]),
    ("mm_omf_read", _I, [ctypes.c_char_p, ctypes.POINTER(mm_omf_header), _I, _VP, _VP]),
    ("mm_omf_format", _I, [ctypes.POINTER(mm_omf_header), _I, _VP, _I, ctypes.POINTER(_VP), ctypes.POINTER(_SZ),
                           _VP]),
    ("mm_omf_free", None, [_VP]),
    ("mm_omf_write", _I, [ctypes.c_char_p, ctypes.POINTER(mm_omf_header), _I, _VP, _I, _VP]),
]

EXPORTED = [p[0] for p in _PROTOS]

_lib = None


def build(force: bool = False) -> str:
    """Compile libmmb200.so for sm_100a with nvcc (micromagnum_b200/csrc/Makefile)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), "-j4"], check=True)
    return LIB_PATH


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with micromagnum_b200.build() "
                "(nvcc, sm_100a); there is no CPU implementation")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _PROTOS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != MM_OK:
        msg = lib().mm_last_error()
        raise MMError(status, msg.decode() if msg else "")


def launches() -> int:
    return int(lib().mm_kernel_launch_count())


def profile_enable(on: bool = True) -> None:
    check(lib().mm_profile_enable(int(on)))


def profile_reset() -> None:
    check(lib().mm_profile_reset())


def profile_read() -> dict:
    """{kernel name: (launches, total device ms, total algorithmic bytes)} (synchronises)."""
    out = {}
    for i in range(lib().mm_profile_count()):
        name = ctypes.c_char_p()
        cnt = ctypes.c_int64()
        ms = ctypes.c_double()
        by = ctypes.c_double()
        check(lib().mm_profile_get(i, ctypes.byref(name), ctypes.byref(cnt), ctypes.byref(ms), ctypes.byref(by)))
        out[name.value.decode()] = (cnt.value, ms.value, by.value)
    return out
