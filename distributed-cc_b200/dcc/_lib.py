"""ctypes binding of libdcc_b200.so, in the manner of the reference's
distr_cc/_lib.py (one CDLL at a fixed in-tree path, argtypes/restype set per
symbol, dtype and contiguity checks before every call).

Differences from the reference loader:
  * buffers are torch CUDA tensors (device pointers), plus a device check;
  * every call returns a status which is turned into DccError;
  * the library must exist: there is no CPU fallback.  A missing library
    raises ImportError telling how to build it.
"""
from __future__ import annotations

import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdcc_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError("libdcc_b200.so not built (%s); run `python distributed-cc_b200/build.py`" % LIB_PATH)

_lib = ctypes.CDLL(LIB_PATH)

c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_int = ctypes.c_int
c_str = ctypes.c_char_p
c_size = ctypes.c_size_t

DCC_OK = 0
STATUS_NAMES = {
    1: "DCC_ERR_PATTERN", 2: "DCC_ERR_SHAPE", 3: "DCC_ERR_NULL", 4: "DCC_ERR_CUDA", 5: "DCC_ERR_TIMEOUT",
    6: "DCC_ERR_UNSUPPORTED", 7: "DCC_ERR_NOT_LOCAL", 8: "DCC_ERR_WORKSPACE",
}


class DccError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS_NAMES.get(code, code), msg))
        self.code = code


_lib.dcc_last_error.restype = c_str
_lib.dcc_last_error.argtypes = []
_lib.dcc_version.restype = c_int
_lib.dcc_version.argtypes = []

# symbol -> argtypes (restype int unless listed in _SIZE_FUNCS)
_SIGS = {
    "dcc_t3_single_spin_summation_inplace": [c_vp, c_i64, c_str, c_dbl, c_dbl, c_vp],
    "dcc_t3_spin_summation_inplace": [c_vp, c_i64, c_i64, c_str, c_dbl, c_dbl, c_vp],
    "dcc_t3_unpack_p3": [c_vp, c_vp, c_vp, c_i64, c_i64, c_str, c_dbl, c_dbl, c_vp],
    "dcc_t3_spin_summation": [c_vp, c_vp, c_i64, c_i64, c_str, c_dbl, c_dbl, c_vp],
    "dcc_t3_spin_summation_f32": [c_vp, c_vp, c_i64, c_i64, c_str, c_dbl, c_dbl, c_vp],
    "dcc_t3_spin_summation_kernel": [c_vp, c_vp, c_i64, c_i64, c_str, c_dbl, c_dbl, c_int, c_vp],
    "dcc_t3_spin_summation_triple_sym": [c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_t3_transpose_add": [c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_t3_symmetrize_status": [c_vp, c_vp],
    "dcc_t3_orbit_roundtrip": [c_vp, c_i64, c_i64, c_vp],
    "dcc_take_t3_ijk_single": [c_vp, c_vp, c_vp] + [c_i64] * 5 + [c_vp],
    "dcc_take_t3_batched": [c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_vp],
    "dcc_fill_local_data_ijk": [c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_r3_tri_divide_e": [c_vp, c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_t3_divide_update": [c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_int, c_vp, c_vp, c_size, c_vp],
    "dcc_redistribute_ijk_to_abc": [c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_fill_t3_from_abc": [c_vp] + [c_i64] * 6 + [c_vp, c_i64, c_vp],
    "dcc_t4_project_1_minus_p4_p31_inplace": [c_vp, c_i64, c_i64, c_dbl, c_dbl, c_vp],
    "dcc_t4_spin_summation_inplace": [c_vp, c_i64, c_i64, c_str, c_dbl, c_dbl, c_vp],
    "dcc_t4_transpose_add": [c_vp, c_vp, c_i64, c_vp],
    "dcc_t4_spin_summation_quadruple_sym": [c_vp] * 5 + [c_i64, c_vp],
    "dcc_t4_transpose_add_batched": [c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_t4_spin_summation_quadruple_sym_batched": [c_vp] * 5 + [c_i64, c_i64, c_vp],
    "dcc_t4_strings": [c_vp, c_vp, ctypes.c_int, c_vp, ctypes.c_int, c_vp, c_i64, c_vp, c_vp, ctypes.c_int, c_i64,
                       c_i64, c_i64, ctypes.c_double, c_vp, c_vp, c_vp],
    "dcc_t4_strings_rows_per_cta": [c_i64, c_i64],
    "dcc_r4_local_tri_divide_e": [c_vp, c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_unpack_t4_ijkl_single": [c_vp, c_vp, c_vp] + [c_i64] * 6 + [c_vp],
    "dcc_fill_local_data_ijkl": [c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_vp],
    "dcc_t4_add": [c_vp, c_vp, c_i64, c_vp],
    "dcc_e_abcdijkl_division": [c_vp, c_vp, c_vp] + [c_i64] * 13 + [c_vp],
    "dcc_t4_multiply_factor": [c_vp, c_vp] + [c_i64] * 5 + [c_vp],
    "dcc_q_task_epilogue": [c_vp] * 6 + [c_i64] * 11 + [c_vp, c_vp, c_size, c_vp],
    "dcc_q_group_epilogue": [c_vp, c_vp, c_int] + [c_vp] * 4 + [c_i64] * 10 + [c_vp, c_vp, c_size, c_vp],
    "dcc_q_group_epilogue_workspace_bytes": [],
    "dcc_t3_update_workspace_bytes": [c_i64, c_i64],
    "dcc_q_epilogue_workspace_bytes": [c_i64, c_i64],
}
_SIZE_FUNCS = {"dcc_t3_update_workspace_bytes", "dcc_q_epilogue_workspace_bytes",
               "dcc_q_group_epilogue_workspace_bytes"}


def _bind(name, args):
    f = getattr(_lib, name, None)
    if f is None:
        return None
    f.argtypes = args
    f.restype = c_size if name in _SIZE_FUNCS else c_int
    return f


for _n, _a in list(_SIGS.items()):
    _bind(_n, _a)


def bind(name, args, restype=c_int):
    """Bind an additional symbol (used by modules that extend the ABI)."""
    f = getattr(_lib, name)
    f.argtypes = args
    f.restype = restype
    return f


def lib():
    return _lib


def last_error():
    return (_lib.dcc_last_error() or b"").decode()


def check(rc):
    if rc != DCC_OK:
        raise DccError(rc, last_error())
    return rc


def call(name, *args):
    return check(getattr(_lib, name)(*args))


def stream_ptr(stream=None):
    s = torch.cuda.current_stream() if stream is None else stream
    return c_vp(s.cuda_stream)


def as_tensor(t, dtype, name, device_required=True):
    """Validate a buffer the way distr_cc/_lib.py:_as_array does (dtype,
    C-contiguity), plus the CUDA-device check of this library."""
    if not isinstance(t, torch.Tensor):
        raise TypeError("%s must be a torch.Tensor on a CUDA device" % name)
    if t.dtype != dtype:
        raise TypeError("%s must have dtype %s" % (name, dtype))
    if not t.is_contiguous():
        raise ValueError("%s must be C-contiguous" % name)
    if device_required and not t.is_cuda:
        raise ValueError("%s must live on a CUDA device" % name)
    return t


def ptr(t):
    return c_vp(t.data_ptr()) if t is not None else c_vp(None)


def pattern(p):
    if not isinstance(p, (str, bytes)):
        raise TypeError("pattern must be a string")
    return p.encode() if isinstance(p, str) else p
