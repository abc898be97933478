"""TEST ORACLE ONLY -- ctypes access to the C restatement (``dcc_oracle.c``) and to
the reference C helpers compiled from the reference sources (``_ref/``).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this module.  The shipped library never calls it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libdcc_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libdistr_cc_ref.so")

P3_PATTERNS = {"P3_full": 0, "P3_422": 1, "P3_201": 2}
P4_PATTERNS = {"P4_full": 0, "P4_444": 1, "P4_442": 2, "P4_201": 3}

_i64 = ctypes.c_int64
_dbl = ctypes.c_double
_vp = ctypes.c_void_p


def build(reference_dir=None):
    """Compile the C restatement, and the reference library when `reference_dir` (default:
    the DCC_REFERENCE environment variable) names a reference checkout with its sources."""
    reference_dir = reference_dir or os.environ.get("DCC_REFERENCE")
    cmd = ["make", "-s", "-C", HERE]
    if reference_dir and os.path.isdir(os.path.join(reference_dir, "src")):
        cmd.append("REF_SRC=%s" % os.path.join(reference_dir, "src"))
    subprocess.run(cmd, check=True)


def _ptr(a):
    return a.ctypes.data_as(_vp)


def _chk(a, dtype):
    if a.dtype != np.dtype(dtype) or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("oracle buffers must be C-contiguous %s" % np.dtype(dtype))
    return a


class Oracle:
    """The C restatement of the reference helpers."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            build()
        self.lib = L = ctypes.CDLL(path)
        L.oracle_ijk_to_linear.restype = _i64
        L.oracle_ijk_to_linear.argtypes = [_i64] * 4
        L.oracle_ijkl_to_linear.restype = _i64
        L.oracle_ijkl_to_linear.argtypes = [_i64] * 5
        L.oracle_abc_index.restype = _i64
        L.oracle_abc_index.argtypes = [_i64] * 4
        L.oracle_q_factor.restype = _dbl
        L.oracle_q_factor.argtypes = [_i64] * 4
        L.oracle_take_t3.restype = ctypes.c_int
        L.oracle_take_t3.argtypes = [_vp, _vp, _vp] + [_i64] * 5
        L.oracle_gather_t3.restype = None
        L.oracle_gather_t3.argtypes = [_vp, _vp, _vp, _vp, _i64, _i64]
        L.oracle_t3_spin_sum.restype = ctypes.c_int
        L.oracle_t3_spin_sum.argtypes = [_vp, _i64, _i64, ctypes.c_int, _dbl, _dbl]
        L.oracle_t3_triple_sym.restype = None
        L.oracle_t3_triple_sym.argtypes = [_vp, _vp, _vp, _vp, _i64]
        L.oracle_t3_transpose_add.restype = None
        L.oracle_t3_transpose_add.argtypes = [_vp, _vp, _i64]
        L.oracle_r3_divide.restype = None
        L.oracle_r3_divide.argtypes = [_vp, _vp, _vp, _i64, _i64]
        L.oracle_t4_spin_sum.restype = ctypes.c_int
        L.oracle_t4_spin_sum.argtypes = [_vp, _i64, _i64, ctypes.c_int, _dbl, _dbl]
        L.oracle_t4_project.restype = None
        L.oracle_t4_project.argtypes = [_vp, _i64, _i64, _dbl, _dbl]
        L.oracle_t4_transpose_add.restype = None
        L.oracle_t4_transpose_add.argtypes = [_vp, _vp, _i64]
        L.oracle_t4_quadruple_sym.restype = None
        L.oracle_t4_quadruple_sym.argtypes = [_vp] * 5 + [_i64]
        L.oracle_r4_divide.restype = None
        L.oracle_r4_divide.argtypes = [_vp, _vp, _vp, _i64, _i64]
        L.oracle_unpack_t4.restype = ctypes.c_int
        L.oracle_unpack_t4.argtypes = [_vp, _vp, _vp] + [_i64] * 6
        L.oracle_e_abcdijkl_division.restype = None
        L.oracle_e_abcdijkl_division.argtypes = [_vp, _vp, _vp] + [_i64] * 12
        L.oracle_t4_multiply_factor.restype = None
        L.oracle_t4_multiply_factor.argtypes = [_vp, _vp] + [_i64] * 5
        L.oracle_fill_t3_abc.restype = _i64
        L.oracle_fill_t3_abc.argtypes = [_vp] + [_i64] * 6 + [_vp, _vp, _i64]
        L.oracle_ijk_to_abc.restype = None
        L.oracle_ijk_to_abc.argtypes = [_vp, _vp, _i64, _i64]

    # --- maps
    def ijk_to_linear(self, i, j, k, nocc):
        return self.lib.oracle_ijk_to_linear(i, j, k, nocc)

    def ijkl_to_linear(self, i, j, k, l, nocc):
        return self.lib.oracle_ijkl_to_linear(i, j, k, l, nocc)

    def abc_index(self, a, b, c, nvir):
        return self.lib.oracle_abc_index(a, b, c, nvir)

    def q_factor(self, a, b, c, d):
        return self.lib.oracle_q_factor(a, b, c, d)

    # --- T3
    def take_t3(self, t3_local, ijk_to_local, i, j, k, nocc, nvir, out=None):
        out = np.zeros((nvir,) * 3) if out is None else out
        rc = self.lib.oracle_take_t3(_ptr(_chk(t3_local, np.float64)), _ptr(_chk(out, np.float64)),
                                     _ptr(_chk(ijk_to_local, np.int64)), i, j, k, nocc, nvir)
        return out, rc

    def gather_t3(self, t3_local, requests, ijk_to_local, nvir):
        out = np.zeros((len(requests),) + (nvir,) * 3)
        self.lib.oracle_gather_t3(_ptr(_chk(t3_local, np.float64)), _ptr(out), _ptr(_chk(requests, np.int32)),
                                  _ptr(_chk(ijk_to_local, np.int64)), len(requests), nvir)
        return out

    def t3_spin_sum(self, A, nvir, pattern, alpha=1.0, beta=0.0):
        A = _chk(A, np.float64)
        nblk = A.size // nvir ** 3
        rc = self.lib.oracle_t3_spin_sum(_ptr(A), nblk, nvir, P3_PATTERNS[pattern], alpha, beta)
        if rc:
            raise ValueError(pattern)
        return A

    def t3_triple_sym(self, A, nvir):
        B = [np.empty_like(A) for _ in range(3)]
        self.lib.oracle_t3_triple_sym(_ptr(_chk(A, np.float64)), _ptr(B[0]), _ptr(B[1]), _ptr(B[2]), nvir)
        return B

    def t3_transpose_add(self, A, nvir):
        B = np.empty_like(A)
        self.lib.oracle_t3_transpose_add(_ptr(_chk(A, np.float64)), _ptr(B), nvir)
        return B

    def r3_divide(self, r3, eia, ijk):
        nblk, nvir = r3.shape[0], r3.shape[1]
        self.lib.oracle_r3_divide(_ptr(_chk(r3, np.float64)), _ptr(_chk(eia, np.float64)),
                                  _ptr(_chk(ijk, np.int32)), nblk, nvir)
        return r3

    # --- T4
    def t4_spin_sum(self, A, nouter, nvir, pattern, alpha=1.0, beta=0.0):
        rc = self.lib.oracle_t4_spin_sum(_ptr(_chk(A, np.float64)), nouter, nvir, P4_PATTERNS[pattern], alpha, beta)
        if rc:
            raise ValueError(pattern)
        return A

    def t4_project(self, A, nouter, nvir, alpha=1.0, beta=0.0):
        self.lib.oracle_t4_project(_ptr(_chk(A, np.float64)), nouter, nvir, alpha, beta)
        return A

    def t4_transpose_add(self, src, nvir):
        dst = np.empty_like(src)
        self.lib.oracle_t4_transpose_add(_ptr(_chk(src, np.float64)), _ptr(dst), nvir)
        return dst

    def t4_quadruple_sym(self, src, nvir):
        B = [np.empty_like(src) for _ in range(4)]
        self.lib.oracle_t4_quadruple_sym(_ptr(_chk(src, np.float64)), *[_ptr(b) for b in B], nvir)
        return B

    def r4_divide(self, r4, eia, ijkl):
        self.lib.oracle_r4_divide(_ptr(_chk(r4, np.float64)), _ptr(_chk(eia, np.float64)),
                                  _ptr(_chk(ijkl, np.int32)), r4.shape[0], r4.shape[1])
        return r4

    def unpack_t4(self, t4_local, ijkl_to_local, i, j, k, l, nocc, nvir, out=None):
        out = np.zeros((nvir,) * 4) if out is None else out
        rc = self.lib.oracle_unpack_t4(_ptr(_chk(t4_local, np.float64)), _ptr(_chk(out, np.float64)),
                                       _ptr(_chk(ijkl_to_local, np.int64)), i, j, k, l, nocc, nvir)
        return out, rc

    # --- (Q)
    def e_abcdijkl_division(self, r4, e_occ, e_vir, a0, a1, b0, b1, c0, c1, d0, d1, blk_b, blk_c, blk_d, nocc):
        self.lib.oracle_e_abcdijkl_division(_ptr(_chk(r4, np.float64)), _ptr(_chk(e_occ, np.float64)),
                                            _ptr(_chk(e_vir, np.float64)), a0, a1, b0, b1, c0, c1, d0, d1,
                                            blk_b, blk_c, blk_d, nocc)
        return r4

    def t4_multiply_factor(self, t4, factor, ba, bb, bc, bd, nocc):
        self.lib.oracle_t4_multiply_factor(_ptr(_chk(t4, np.float64)), _ptr(_chk(factor, np.float64)),
                                           ba, bb, bc, bd, nocc)
        return t4

    def fill_t3_abc(self, target, a0, a1, b0, b1, nvir, nocc, t3_abc, present, ld_b):
        pres = None if present is None else _chk(present, np.uint8)
        return self.lib.oracle_fill_t3_abc(_ptr(_chk(target, np.float64)), a0, a1, b0, b1, nvir, nocc,
                                           _ptr(_chk(t3_abc, np.float64)), None if pres is None else _ptr(pres),
                                           ld_b)

    def ijk_to_abc(self, t3_ijk, nocc, nvir):
        nabc = nvir * (nvir + 1) * (nvir + 2) // 6
        out = np.zeros((nabc, nocc, nocc, nocc))
        self.lib.oracle_ijk_to_abc(_ptr(_chk(t3_ijk, np.float64)), _ptr(out), nocc, nvir)
        return out


class Reference:
    """The reference's own C helpers, compiled from the reference sources by
    ``oracle/Makefile`` (ctypes signatures follow distr_cc/_c_rccsdt.py,
    distr_cc/_c_rccsdt_q.py and distr_cc/_c_rccsdtq.py)."""

    def __init__(self, path=REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = L = ctypes.CDLL(path)
        cp = ctypes.c_char_p
        sig = {
            "t3_single_spin_summation_inplace_": [_vp, _i64, cp, _dbl, _dbl],
            "t3_transpose_add_": [_vp, _vp, _i64],
            "t3_spin_summation_triple_sym_": [_vp, _vp, _vp, _vp, _i64],
            "fill_local_data_ijk_": [_vp, _vp, _vp, _vp, _i64, _i64],
            "take_t3_ijk_single_": [_vp, _vp, _vp] + [_i64] * 5,
            "pack_redistributed_send_buffer_c": [_i64, _i64, _i64] + [_vp] * 9,
            "unpack_received_data_indices": [_vp, _vp, _vp, _vp, _vp, ctypes.c_int, _i64, _i64],
            "t4_spin_summation_inplace_": [_vp, _i64, _i64, cp, _dbl, _dbl],
            "fill_t3_from_ptr_array": [_vp] + [_i64] * 6 + [_vp, _i64, _i64, _i64],
            "e_abcdijkl_division_": [_vp, _vp, _vp] + [_i64] * 13,
            "t4_multiply_factor_": [_vp, _vp] + [_i64] * 5,
            "t4_project_1_minus_p4_p31_inplace_": [_vp, _i64, _i64, _dbl, _dbl],
            "t4_single_spin_summation_inplace_": [_vp, _i64, cp, _dbl, _dbl],
            "t4_transpose_add_": [_vp, _vp, _i64],
            "t4_spin_summation_quadruple_sym_": [_vp] * 5 + [_i64],
            "r4_local_tri_divide_e_": [_vp, _vp, _vp, _i64, _i64],
            "fill_local_data_ijkl_": [_vp, _vp, _vp, _vp, _i64, _i64],
            "unpack_t4_ijkl_single_": [_vp, _vp, _vp] + [_i64] * 6,
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = None

    def __getattr__(self, name):
        return getattr(self.lib, name)

    def ijk_to_abc_records(self, t3_ijk, nocc, nvir):
        """Run the reference IJK->ABC record pack + unpack at one rank.  The pack
        maps of distr_cc/distribute_t3.py:1419-1488 are restated in numpy; the
        packing and scattering are the reference's C code."""
        a, b, c = np.mgrid[0:nvir, 0:nvir, 0:nvir]
        perms = [(a, b, c), (a, c, b), (b, a, c), (b, c, a), (c, a, b), (c, b, a)]
        abc_list = [(x, y, z) for x in range(nvir) for y in range(x, nvir) for z in range(y, nvir)]
        gidx = {t: g for g, t in enumerate(abc_list)}
        flat = np.arange(nvir ** 3).reshape(nvir, nvir, nvir)
        pk_idx, pk_g, pk_p = [], [], []
        for p, (pa, pb, pc) in enumerate(perms):
            m = (pa <= pb) & (pb <= pc)
            pk_idx.append(flat[m])
            pk_g.append(np.array([gidx[(x, y, z)] for x, y, z in zip(pa[m], pb[m], pc[m])], dtype=np.int64))
            pk_p.append(np.full(int(m.sum()), p))
        pk_idx = np.ascontiguousarray(np.concatenate(pk_idx).astype(np.int64))
        pk_g = np.ascontiguousarray(np.concatenate(pk_g).astype(np.int64))
        pk_p = np.ascontiguousarray(np.concatenate(pk_p).astype(np.int64))
        offsets = np.array([0, len(pk_idx)], dtype=np.int64)
        trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
        ci, cj, ck = (np.array([t[m] for t in trip], dtype=np.int64) for m in range(3))
        send = np.zeros(len(trip) * len(pk_idx) * 5)
        t3_ijk = np.ascontiguousarray(t3_ijk, dtype=np.float64)
        self.lib.pack_redistributed_send_buffer_c(len(trip), nvir, 1, _ptr(ci), _ptr(cj), _ptr(ck), _ptr(t3_ijk),
                                                  _ptr(offsets), _ptr(pk_idx), _ptr(pk_g), _ptr(pk_p), _ptr(send))
        out = np.zeros((len(abc_list), nocc, nocc, nocc))
        counts = np.array([send.size], dtype=np.int64)
        displs = np.array([0], dtype=np.int64)
        table = np.arange(len(abc_list), dtype=np.int64)
        self.lib.unpack_received_data_indices(_ptr(send), _ptr(counts), _ptr(displs), _ptr(out), _ptr(table), 1,
                                              nocc, nvir)
        return out


def reference_available():
    return os.path.exists(REF_SO)
