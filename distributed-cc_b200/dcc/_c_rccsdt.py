"""T3 helpers on the GPU, mirroring distr_cc/_c_rccsdt.py of the reference:
same function names, argument meaning and in-place behaviour, with torch CUDA
tensors in place of numpy arrays.  Every call is asynchronous on the current
torch stream."""
from __future__ import annotations

import numpy as np
import torch

from . import _lib as L

f64, i32, i64 = torch.float64, torch.int32, torch.int64


def t3_single_spin_summation_inplace_(A, nvir, pattern, alpha=1.0, beta=0.0):
    """A <- beta*A + alpha*P(A) on one nvir^3 block (src/rccsdt.c:131-233)."""
    A = L.as_tensor(A, f64, "A")
    if A.numel() != nvir ** 3:
        raise ValueError("A must hold one nvir^3 block")
    L.call("dcc_t3_single_spin_summation_inplace", L.ptr(A), nvir, L.pattern(pattern), float(alpha), float(beta),
           L.stream_ptr())
    return A


def t3_spin_summation_inplace_(A, nblocks, nvir, pattern, alpha=1.0, beta=0.0):
    """Multi-block form used on r3 at distr_cc/rccsdt.py:947."""
    A = L.as_tensor(A, f64, "A")
    if A.numel() != nblocks * nvir ** 3:
        raise ValueError("A must hold nblocks nvir^3 blocks")
    L.call("dcc_t3_spin_summation_inplace", L.ptr(A), nblocks, nvir, L.pattern(pattern), float(alpha),
           float(beta), L.stream_ptr())
    return A


def t3_spin_summation(A, B, nblocks, nvir, pattern, alpha=1.0, beta=0.0, kernel=0):
    """B = beta*A + alpha*P(A) block by block, out of place (PySCF's t3_spin_summation as
    distr_cc/rccsdtq.py:853 calls it); B may be A itself.  kernel: 0 the library's choice, or
    1 strips (P3_201, nvir <= 104), 2 orbit tiles (an error where that kernel does not apply)."""
    A = L.as_tensor(A, f64, "A")
    B = L.as_tensor(B, f64, "B")
    if A.numel() != nblocks * nvir ** 3 or B.numel() != A.numel():
        raise ValueError("A and B must hold nblocks nvir^3 blocks")
    if kernel:
        L.call("dcc_t3_spin_summation_kernel", L.ptr(A), L.ptr(B), nblocks, nvir, L.pattern(pattern), float(alpha),
               float(beta), int(kernel), L.stream_ptr())
    else:
        L.call("dcc_t3_spin_summation", L.ptr(A), L.ptr(B), nblocks, nvir, L.pattern(pattern), float(alpha),
               float(beta), L.stream_ptr())
    return B


def t3_spin_summation_f32(A, B, nblocks, nvir, pattern="P3_201", alpha=1.0, beta=0.0):
    """B = beta*A + alpha*P(A) out of place on FP32 blocks (FP64 arithmetic on the FP32 values,
    the result rounded once); the patterns without a p4 term, nvir <= 104."""
    A = L.as_tensor(A, torch.float32, "A")
    B = L.as_tensor(B, torch.float32, "B")
    if A.numel() != nblocks * nvir ** 3 or B.numel() != A.numel():
        raise ValueError("A and B must hold nblocks nvir^3 blocks")
    L.call("dcc_t3_spin_summation_f32", L.ptr(A), L.ptr(B), nblocks, nvir, L.pattern(pattern), float(alpha),
           float(beta), L.stream_ptr())
    return B


def t3_unpack_p3(t3, U, X, nocc, nvir, pattern="P3_201", alpha=1.0, beta=0.0):
    """U[o] = the canonical T3 unpacked to every ordered (i,j,k) o, and X[o] = beta U[o] +
    alpha P(U[o]), in one pass over the canonical blocks (U may be None: X alone)."""
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = L.as_tensor(t3, f64, "t3")
    X = L.as_tensor(X, f64, "X")
    if t3.numel() != n3 * nvir ** 3 or X.numel() != nocc ** 3 * nvir ** 3:
        raise ValueError("t3 must hold the canonical blocks and X every ordered block")
    if U is not None:
        U = L.as_tensor(U, f64, "U")
        if U.numel() != X.numel():
            raise ValueError("U must hold every ordered block")
    L.call("dcc_t3_unpack_p3", L.ptr(t3), L.ptr(U), L.ptr(X), nocc, nvir, L.pattern(pattern), float(alpha),
           float(beta), L.stream_ptr())
    return U, X


def symmetrize_status():
    """Status word of the bounded waits in the TMA spin-summation kernel on the current
    device (0, or DCC_ERR_TIMEOUT once a wait gave up); reading clears it and
    synchronizes the current stream."""
    import ctypes
    out = ctypes.c_int(0)
    L.call("dcc_t3_symmetrize_status", ctypes.addressof(out), L.stream_ptr())
    return out.value


def t3_orbit_roundtrip_(A, nblocks, nvir):
    """Diagnostic: the spin-summation kernel's tile traffic with no arithmetic (A unchanged)."""
    A = L.as_tensor(A, f64, "A")
    if A.numel() != nblocks * nvir ** 3:
        raise ValueError("A must hold nblocks nvir^3 blocks")
    L.call("dcc_t3_orbit_roundtrip", L.ptr(A), nblocks, nvir, L.stream_ptr())
    return A


def _nblk(A, nvir):
    if A.numel() % max(nvir ** 3, 1):
        raise ValueError("buffer is not a whole number of nvir^3 blocks")
    return A.numel() // max(nvir ** 3, 1)


def t3_transpose_add_(A, B, nvir):
    """B[a,b,c] = A[a,b,c] + A[c,a,b] (src/rccsdt.c:320-375); A may hold several blocks."""
    A = L.as_tensor(A, f64, "A")
    B = L.as_tensor(B, f64, "B")
    if A.shape != B.shape:
        raise ValueError("A and B must have the same shape")
    L.call("dcc_t3_transpose_add", L.ptr(A), L.ptr(B), _nblk(A, nvir), nvir, L.stream_ptr())
    return B


def t3_spin_summation_triple_sym_(A, B0, B1, B2, nvir):
    """B0/B1/B2 spin-summed variants (src/rccsdt.c:245-310); A may hold several blocks."""
    A = L.as_tensor(A, f64, "A")
    B0, B1, B2 = (L.as_tensor(b, f64, n) for b, n in ((B0, "B0"), (B1, "B1"), (B2, "B2")))
    if not (A.shape == B0.shape == B1.shape == B2.shape):
        raise ValueError("A, B0, B1, B2 must have the same shape")
    L.call("dcc_t3_spin_summation_triple_sym", L.ptr(A), L.ptr(B0), L.ptr(B1), L.ptr(B2), _nblk(A, nvir), nvir,
           L.stream_ptr())
    return B0, B1, B2


def fill_local_data_ijk_(t3_local, send_data, requests, ijk_to_local_idx, n_requests, nvir):
    """Gather requested canonical blocks (src/rccsdt.c:105-117)."""
    t3_local = L.as_tensor(t3_local, f64, "t3_local")
    send_data = L.as_tensor(send_data, f64, "send_data")
    requests = L.as_tensor(requests, i32, "requests")
    ijk_to_local_idx = L.as_tensor(ijk_to_local_idx, i64, "ijk_to_local_idx")
    L.call("dcc_fill_local_data_ijk", L.ptr(t3_local), L.ptr(send_data), L.ptr(requests), L.ptr(ijk_to_local_idx),
           n_requests, nvir, L.stream_ptr())
    return send_data


def take_t3_ijk_single_(t3_local, t3_blk, ijk_to_local_idx, i, j, k, nocc, nvir):
    """T3[i,j,k] for any ordering (src/rccsdt.c:119-129).  ijk_to_local_idx is a
    host int64 array.  Raises DccError(DCC_ERR_NOT_LOCAL) where the reference
    silently returns."""
    t3_local = L.as_tensor(t3_local, f64, "t3_local")
    t3_blk = L.as_tensor(t3_blk, f64, "t3_blk")
    m = np.ascontiguousarray(np.asarray(ijk_to_local_idx, dtype=np.int64))
    L.call("dcc_take_t3_ijk_single", L.ptr(t3_local), L.ptr(t3_blk), m.ctypes.data_as(L.c_vp), i, j, k, nocc, nvir,
           L.stream_ptr())
    return t3_blk


def take_t3_batched(t3_local, out, ijk, ijk_to_local_idx, nocc, nvir):
    """out[n] = T3[ijk[n]] for a device list of ordered triples (int32 [n,3])."""
    t3_local = L.as_tensor(t3_local, f64, "t3_local")
    out = L.as_tensor(out, f64, "out")
    ijk = L.as_tensor(ijk, i32, "ijk")
    ijk_to_local_idx = L.as_tensor(ijk_to_local_idx, i64, "ijk_to_local_idx")
    n = ijk.shape[0]
    if out.numel() != n * nvir ** 3:
        raise ValueError("out must hold one nvir^3 block per triple")
    L.call("dcc_take_t3_batched", L.ptr(t3_local), L.ptr(out), L.ptr(ijk), L.ptr(ijk_to_local_idx), n, nocc, nvir,
           L.stream_ptr())
    return out


def r3_tri_divide_e_(r3, eia, ijk):
    """r3[q] /= eia[i,a]+eia[j,b]+eia[k,c] (distr_cc/rccsdt.py:734-744); eia already
    includes -level_shift, ijk is the device list of canonical triples."""
    r3 = L.as_tensor(r3, f64, "r3")
    eia = L.as_tensor(eia, f64, "eia")
    ijk = L.as_tensor(ijk, i32, "ijk")
    L.call("dcc_r3_tri_divide_e", L.ptr(r3), L.ptr(eia), L.ptr(ijk), r3.shape[0], eia.shape[1], L.stream_ptr())
    return r3


def t3_divide_update_(t3, r3, eia, ijk, nvir_active=None, write_r3=True, norms=None, workspace=None):
    """r3 /= D, t3 += r3 and the two squared residual norms in one pass
    (distr_cc/rccsdt.py:949-971).  Returns the device tensor [|r3|^2, |r3_active|^2]."""
    t3 = L.as_tensor(t3, f64, "t3")
    r3 = L.as_tensor(r3, f64, "r3")
    eia = L.as_tensor(eia, f64, "eia")
    ijk = L.as_tensor(ijk, i32, "ijk")
    nblk, nvir = r3.shape[0], eia.shape[1]
    nact = nvir if nvir_active is None else int(nvir_active)
    if norms is None:
        norms = torch.empty(2, dtype=f64, device=r3.device)
    need = L.lib().dcc_t3_update_workspace_bytes(nblk, nvir)
    if workspace is None:
        workspace = torch.empty((need + 7) // 8, dtype=f64, device=r3.device)
    L.call("dcc_t3_divide_update", L.ptr(t3), L.ptr(r3), L.ptr(eia), L.ptr(ijk), nblk, nvir, nact, int(bool(write_r3)),
           L.ptr(norms), L.ptr(workspace), workspace.numel() * 8, L.stream_ptr())
    return norms


def redistribute_ijk_to_abc(t3_ijk, nocc, nvir, out=None):
    """T3[i<=j<=k][abc] -> T3[a<=b<=c][ijk] at one rank
    (distr_cc/distribute_t3.py:1544-1642 with src/rccsdt.c:411-561)."""
    t3_ijk = L.as_tensor(t3_ijk, f64, "t3_ijk")
    nabc = nvir * (nvir + 1) * (nvir + 2) // 6
    if out is None:
        out = torch.empty((nabc, nocc, nocc, nocc), dtype=f64, device=t3_ijk.device)
    L.as_tensor(out, f64, "out")
    L.call("dcc_redistribute_ijk_to_abc", L.ptr(t3_ijk), L.ptr(out), nocc, nvir, L.stream_ptr())
    return out
