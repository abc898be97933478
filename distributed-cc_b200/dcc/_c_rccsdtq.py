"""T4 helpers on the GPU, mirroring distr_cc/_c_rccsdtq.py and the t4_add_ of
distr_cc/_rccsdtq_core.py (same names and argument meaning, torch CUDA tensors)."""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib as L

f64, i32, i64 = torch.float64, torch.int32, torch.int64


def t4_project_1_minus_p4_p31_inplace_(A, nocc4, nvir, alpha=1.0, beta=0.0):
    """A <- beta*A + alpha*(1 - P[4] - P[3,1])A (src/rccsdtq.c:262-308)."""
    A = L.as_tensor(A, f64, "A")
    if A.numel() != nocc4 * nvir ** 4:
        raise ValueError("A must hold nocc4 blocks of nvir^4")
    L.call("dcc_t4_project_1_minus_p4_p31_inplace", L.ptr(A), nocc4, nvir, float(alpha), float(beta),
           L.stream_ptr())
    return A


def t4_single_spin_summation_inplace_(A, nvir, pattern, alpha=1.0, beta=0.0):
    """P4_full | P4_442 | P4_201 on one nvir^4 block (src/rccsdtq.c:316-916)."""
    A = L.as_tensor(A, f64, "A")
    if A.numel() != nvir ** 4:
        raise ValueError("A must hold one nvir^4 block")
    if pattern not in ("P4_full", "P4_442", "P4_201"):
        raise ValueError('unrecognized pattern "%s"' % pattern)
    L.call("dcc_t4_spin_summation_inplace", L.ptr(A), 1, nvir, L.pattern(pattern), float(alpha), float(beta),
           L.stream_ptr())
    return A


def t4_transpose_add_(src, dst, nvir):
    """dst = src + src[c,a,b,d] + src[d,a,c,b] (src/rccsdtq.c:990-1005)."""
    src = L.as_tensor(src, f64, "src")
    dst = L.as_tensor(dst, f64, "dst")
    if tuple(src.shape) != (nvir,) * 4 or tuple(dst.shape) != (nvir,) * 4:
        raise ValueError("src and dst must have shape (nvir, nvir, nvir, nvir)")
    L.call("dcc_t4_transpose_add", L.ptr(src), L.ptr(dst), nvir, L.stream_ptr())
    return dst


def t4_spin_summation_quadruple_sym_(src, B0, B1, B2, B3, nvir):
    """The four P4_201 variants (src/rccsdtq.c:1018-1047)."""
    bufs = [L.as_tensor(b, f64, n) for b, n in ((src, "src"), (B0, "B0"), (B1, "B1"), (B2, "B2"), (B3, "B3"))]
    if any(tuple(b.shape) != (nvir,) * 4 for b in bufs):
        raise ValueError("all T4 buffers must have shape (nvir, nvir, nvir, nvir)")
    L.call("dcc_t4_spin_summation_quadruple_sym", *[L.ptr(b) for b in bufs], nvir, L.stream_ptr())
    return B0, B1, B2, B3


def t4_forms_batched(t4, nvir, T3=None, V=None):
    """The transpose-add and the four quadruple-symmetrized forms of every block of t4
    [n, nvir^4] in two launches (the forms the OO batch of compute_r4_tri takes per source
    block, distr_cc/rccsdtq.py:1168-1169).  Returns (T3, [V0, V1, V2, V3])."""
    t4 = L.as_tensor(t4, f64, "t4")
    n = t4.shape[0]
    if t4.numel() != n * nvir ** 4:
        raise ValueError("t4 must hold n nvir^4 blocks")
    T3 = torch.empty_like(t4) if T3 is None else L.as_tensor(T3, f64, "T3")
    V = [torch.empty_like(t4) for _ in range(4)] if V is None else [L.as_tensor(v, f64, "V") for v in V]
    if any(x.numel() != t4.numel() for x in [T3] + V):
        raise ValueError("T3 and V must have t4's size")
    L.call("dcc_t4_transpose_add_batched", L.ptr(t4), L.ptr(T3), n, nvir, L.stream_ptr())
    L.call("dcc_t4_spin_summation_quadruple_sym_batched", L.ptr(t4), *[L.ptr(v) for v in V], n, nvir,
           L.stream_ptr())
    return T3, V


def r4_local_tri_divide(r4_local, eia, local_ijkl):
    """r4[q] /= eia[i,a]+eia[j,b]+eia[k,c]+eia[l,d] (src/rccsdtq.c:1055-1088)."""
    r4_local = L.as_tensor(r4_local, f64, "r4_local")
    eia = L.as_tensor(eia, f64, "eia")
    local_ijkl = L.as_tensor(local_ijkl, i32, "local_ijkl")
    nvir = eia.shape[1]
    if r4_local.shape != (local_ijkl.shape[0],) + (nvir,) * 4:
        raise ValueError("r4_local has inconsistent local T4 shape")
    L.call("dcc_r4_local_tri_divide_e", L.ptr(r4_local), L.ptr(eia), L.ptr(local_ijkl), local_ijkl.shape[0], nvir,
           L.stream_ptr())
    return r4_local


def r4_local_tri_divide_e_(mycc, dt4, r4_local, mo_energy):
    """Reference-shaped wrapper (distr_cc/_c_rccsdtq.py:63-74)."""
    nocc = mycc.nocc
    mo = torch.as_tensor(np.asarray(mo_energy), dtype=f64, device=r4_local.device)
    eia = (mo[:nocc, None] - mo[None, nocc:] - mycc.level_shift).contiguous()
    ijkl = torch.as_tensor(np.asarray(dt4.local_quadruples, dtype=np.int32).reshape(-1, 4), device=r4_local.device)
    return r4_local_tri_divide(r4_local, eia, ijkl)


def fill_local_data_ijkl_(t4_local, send_data, requests, ijkl_to_local_idx, n_requests, nvir):
    """Gather requested T4 blocks (src/rccsdtq.c:1090-1102)."""
    t4_local = L.as_tensor(t4_local, f64, "t4_local")
    send_data = L.as_tensor(send_data, f64, "send_data")
    requests = L.as_tensor(requests, i32, "requests")
    ijkl_to_local_idx = L.as_tensor(ijkl_to_local_idx, i64, "ijkl_to_local_idx")
    L.call("dcc_fill_local_data_ijkl", L.ptr(t4_local), L.ptr(send_data), L.ptr(requests),
           L.ptr(ijkl_to_local_idx), n_requests, nvir, L.stream_ptr())
    return send_data


def unpack_t4_ijkl_single_(t4_local, t4_blk, ijkl_to_local_idx, i, j, k, l, nocc, nvir):
    """T4[i,j,k,l] for any ordering; zero-rule blocks come back zero
    (src/rccsdtq.c:1104-1125).  ijkl_to_local_idx is a host int64 array."""
    t4_local = L.as_tensor(t4_local, f64, "t4_local")
    t4_blk = L.as_tensor(t4_blk, f64, "t4_blk")
    m = np.ascontiguousarray(np.asarray(ijkl_to_local_idx, dtype=np.int64))
    L.call("dcc_unpack_t4_ijkl_single", L.ptr(t4_local), L.ptr(t4_blk), m.ctypes.data_as(L.c_vp), i, j, k, l, nocc,
           nvir, L.stream_ptr())
    return t4_blk


def t4_add_(t4, r4, nocc4, nvir):
    """t4 += r4 over nocc4 blocks of nvir^4 (PySCF libccsdt t4_add_, distr_cc/_rccsdtq_core.py:43-48)."""
    t4 = L.as_tensor(t4, f64, "t4")
    r4 = L.as_tensor(r4, f64, "r4")
    n = nocc4 * nvir ** 4
    if t4.numel() < n or r4.numel() < n:
        raise ValueError("t4/r4 smaller than nocc4 * nvir^4")
    L.call("dcc_t4_add", L.ptr(t4), L.ptr(r4), n, L.stream_ptr())
    return t4


def t4_strings(ops, desc, quads, nocc, nvir, r4, beta=0.0, status=None, pairs=None):
    """r4 = beta r4 + every string of the descriptor table `desc` [nstr, 32] (int64, device)
    over every stored block of `quads` [nq, 4] (int32, device), one launch (the per-block
    strings of compute_r4_tri and its OO batch, distr_cc/rccsdtq.py:862-1349).  ops: the
    operand tensors the descriptors index (contiguous FP64, device).  pairs: None, or
    (pair_off [nq, ngroups+1], pair_sm [npairs, 2]) int32 device tensors for the pair-mode
    strings.  status: int32 device word, bits set by the kernel's checks (a new zero word
    when None).  Returns status."""
    n = len(ops)
    ops = [L.as_tensor(t, f64, "operand") for t in ops]
    desc = L.as_tensor(desc, torch.int64, "desc")
    quads = L.as_tensor(quads, torch.int32, "quads")
    r4 = L.as_tensor(r4, f64, "r4")
    if desc.dim() != 2 or desc.shape[1] != 32:
        raise ValueError("desc must be [nstr, 32]")
    nq = quads.shape[0]
    if quads.shape != (nq, 4) or r4.numel() != nq * nvir ** 4:
        raise ValueError("quads must be [nq, 4] and r4 [nq, nvir^4]")
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=r4.device)
    if pairs is None:
        off = sm = None
        ngroups = npairs = 0
    else:
        off = L.as_tensor(pairs[0], torch.int32, "pair_off")
        sm = L.as_tensor(pairs[1], torch.int32, "pair_sm")
        ngroups, npairs = off.shape[1] - 1, sm.shape[0]
        if off.shape[0] != nq or sm.dim() != 2 or sm.shape[1] != 2:
            raise ValueError("pair_off must be [nq, ngroups+1] and pair_sm [npairs, 2]")
    ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in ops])
    numel = (ctypes.c_int64 * n)(*[t.numel() for t in ops])
    L.call("dcc_t4_strings", ptrs, numel, n, L.ptr(desc), desc.shape[0], L.ptr(quads), nq, L.ptr(off), L.ptr(sm),
           ngroups, npairs, nocc, nvir, float(beta), L.ptr(r4), L.ptr(status), L.stream_ptr())
    return status


def t4_strings_rows_per_cta(nq, nvir):
    """Output rows a that one CTA of t4_strings holds (-1 when nvir^3 doubles exceed its
    shared-memory accumulator)."""
    return int(L.lib().dcc_t4_strings_rows_per_cta(int(nq), int(nvir)))
