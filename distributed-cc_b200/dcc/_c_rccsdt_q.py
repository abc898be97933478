"""(Q) helpers on the GPU, mirroring distr_cc/_c_rccsdt_q.py of the reference
(same names and argument meaning, torch CUDA tensors), plus the fused
per-task epilogue that replaces the reference's sequence of t4_add_,
e_abcdijkl_division_, t4_spin_summation_inplace_(P4_444),
t4_multiply_factor_ and the two dot products (distr_cc/rccsdt_q.py:1131-1154)."""
from __future__ import annotations

import torch

from . import _lib as L

f64 = torch.float64


def t4_spin_summation_inplace_(A, nvir4, nocc, pattern, alpha=1.0, beta=0.0):
    """A <- alpha*P(A) + beta*A over nvir4 outer blocks of nocc^4 (src/rccsdt_q.c:33-472)."""
    A = L.as_tensor(A, f64, "A")
    if A.numel() != nvir4 * nocc ** 4:
        raise ValueError("A must hold nvir4 blocks of nocc^4")
    L.call("dcc_t4_spin_summation_inplace", L.ptr(A), nvir4, nocc, L.pattern(pattern), float(alpha), float(beta),
           L.stream_ptr())
    return A


def fill_t3_from_abc(t3_blk_target, a0, a1, b0, b1, nvir, nocc, t3_abc, ld_b):
    """t3_blk[ia,ib,c,i,j,k] from ABC-ordered T3 (src/rccsdt_q.c:655-828; the pointer
    table of fill_t3_from_ptr_array becomes the contiguous ABC array at one rank)."""
    t3_blk_target = L.as_tensor(t3_blk_target, f64, "t3_blk_target")
    t3_abc = L.as_tensor(t3_abc, f64, "t3_abc")
    if t3_blk_target.numel() < (a1 - a0) * ld_b * nvir * nocc ** 3:
        raise ValueError("t3_blk_target too small")
    L.call("dcc_fill_t3_from_abc", L.ptr(t3_blk_target), a0, a1, b0, b1, nvir, nocc, L.ptr(t3_abc), ld_b,
           L.stream_ptr())
    return t3_blk_target


def e_abcdijkl_division_(r4, e_occ, e_vir, a0, a1, b0, b1, c0, c1, d0, d1, blk_a, blk_b, blk_c, blk_d, nocc):
    """r4 /= (e_i+e_j+e_k+e_l - e_a-e_b-e_c-e_d), zero where |D| <= 1e-15 (src/rccsdt_q.c:474-588)."""
    r4 = L.as_tensor(r4, f64, "r4")
    e_occ = L.as_tensor(e_occ, f64, "e_occ")
    e_vir = L.as_tensor(e_vir, f64, "e_vir")
    L.call("dcc_e_abcdijkl_division", L.ptr(r4), L.ptr(e_occ), L.ptr(e_vir), a0, a1, b0, b1, c0, c1, d0, d1,
           blk_a, blk_b, blk_c, blk_d, nocc, L.stream_ptr())
    return r4


def t4_multiply_factor_(t4_blk, factor_blk, blk_a, blk_b, blk_c, blk_d, nocc):
    """t4[abcd] *= factor[abcd], exact zero where factor == 0 (src/rccsdt_q.c:590-650)."""
    t4_blk = L.as_tensor(t4_blk, f64, "t4_blk")
    factor_blk = L.as_tensor(factor_blk, f64, "factor_blk")
    L.call("dcc_t4_multiply_factor", L.ptr(t4_blk), L.ptr(factor_blk), blk_a, blk_b, blk_c, blk_d, nocc,
           L.stream_ptr())
    return t4_blk


def q_task_epilogue(t4, z4, eris_vvoo, t2_vvoo, e_occ, e_vir, task, blksize, nocc, nvir, out, workspace=None):
    """Accumulate one task's [Q] and (Q) contributions into out = [bracket, paren]
    (device float64[2]); t4/z4 are the task's T2- and T3-connected blocks."""
    for t, n in ((t4, "t4"), (z4, "z4"), (eris_vvoo, "eris_vvoo"), (t2_vvoo, "t2_vvoo"), (e_occ, "e_occ"),
                 (e_vir, "e_vir"), (out, "out")):
        L.as_tensor(t, f64, n)
    a0, a1, b0, b1, c0, c1, d0, d1 = task
    need = L.lib().dcc_q_epilogue_workspace_bytes(blksize, nocc)
    if workspace is None:
        workspace = torch.empty((need + 7) // 8, dtype=f64, device=t4.device)
    L.call("dcc_q_task_epilogue", L.ptr(t4), L.ptr(z4), L.ptr(eris_vvoo), L.ptr(t2_vvoo), L.ptr(e_occ),
           L.ptr(e_vir), a0, a1, b0, b1, c0, c1, d0, d1, blksize, nocc, nvir, L.ptr(out), L.ptr(workspace),
           workspace.numel() * 8, L.stream_ptr())
    return out


def q_epilogue_workspace_bytes(blksize, nocc):
    return int(L.lib().dcc_q_epilogue_workspace_bytes(blksize, nocc))


def q_group_epilogue(t4, z4, vvooT, t2T, e_occ, e_vir, ranges, nocc, nvir, out, workspace=None):
    """Accumulate a task group's [Q] and (Q) contributions into out = [bracket, paren]
    (device float64[2]).  t4 / z4: the group's T2- and T3-connected blocks stored
    [i][j][k][l][a][b][c][d] (float64 or float32, same dtype) for the virtual ranges
    (a0, a1, b0, b1, c0, c1, d0, d1); vvooT / t2T: eris_vvoo / t2 as [x][p][q][y]
    (= [x][y][p][q] with the second virtual fastest)."""
    if t4.dtype != z4.dtype or t4.dtype not in (torch.float32, f64):
        raise TypeError("t4 and z4 must both be float64 or both float32")
    for t, n in ((t4, "t4"), (z4, "z4")):
        L.as_tensor(t, t4.dtype, n)
    for t, n in ((vvooT, "vvooT"), (t2T, "t2T"), (e_occ, "e_occ"), (e_vir, "e_vir"), (out, "out")):
        L.as_tensor(t, f64, n)
    a0, a1, b0, b1, c0, c1, d0, d1 = ranges
    V = (a1 - a0) * (b1 - b0) * (c1 - c0) * (d1 - d0)
    if t4.numel() < V * nocc ** 4 or z4.numel() < V * nocc ** 4:
        raise ValueError("t4 / z4 hold fewer than the group's elements")
    if vvooT.numel() != nvir * nvir * nocc * nocc or t2T.numel() != vvooT.numel():
        raise ValueError("vvooT / t2T must be nvir^2 nocc^2")
    need = int(L.lib().dcc_q_group_epilogue_workspace_bytes())
    if workspace is None:
        workspace = torch.empty((need + 7) // 8, dtype=f64, device=t4.device)
    L.call("dcc_q_group_epilogue", L.ptr(t4), L.ptr(z4), int(t4.dtype == torch.float32), L.ptr(vvooT), L.ptr(t2T),
           L.ptr(e_occ), L.ptr(e_vir), a0, a1, b0, b1, c0, c1, d0, d1, nocc, nvir, L.ptr(out), L.ptr(workspace),
           workspace.numel() * 8, L.stream_ptr())
    return out


def q_group_epilogue_workspace_bytes():
    return int(L.lib().dcc_q_group_epilogue_workspace_bytes())
