"""RCCSDT(Q) energy on the GPU (distr_cc/rccsdt_q.py:227-1175).

The reference walks tasks (a-block <= b-block <= c-block <= d-block of
`blksize` virtuals, distr_cc/rccsdt_q.py:302-314) and per task builds the
T3-connected z4 (24 einsums, :1014-1071), the T2-connected t4 (12 W_vvvvoo
and 6 W_vvoooo builds with 24 contractions, :390-408, :1073-1129), then the
epilogue (division, P4_444, factor, the two dot products and the
disconnected z4_sq, :1131-1154).

Here the tasks that share (a-block, b-block, c-block) are one group: every
contraction runs once for the whole d range [c0, nvir) of the group, so each
einsum is a GEMM over all of the group's d-blocks instead of one per task,
and the T3 slabs are unpacked on the device from the ABC-ordered T3
(dcc_fill_t3_from_abc).  Each task's epilogue is the fused
dcc_q_task_epilogue kernel.  The energies are the sums over the same task
set as the reference; only the summation order of the contractions differs.

precision = "fp64": every contraction in FP64 (cuBLAS through torch).
"bf16x3" / "tf32x3": every contraction is one split-precision tcgen05 GEMM
that reads its operands in place and accumulates into the group tensor
through its epilogue maps (contract.einsum_into); denominators,
symmetrization, factors and energies stay FP64.
"""
from __future__ import annotations

import torch

from . import _c_rccsdt, _c_rccsdt_q, contract

f64 = torch.float64


def prange(start, stop, step):
    return [(i, min(i + step, stop)) for i in range(start, stop, step)]


def task_list(nvir, blksize):
    """The reference's canonical task order (distr_cc/rccsdt_q.py:302-314)."""
    tasks = []
    for d0, d1 in prange(0, nvir, blksize):
        for c0, c1 in prange(0, d1, blksize):
            for b0, b1 in prange(0, c1, blksize):
                for a0, a1 in prange(0, b1, blksize):
                    tasks.append((a0, a1, a1 - a0, b0, b1, b1 - b0, c0, c1, c1 - c0, d0, d1, d1 - d0))
    return tasks


def groups(nvir, blksize):
    """(a0, a1, b0, b1, c0, c1) of every (a-block <= b-block <= c-block) group; the group's
    tasks are the d-blocks d0 >= c0."""
    out = []
    for c0, c1 in prange(0, nvir, blksize):
        for b0, b1 in prange(0, c1, blksize):
            for a0, a1 in prange(0, b1, blksize):
                out.append((a0, a1, b0, b1, c0, c1))
    return out


class QEnergy:
    """[Q] and (Q) energies for fixed (nocc, nvir, blksize) on one GPU.

    eris: dict of device FP64 tensors vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo
    (physicist slices, the reference's eris.pppp cuts); t2 [a,b,i,j] (vvoo order);
    e_occ, e_vir; t3_abc: T3[a<=b<=c][i][j][k] (dcc.rccsdt.redistribute_ijk_to_abc)."""

    def __init__(self, nocc, nvir, blksize=4, precision="fp64", device="cuda"):
        self.no, self.nv, self.blk, self.precision = int(nocc), int(nvir), int(blksize), precision
        self.kind = None if precision == "fp64" else contract.KIND[precision]
        self.dev = device
        blk, no = self.blk, self.no
        self.t4_task = torch.zeros((blk,) * 4 + (no,) * 4, dtype=f64, device=device)
        self.z4_task = torch.zeros_like(self.t4_task)
        self.ws = torch.empty((_c_rccsdt_q.q_epilogue_workspace_bytes(blk, no) + 7) // 8, dtype=f64, device=device)
        self.out = torch.zeros(2, dtype=f64, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)

    def E(self, subs, X, Y, out, alpha=1.0, beta=1.0):
        """out = alpha * einsum(subs, X, Y) + beta * out: one split GEMM accumulating in place
        (contract.einsum_into), or FP64 torch for precision="fp64"."""
        return contract.einsum_into(subs, X, Y, out, alpha, beta, self.kind, self.status)

    def status_ok(self):
        return self.kind is None or int(self.status.item()) == 0

    def slab(self, t3_abc, a0, a1, b0, b1):
        """T[a0:a1, b0:b1, :, :, :, :] from the ABC-ordered T3."""
        nv, no = self.nv, self.no
        out = torch.empty((a1 - a0, b1 - b0, nv, no, no, no), dtype=f64, device=self.dev)
        _c_rccsdt_q.fill_t3_from_abc(out, a0, a1, b0, b1, nv, no, t3_abc, b1 - b0)
        return out

    def W_vvvvoo(self, er, t2, a0, a1, b0, b1, c0, c1):
        """distr_cc/rccsdt_q.py:390-399 for the index ranges given."""
        E, no, nv = self.E, self.no, self.nv
        W = torch.empty((a1 - a0, b1 - b0, c1 - c0, nv, no, no), dtype=f64, device=self.dev)
        E('abef,fcjk->abcejk', er["vvvv"][a0:a1, b0:b1], t2[:, c0:c1], W, 0.5, 0.0)
        E('acef,fbkj->abcejk', er["vvvv"][a0:a1, c0:c1], t2[:, b0:b1], W, 0.5)
        E('mbej,acmk->abcejk', er["ovvo"][:, b0:b1], t2[a0:a1, c0:c1], W, -1.0)
        E('mcek,abmj->abcejk', er["ovvo"][:, c0:c1], t2[a0:a1, b0:b1], W, -1.0)
        E('maje,bcmk->abcejk', er["ovov"][:, a0:a1], t2[b0:b1, c0:c1], W, -1.0)
        E('make,cbmj->abcejk', er["ovov"][:, a0:a1], t2[c0:c1, b0:b1], W, -1.0)
        return W

    def W_vvoooo(self, er, t2, a0, a1, b0, b1):
        """distr_cc/rccsdt_q.py:401-408."""
        no = self.no
        W = torch.empty((a1 - a0, b1 - b0) + (no,) * 4, dtype=f64, device=self.dev)
        self.E('mnki,abnj->abmijk', er["oooo"], t2[a0:a1, b0:b1], W, -0.5, 0.0)
        self.E('mnkj,bani->abmijk', er["oooo"], t2[b0:b1, a0:a1], W, -0.5)
        return W

    def group(self, er, t2, t3_abc, a0, a1, b0, b1, c0, c1):
        """z4 and t4 [a, b, c, d, i, j, k, l] of a group, d over [c0, nvir)."""
        E, nv, no = self.E, self.nv, self.no
        A, B, C, D = slice(a0, a1), slice(b0, b1), slice(c0, c1), slice(c0, nv)
        vvvo, vooo = er["vvvo"], er["vooo"]
        shape = (a1 - a0, b1 - b0, c1 - c0, nv - c0) + (no,) * 4
        z = torch.empty(shape, dtype=f64, device=self.dev)
        x = torch.empty(shape, dtype=f64, device=self.dev)
        # T3-connected (distr_cc/rccsdt_q.py:1014-1071)
        t = self.slab(t3_abc, a0, a1, b0, b1)
        E('cdel,abeijk->abcdijkl', vvvo[C, D], t, z, 1.0, 0.0)
        E('dcek,abeijl->abcdijkl', vvvo[D, C], t, z)
        E('dmli,abcmjk->abcdijkl', vooo[D], t[:, :, C], z, -1.0)
        E('dmlj,abcimk->abcdijkl', vooo[D], t[:, :, C], z, -1.0)
        E('cmki,abdmjl->abcdijkl', vooo[C], t[:, :, D], z, -1.0)
        E('cmkj,abdiml->abcdijkl', vooo[C], t[:, :, D], z, -1.0)
        t = self.slab(t3_abc, a0, a1, c0, c1)
        E('bdel,aceikj->abcdijkl', vvvo[B, D], t, z)
        E('dbej,aceikl->abcdijkl', vvvo[D, B], t, z)
        E('bmji,acdmkl->abcdijkl', vooo[B], t[:, :, D], z, -1.0)
        E('bmjk,acdiml->abcdijkl', vooo[B], t[:, :, D], z, -1.0)
        E('dmlk,acbimj->abcdijkl', vooo[D], t[:, :, B], z, -1.0)
        t = self.slab(t3_abc, a0, a1, c0, nv)
        E('bcek,adeilj->abcdijkl', vvvo[B, C], t, z)
        E('cbej,adeilk->abcdijkl', vvvo[C, B], t, z)
        E('bmjl,adcimk->abcdijkl', vooo[B], t[:, :, C], z, -1.0)
        E('cmkl,adbimj->abcdijkl', vooo[C], t[:, :, B], z, -1.0)
        t = self.slab(t3_abc, b0, b1, c0, c1)
        E('adel,bcejki->abcdijkl', vvvo[A, D], t, z)
        E('daei,bcejkl->abcdijkl', vvvo[D, A], t, z)
        E('amij,bcdmkl->abcdijkl', vooo[A], t[:, :, D], z, -1.0)
        E('amik,bcdjml->abcdijkl', vooo[A], t[:, :, D], z, -1.0)
        t = self.slab(t3_abc, b0, b1, c0, nv)
        E('acek,bdejli->abcdijkl', vvvo[A, C], t, z)
        E('caei,bdejlk->abcdijkl', vvvo[C, A], t, z)
        E('amil,bdcjmk->abcdijkl', vooo[A], t[:, :, C], z, -1.0)
        t = self.slab(t3_abc, c0, c1, c0, nv)
        E('abej,cdekli->abcdijkl', vvvo[A, B], t, z)
        E('baei,cdeklj->abcdijkl', vvvo[B, A], t, z)
        del t
        # T2-connected (distr_cc/rccsdt_q.py:1073-1129)
        W = self.W_vvvvoo
        d0, d1 = c0, nv
        E('abcejk,edil->abcdijkl', W(er, t2, a0, a1, b0, b1, c0, c1), t2[:, D], x, 1.0, 0.0)
        E('abdejl,ecik->abcdijkl', W(er, t2, a0, a1, b0, b1, d0, d1), t2[:, C], x)
        E('acdekl,ebij->abcdijkl', W(er, t2, a0, a1, c0, c1, d0, d1), t2[:, B], x)
        E('baceik,edjl->abcdijkl', W(er, t2, b0, b1, a0, a1, c0, c1), t2[:, D], x)
        E('badeil,ecjk->abcdijkl', W(er, t2, b0, b1, a0, a1, d0, d1), t2[:, C], x)
        E('bcdekl,eaji->abcdijkl', W(er, t2, b0, b1, c0, c1, d0, d1), t2[:, A], x)
        E('cabeij,edkl->abcdijkl', W(er, t2, c0, c1, a0, a1, b0, b1), t2[:, D], x)
        E('cadeil,ebkj->abcdijkl', W(er, t2, c0, c1, a0, a1, d0, d1), t2[:, B], x)
        E('cbdejl,eaki->abcdijkl', W(er, t2, c0, c1, b0, b1, d0, d1), t2[:, A], x)
        E('dabeij,eclk->abcdijkl', W(er, t2, d0, d1, a0, a1, b0, b1), t2[:, C], x)
        E('daceik,eblj->abcdijkl', W(er, t2, d0, d1, a0, a1, c0, c1), t2[:, B], x)
        E('dbcejk,eali->abcdijkl', W(er, t2, d0, d1, b0, b1, c0, c1), t2[:, A], x)
        V = self.W_vvoooo
        Wv = V(er, t2, a0, a1, b0, b1)
        E('abmijk,cdml->abcdijkl', Wv, t2[C, D], x, -1.0)
        E('abmijl,dcmk->abcdijkl', Wv, t2[D, C], x, -1.0)
        Wv = V(er, t2, a0, a1, c0, c1)
        E('acmikj,bdml->abcdijkl', Wv, t2[B, D], x, -1.0)
        E('acmikl,dbmj->abcdijkl', Wv, t2[D, B], x, -1.0)
        Wv = V(er, t2, a0, a1, d0, d1)
        E('admilj,bcmk->abcdijkl', Wv, t2[B, C], x, -1.0)
        E('admilk,cbmj->abcdijkl', Wv, t2[C, B], x, -1.0)
        Wv = V(er, t2, b0, b1, c0, c1)
        E('bcmjki,adml->abcdijkl', Wv, t2[A, D], x, -1.0)
        E('bcmjkl,dami->abcdijkl', Wv, t2[D, A], x, -1.0)
        Wv = V(er, t2, b0, b1, d0, d1)
        E('bdmjli,acmk->abcdijkl', Wv, t2[A, C], x, -1.0)
        E('bdmjlk,cami->abcdijkl', Wv, t2[C, A], x, -1.0)
        Wv = V(er, t2, c0, c1, d0, d1)
        E('cdmkli,abmj->abcdijkl', Wv, t2[A, B], x, -1.0)
        E('cdmklj,bami->abcdijkl', Wv, t2[B, A], x, -1.0)
        return z, x

    def run(self, er, t2, t3_abc, e_occ, e_vir, group_list=None):
        """Accumulate [Q] and (Q) over the tasks of `group_list` (default: all groups).
        Returns the device tensor [e_bracket, e_paren]."""
        blk, nv = self.blk, self.nv
        for (a0, a1, b0, b1, c0, c1) in (group_list if group_list is not None else groups(nv, blk)):
            z, x = self.group(er, t2, t3_abc, a0, a1, b0, b1, c0, c1)
            ba, bb, bc = a1 - a0, b1 - b0, c1 - c0
            for d0, d1 in prange(c0, nv, blk):
                bd = d1 - d0
                self.z4_task[:ba, :bb, :bc, :bd].copy_(z[:, :, :, d0 - c0:d1 - c0])
                self.t4_task[:ba, :bb, :bc, :bd].copy_(x[:, :, :, d0 - c0:d1 - c0])
                _c_rccsdt_q.q_task_epilogue(self.t4_task, self.z4_task, er["vvoo"], t2, e_occ, e_vir,
                                            (a0, a1, b0, b1, c0, c1, d0, d1), blk, self.no, nv, self.out,
                                            workspace=self.ws)
        return self.out


def q_energy(er, t2, t3_ijk, e_occ, e_vir, nocc, nvir, blksize=4, precision="fp64", group_list=None):
    """(e_bracket, e_paren) from canonical IJK-ordered T3 on the device."""
    t3_abc = _c_rccsdt.redistribute_ijk_to_abc(t3_ijk, nocc, nvir)
    q = QEnergy(nocc, nvir, blksize, precision, device=t3_ijk.device)
    out = q.run(er, t2, t3_abc, e_occ, e_vir, group_list)
    eb, ep = float(out[0]), float(out[1])
    if not q.status_ok():
        raise RuntimeError("split GEMM reported a timeout")
    return eb, ep
