"""RCCSDT(Q) energy on the GPU (distr_cc/rccsdt_q.py:227-1175).

The reference walks tasks (a-block <= b-block <= c-block <= d-block of
`blksize` virtuals, distr_cc/rccsdt_q.py:302-314) and per task builds the
T3-connected z4 (24 einsums, :1014-1071), the T2-connected t4 (12 W_vvvvoo
and 6 W_vvoooo builds with 24 contractions, :390-408, :1073-1129), then the
epilogue (division, P4_444, factor, the two dot products and the
disconnected z4_sq, :1131-1154).

Here the tasks that share (a-block, b-block, c-block) are one group: every
contraction runs once for the whole d range [c0, nvir) of the group, so each
einsum covers all of the group's d-blocks, and the T3 slabs are unpacked on
the device from the ABC-ordered T3 (dcc_fill_t3_from_abc).  The group's z4 and
t4 are stored [i][j][k][l][a][b][c][d] (virtual quadruple fastest), which is
what the group epilogue (dcc_q_group_epilogue) reads with coalesced rows.  The
energies are the sums over the same task set as the reference; only the
summation order differs.

The 132 einsums of a group are data (`group_terms`): (subscripts, operand,
operand, output, alpha) with each operand a named tensor cut by range starts.

precision = "fp64": every einsum in FP64 through torch (cuBLAS), accumulated
into FP64 group blocks.
"bf16x3" / "tf32x3": the einsums of a group run as two grouped split-precision
tcgen05 GEMMs (builds of the W intermediates and z4 first, then t4), each
preceded by one grouped split of its operands; results are added into FP32
group blocks by reductions in L2.  Splits and GEMM tables are planned once
per group shape; a group only supplies new operand addresses.  Denominators,
symmetrization, factors and energies stay FP64.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _c_rccsdt, _c_rccsdt_q, contract
from . import _lib as L

f64 = torch.float64
f32 = torch.float32


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


def default_dchunk(nocc, nvir, blksize, limit=1 << 28):
    """Virtuals per d-chunk of the split path: the largest multiple of blksize whose two FP32
    group blocks (blksize^3 x chunk x nocc^4 each) fit in `limit` bytes, at least blksize and at
    most nvir (one pass over the whole d range).  The grouped GEMMs add into these blocks by
    reductions in L2; blocks of about twice L2 (each phase writes one of the two) keep most
    reductions there.  At nocc=15 / nvir=93 (12 sampled groups) chunks of 4 / 8 / 16 / 40
    virtuals measured 186 / 164 / 170 / 188 ms."""
    per_d = 2 * 4 * blksize ** 3 * nocc ** 4
    return min(nvir, max(blksize, limit // per_d // blksize * blksize))


def job_d_ranges(nvir, blksize, job_idx=0, n_jobs=1):
    """{(a0, a1, b0, b1, c0, c1): (d0, d1)}: the tasks of job `job_idx` of `n_jobs` as group d
    ranges.  A job takes the contiguous slice [j*ceil(T/n), min((j+1)*ceil(T/n), T)) of the
    canonical task order (distr_cc/rccsdt_q.py:359-366); that order runs d-blocks outermost, so
    within one (a, b, c) group a job's d-blocks are consecutive."""
    if n_jobs < 1 or not 0 <= job_idx < n_jobs:
        raise ValueError("job_idx must be in [0, n_jobs)")
    tasks = task_list(nvir, blksize)
    per = (len(tasks) + n_jobs - 1) // n_jobs
    start, end = job_idx * per, min(job_idx * per + per, len(tasks))
    out, nblk = {}, {}
    for t in tasks[start:end]:
        key = (t[0], t[1], t[3], t[4], t[6], t[7])
        d0, d1 = out.get(key, (t[9], t[10]))
        out[key] = (min(d0, t[9]), max(d1, t[10]))
        nblk[key] = nblk.get(key, 0) + 1
    for key, (d0, d1) in out.items():
        if len(prange(d0, d1, blksize)) != nblk[key]:
            raise AssertionError("d-blocks of group %s are not consecutive in job %d" % (key, job_idx))
    return out


# ----------------------------------------------------------------------------
# The einsums of one group as data.  Range letters: A = [a0, a0+ba),
# B = [b0, b0+bb), C = [c0, c0+bc), D = [d0, d0+dn) (d0 = c0, dn = nvir - c0);
# "F" is the full range of the dimension.  Operands are named tensors:
#   integrals vvvo [nv,nv,nv,no], vooo [nv,no,no,no], vvvv [nv]^4,
#   ovvo [no,nv,nv,no], ovov [no,nv,no,nv], oooo [no]^4, t2 [nv,nv,no,no];
#   slabs S<xy> = T[X, Y, :, :, :, :] of the ABC-ordered T3 (x, y in a, b, c, d);
#   intermediates W<xyw> = W_vvvvoo[X, Y, W] (distr_cc/rccsdt_q.py:390-399) and
#   V<xy> = W_vvoooo[X, Y] (:401-408); outputs z (T3-connected), x (T2-connected).
# ----------------------------------------------------------------------------

_Z_TERMS = [
    # (subscripts, (tensor, ranges), (tensor, ranges), alpha)        distr_cc/rccsdt_q.py:1014-1071
    ('cdel,abeijk->abcdijkl', ("vvvo", "CDFF"), ("Sab", "FFFFFF"), 1.0),
    ('dcek,abeijl->abcdijkl', ("vvvo", "DCFF"), ("Sab", "FFFFFF"), 1.0),
    ('dmli,abcmjk->abcdijkl', ("vooo", "DFFF"), ("Sab", "FFCFFF"), -1.0),
    ('dmlj,abcimk->abcdijkl', ("vooo", "DFFF"), ("Sab", "FFCFFF"), -1.0),
    ('cmki,abdmjl->abcdijkl', ("vooo", "CFFF"), ("Sab", "FFDFFF"), -1.0),
    ('cmkj,abdiml->abcdijkl', ("vooo", "CFFF"), ("Sab", "FFDFFF"), -1.0),
    ('bdel,aceikj->abcdijkl', ("vvvo", "BDFF"), ("Sac", "FFFFFF"), 1.0),
    ('dbej,aceikl->abcdijkl', ("vvvo", "DBFF"), ("Sac", "FFFFFF"), 1.0),
    ('bmji,acdmkl->abcdijkl', ("vooo", "BFFF"), ("Sac", "FFDFFF"), -1.0),
    ('bmjk,acdiml->abcdijkl', ("vooo", "BFFF"), ("Sac", "FFDFFF"), -1.0),
    ('dmlk,acbimj->abcdijkl', ("vooo", "DFFF"), ("Sac", "FFBFFF"), -1.0),
    ('bcek,adeilj->abcdijkl', ("vvvo", "BCFF"), ("Sad", "FFFFFF"), 1.0),
    ('cbej,adeilk->abcdijkl', ("vvvo", "CBFF"), ("Sad", "FFFFFF"), 1.0),
    ('bmjl,adcimk->abcdijkl', ("vooo", "BFFF"), ("Sad", "FFCFFF"), -1.0),
    ('cmkl,adbimj->abcdijkl', ("vooo", "CFFF"), ("Sad", "FFBFFF"), -1.0),
    ('adel,bcejki->abcdijkl', ("vvvo", "ADFF"), ("Sbc", "FFFFFF"), 1.0),
    ('daei,bcejkl->abcdijkl', ("vvvo", "DAFF"), ("Sbc", "FFFFFF"), 1.0),
    ('amij,bcdmkl->abcdijkl', ("vooo", "AFFF"), ("Sbc", "FFDFFF"), -1.0),
    ('amik,bcdjml->abcdijkl', ("vooo", "AFFF"), ("Sbc", "FFDFFF"), -1.0),
    ('acek,bdejli->abcdijkl', ("vvvo", "ACFF"), ("Sbd", "FFFFFF"), 1.0),
    ('caei,bdejlk->abcdijkl', ("vvvo", "CAFF"), ("Sbd", "FFFFFF"), 1.0),
    ('amil,bdcjmk->abcdijkl', ("vooo", "AFFF"), ("Sbd", "FFCFFF"), -1.0),
    ('abej,cdekli->abcdijkl', ("vvvo", "ABFF"), ("Scd", "FFFFFF"), 1.0),
    ('baei,cdeklj->abcdijkl', ("vvvo", "BAFF"), ("Scd", "FFFFFF"), 1.0),
]

# W_vvvvoo[X, Y, W] = the six strings of distr_cc/rccsdt_q.py:390-399
_W_BUILD = [
    ('abef,fcjk->abcejk', ("vvvv", "XYFF"), ("t2", "FWFF"), 0.5),
    ('acef,fbkj->abcejk', ("vvvv", "XWFF"), ("t2", "FYFF"), 0.5),
    ('mbej,acmk->abcejk', ("ovvo", "FYFF"), ("t2", "XWFF"), -1.0),
    ('mcek,abmj->abcejk', ("ovvo", "FWFF"), ("t2", "XYFF"), -1.0),
    ('maje,bcmk->abcejk', ("ovov", "FXFF"), ("t2", "YWFF"), -1.0),
    ('make,cbmj->abcejk', ("ovov", "FXFF"), ("t2", "WYFF"), -1.0),
]
# W_vvoooo[X, Y] (distr_cc/rccsdt_q.py:401-408)
_V_BUILD = [
    ('mnki,abnj->abmijk', ("oooo", "FFFF"), ("t2", "XYFF"), -0.5),
    ('mnkj,bani->abmijk', ("oooo", "FFFF"), ("t2", "YXFF"), -0.5),
]
_W_NAMES = ["abc", "abd", "acd", "bac", "bad", "bcd", "cab", "cad", "cbd", "dab", "dac", "dbc"]
_V_NAMES = ["ab", "ac", "ad", "bc", "bd", "cd"]
_X_TERMS = [
    # distr_cc/rccsdt_q.py:1073-1129
    ('abcejk,edil->abcdijkl', "Wabc", ("t2", "FDFF"), 1.0),
    ('abdejl,ecik->abcdijkl', "Wabd", ("t2", "FCFF"), 1.0),
    ('acdekl,ebij->abcdijkl', "Wacd", ("t2", "FBFF"), 1.0),
    ('baceik,edjl->abcdijkl', "Wbac", ("t2", "FDFF"), 1.0),
    ('badeil,ecjk->abcdijkl', "Wbad", ("t2", "FCFF"), 1.0),
    ('bcdekl,eaji->abcdijkl', "Wbcd", ("t2", "FAFF"), 1.0),
    ('cabeij,edkl->abcdijkl', "Wcab", ("t2", "FDFF"), 1.0),
    ('cadeil,ebkj->abcdijkl', "Wcad", ("t2", "FBFF"), 1.0),
    ('cbdejl,eaki->abcdijkl', "Wcbd", ("t2", "FAFF"), 1.0),
    ('dabeij,eclk->abcdijkl', "Wdab", ("t2", "FCFF"), 1.0),
    ('daceik,eblj->abcdijkl', "Wdac", ("t2", "FBFF"), 1.0),
    ('dbcejk,eali->abcdijkl', "Wdbc", ("t2", "FAFF"), 1.0),
    ('abmijk,cdml->abcdijkl', "Vab", ("t2", "CDFF"), -1.0),
    ('abmijl,dcmk->abcdijkl', "Vab", ("t2", "DCFF"), -1.0),
    ('acmikj,bdml->abcdijkl', "Vac", ("t2", "BDFF"), -1.0),
    ('acmikl,dbmj->abcdijkl', "Vac", ("t2", "DBFF"), -1.0),
    ('admilj,bcmk->abcdijkl', "Vad", ("t2", "BCFF"), -1.0),
    ('admilk,cbmj->abcdijkl', "Vad", ("t2", "CBFF"), -1.0),
    ('bcmjki,adml->abcdijkl', "Vbc", ("t2", "ADFF"), -1.0),
    ('bcmjkl,dami->abcdijkl', "Vbc", ("t2", "DAFF"), -1.0),
    ('bdmjli,acmk->abcdijkl', "Vbd", ("t2", "ACFF"), -1.0),
    ('bdmjlk,cami->abcdijkl', "Vbd", ("t2", "CAFF"), -1.0),
    ('cdmkli,abmj->abcdijkl', "Vcd", ("t2", "ABFF"), -1.0),
    ('cdmklj,bami->abcdijkl', "Vcd", ("t2", "BAFF"), -1.0),
]
_SLABS = ["Sab", "Sac", "Sad", "Sbc", "Sbd", "Scd"]


def group_terms():
    """(phase, subscripts, X, Y, output, alpha) of every einsum of a group; X, Y =
    (tensor name, ranges) with one range letter per dimension (F: full; a tensor
    that is an intermediate or output carries its own ranges).  Phase 0: the
    intermediates and z4; phase 1: t4 (reads the intermediates)."""
    out = []
    for w in _W_NAMES:
        sub = dict(X=w[0].upper(), Y=w[1].upper(), W=w[2].upper())
        for s, (xn, xr), (yn, yr), al in _W_BUILD:
            out.append((0, s, (xn, "".join(sub.get(c, c) for c in xr)), (yn, "".join(sub.get(c, c) for c in yr)),
                        "W" + w, al))
    for v in _V_NAMES:
        sub = dict(X=v[0].upper(), Y=v[1].upper())
        for s, (xn, xr), (yn, yr), al in _V_BUILD:
            out.append((0, s, (xn, xr), (yn, "".join(sub.get(c, c) for c in yr)), "V" + v, al))
    for s, X, Y, al in _Z_TERMS:
        out.append((0, s, X, Y, "z", al))
    for s, wn, Y, al in _X_TERMS:
        out.append((1, s, (wn, None), Y, "x", al))
    return out


class _Shapes:
    """Lengths, strides and range starts of every named tensor of a group shape."""

    def __init__(self, no, nv, ba, bb, bc, dn):
        self.no, self.nv = no, nv
        self.len = {"A": ba, "B": bb, "C": bc, "D": dn}
        L_ = self.len
        self.shape = {"vvvo": (nv, nv, nv, no), "vooo": (nv, no, no, no), "vvvv": (nv,) * 4,
                      "ovvo": (no, nv, nv, no), "ovov": (no, nv, no, nv), "oooo": (no,) * 4, "t2": (nv, nv, no, no)}
        for s in _SLABS:
            self.shape[s] = (L_[s[1].upper()], L_[s[2].upper()], nv, no, no, no)
        for w in _W_NAMES:
            self.shape["W" + w] = (L_[w[0].upper()], L_[w[1].upper()], L_[w[2].upper()], nv, no, no)
        for v in _V_NAMES:
            self.shape["V" + v] = (L_[v[0].upper()], L_[v[1].upper()], no, no, no, no)

    def strides(self, name):
        if name in ("z", "x"):
            L_, no = self.len, self.no
            Vv = L_["A"] * L_["B"] * L_["C"] * L_["D"]
            # [i][j][k][l][a][b][c][d]; logical order a b c d i j k l
            return (L_["B"] * L_["C"] * L_["D"], L_["C"] * L_["D"], L_["D"], 1, no ** 3 * Vv, no * no * Vv, no * Vv, Vv)
        sh = self.shape[name]
        st, acc = [], 1
        for n in reversed(sh):
            st.append(acc)
            acc *= n
        return tuple(reversed(st))

    def lengths(self, name, ranges):
        if name in ("z", "x"):
            L_ = self.len
            return (L_["A"], L_["B"], L_["C"], L_["D"]) + (self.no,) * 4
        sh = self.shape[name]
        if ranges is None:
            return sh
        return tuple(sh[i] if r == "F" else self.len[r] for i, r in enumerate(ranges))


def _starts(ranges, origin):
    """Start index per dimension: origin[letter] for a range letter, 0 for F."""
    if ranges is None:
        return None
    return tuple(0 if r == "F" else origin[r] for r in ranges)


_ORIGIN_KEYS = ("A", "B", "C", "D")


def plan_problems(no, nv, sig, terms=None):
    """The einsums of a group shape sig = (ba, bb, bc, dn) as GEMM problems on split
    operands.  Each problem: phase, out (z, x or an intermediate), alpha, m, n, k,
    A / B = {src: tensor name, fm: row map, fk: contraction map, coef: element
    offset of the operand's first element per unit of (a0, b0, c0, d0), off: a
    constant element offset}, the output maps orow / ocol (four-digit maps,
    contract.four order) and the output's constant offset ooff.  Rows come from
    whichever operand wastes less of the 128 x 256 output tiles.  An einsum whose
    free indices do not fold into four digits for both its operand and the output
    runs as one problem per value of one of them (the shortest).
    Also returns [(output name, elements)] of the FP32 outputs."""
    sh = _Shapes(no, nv, *sig)
    probs = []

    def add(phase, subs, xn, xr, yn, yr, on, al, size, sx, sy, so, xoff, yoff, ooff):
        ins, o = subs.split("->")
        xs, ys = ins.split(",")
        K = [c for c in xs if c in ys]
        Mi = [c for c in xs if c not in ys and c in size]
        Ni = [c for c in ys if c not in xs and c in size]
        # enumerate rows and columns in the output's stride order: consecutive rows (or
        # columns) of a tile are then neighbours in the output, so its reductions coalesce
        gM = contract._digit_orders_each(Mi, size, [sx, so], prefer=so)
        gN = contract._digit_orders_each(Ni, size, [sy, so], prefer=so)
        gK = contract._digit_orders_each(K, size, [sx, sy])
        if gK is None:
            raise RuntimeError("einsum %s: contraction does not fold into four-digit maps" % subs)
        if gM is None or gN is None:
            free = Mi if gM is None else Ni
            # the shortest index, but not the one contiguous in the output (kept for coalescing)
            keep_fast = min(free, key=lambda q: so[q])
            c = min([q for q in free if q != keep_fast] or free, key=lambda q: size[q])
            sub = {q: v for q, v in size.items() if q != c}
            for v in range(size[c]):
                add(phase, subs, xn, xr, yn, yr, on, al, sub, sx, sy, so, xoff + v * sx.get(c, 0),
                    yoff + v * sy.get(c, 0), ooff + v * so[c])
            return
        mx, ny = int(np.prod([size[q] for q in Mi])), int(np.prod([size[q] for q in Ni]))
        waste_xy = -(-mx // 128) * 128 * (-(-ny // 256) * 256)
        waste_yx = -(-ny // 128) * 128 * (-(-mx // 256) * 256)

        def operand(name, rng, gR, gk, off):
            coef = np.zeros(4, dtype=np.int64)
            if rng is not None:
                for r_, d_ in zip(rng, sh.strides(name)):
                    if r_ != "F":
                        coef[_ORIGIN_KEYS.index(r_)] += d_
            return {"src": name, "fm": contract._map_of(gR, 0), "fk": contract._map_of(gk, 0), "coef": coef,
                    "off": int(off)}

        opX, opY = operand(xn, xr, gM[0], gK[0], xoff), operand(yn, yr, gN[0], gK[1], yoff)
        pr = {"phase": phase, "subs": subs, "out": on, "alpha": al, "m": mx, "n": ny,
              "k": int(np.prod([size[q] for q in K])), "A": opX, "B": opY,
              "orow": contract._map_of(gM[1], 0), "ocol": contract._map_of(gN[1], 0), "ooff": int(ooff)}
        if waste_yx < waste_xy:  # the other operand takes the rows
            pr.update(m=ny, n=mx, A=opY, B=opX, orow=pr["ocol"], ocol=pr["orow"])
        probs.append(pr)

    for phase, subs, (xn, xr), (yn, yr), on, al in (terms if terms is not None else group_terms()):
        ins, o = subs.split("->")
        xs, ys = ins.split(",")
        lx, ly = sh.lengths(xn, xr), sh.lengths(yn, yr)
        size = {c: n for c, n in zip(xs, lx)}
        size.update({c: n for c, n in zip(ys, ly)})
        sx, sy = dict(zip(xs, sh.strides(xn))), dict(zip(ys, sh.strides(yn)))
        so = dict(zip(o, sh.strides(on)))
        add(phase, subs, xn, xr, yn, yr, on, al, size, sx, sy, so, 0, 0, 0)
    nzx = int(np.prod(sh.lengths("z", None)))
    outs = [("z", nzx), ("x", nzx)] + [(nm, int(np.prod(sh.shape[nm])))
                                         for nm in ["W" + w for w in _W_NAMES] + ["V" + v for v in _V_NAMES]]
    return probs, outs


class QEnergy:
    """[Q] and (Q) energies for fixed (nocc, nvir, blksize) on one GPU.

    eris: dict of device FP64 tensors vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo
    (physicist slices, the reference's eris.pppp cuts); t2 [a,b,i,j] (vvoo order);
    e_occ, e_vir; t3_abc: T3[a<=b<=c][i][j][k] (dcc.rccsdt.redistribute_ijk_to_abc)."""

    def __init__(self, nocc, nvir, blksize=4, precision="fp64", device="cuda", dchunk=None):
        self.no, self.nv, self.blk, self.precision = int(nocc), int(nvir), int(blksize), precision
        # dchunk: the split path may run a group's d range in chunks of this many virtuals.
        # Default: chunks whose two FP32 group blocks (blk^3 x chunk x nocc^4) stay within about
        # 1 GB, which is the whole range up to nocc ~ 12 at nvir ~ 90 (one pass measured fastest
        # at nocc=10: the reductions go through L2 whether or not the blocks fit in it); at
        # nocc=15 / nvir=93 chunks of 24 and 48 measured 7 % and 3 % faster than one pass.
        self.dchunk = int(dchunk) if dchunk else default_dchunk(self.no, self.nv, self.blk)
        self.kind = None if precision == "fp64" else contract.KIND[precision]
        self.dev = torch.device(device)
        self.ws = torch.empty((_c_rccsdt_q.q_group_epilogue_workspace_bytes() + 7) // 8, dtype=f64,
                              device=self.dev)
        self.out = torch.zeros(2, dtype=f64, device=self.dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.terms = group_terms()
        self._plans = {}
        self._arena = self._pool = None
        self._vvooT = self._t2T = None

    def status_ok(self):
        return self.kind is None or int(self.status.item()) == 0

    # ------------------------------------------------------------------ group data
    def _slabs(self, t3_abc, r, which=_SLABS, out=None):
        """T3 slabs of the group / d-chunk r (FP64, filled on the device)."""
        nv, no = self.nv, self.no
        rng = {"a": (r[0], r[1]), "b": (r[2], r[3]), "c": (r[4], r[5]), "d": (r[6], r[7])}
        out = {} if out is None else out
        for s in which:
            (x0, x1), (y0, y1) = rng[s[1]], rng[s[2]]
            t = torch.empty((x1 - x0, y1 - y0, nv, no, no, no), dtype=f64, device=self.dev)
            _c_rccsdt_q.fill_t3_from_abc(t, x0, x1, y0, y1, nv, no, t3_abc, y1 - y0)
            out[s] = t
        return out

    def _chunks(self, d0, d1=None):
        d1 = self.nv if d1 is None else d1
        return [(d0, d1)] if self.kind is None else prange(d0, d1, self.dchunk)

    def _work(self, group_list, d_ranges):
        """(group, d0, d1) to run: every group's tasks (d from the c-block on), or those of
        d_ranges (job_d_ranges) when given."""
        gl = group_list if group_list is not None else groups(self.nv, self.blk)
        if d_ranges is None:
            return [(g, g[4], self.nv) for g in gl]
        return [(g,) + tuple(d_ranges[g]) for g in gl if g in d_ranges]

    def _transposed(self, er, t2):
        if self._vvooT is None:
            self._vvooT = er["vvoo"].permute(0, 2, 3, 1).contiguous()
            self._t2T = t2.permute(0, 2, 3, 1).contiguous()
        return self._vvooT, self._t2T

    # ------------------------------------------------------------------ FP64 path
    def _run_fp64(self, er, t2, slabs, r):
        no, nv = self.no, self.nv
        a0, a1, b0, b1, c0, c1, d0, d1 = r
        sh = _Shapes(no, nv, a1 - a0, b1 - b0, c1 - c0, d1 - d0)
        origin = {"A": a0, "B": b0, "C": c0, "D": d0}
        bufs = dict(er)
        bufs["t2"] = t2
        bufs.update(slabs)
        V = sh.len["A"] * sh.len["B"] * sh.len["C"] * sh.len["D"]
        z = torch.zeros((no,) * 4 + (sh.len["A"], sh.len["B"], sh.len["C"], sh.len["D"]), dtype=f64, device=self.dev)
        x = torch.zeros_like(z)
        outs = {"z": z, "x": x}

        def view(name, ranges):
            t = bufs[name]
            if ranges is None:
                return t
            st = _starts(ranges, origin)
            ln = sh.lengths(name, ranges)
            for dim, (s0, n) in enumerate(zip(st, ln)):
                if s0 != 0 or n != t.shape[dim]:
                    t = t.narrow(dim, s0, n)
            return t

        for phase, subs, (xn, xr), (yn, yr), on, al in self.terms:
            X, Y = view(xn, xr), view(yn, yr)
            ins, o = subs.split("->")
            if on in ("z", "x"):
                res = torch.einsum(ins + "->" + o[4:] + o[:4], X, Y)  # storage order ijkl abcd
                outs[on].add_(res, alpha=al)
            else:
                if on not in bufs:
                    bufs[on] = torch.zeros(sh.shape[on], dtype=f64, device=self.dev)
                bufs[on].add_(torch.einsum(subs, X, Y), alpha=al)
        return z, x

    # ------------------------------------------------------------------ split path
    @staticmethod
    def _need(probs, outs, kind):
        """(split-buffer bytes, FP32 output elements) of a plan, 256-byte aligned pieces."""
        esz = 2 if kind == 0 else 4
        nb = 0
        for pr in probs:
            k8 = (pr["k"] + 7) // 8 * 8
            nb += 2 * ((pr["m"] * k8 * esz + 255) // 256 * 256) + 2 * ((pr["n"] * k8 * esz + 255) // 256 * 256)
        ne = sum((n + 63) // 64 * 64 for _, n in outs)
        return nb, ne

    def _reserve(self, nb, ne):
        """Shared split arena and FP32 output pool of at least nb bytes / ne elements.  All
        group shapes reuse them (groups run in stream order); growing them drops the
        tables that point into the old ones."""
        if self._arena is None or self._arena.numel() < nb or self._pool.numel() < ne:
            self._plans.clear()
            self._arena = self._pool = None
            self._arena = torch.empty(max(nb, 256), dtype=torch.uint8, device=self.dev)
            self._pool = torch.empty(max(ne, 64), dtype=f32, device=self.dev)

    def _plan(self, sig):
        """Device tables of plan_problems(...) for one group shape (ba, bb, bc, dn)."""
        no, nv, kind, dev = self.no, self.nv, self.kind, self.dev
        probs, outs = plan_problems(no, nv, sig)
        nb, ne = self._need(probs, outs, kind)
        if self._arena is None:
            # size the shared buffers for the largest group shape once
            big = plan_problems(no, nv, (min(self.blk, nv),) * 3 + (min(self.dchunk, nv),))
            nb0, ne0 = self._need(*big, kind)
            self._reserve(max(nb, nb0), max(ne, ne0))
        self._reserve(nb, ne)
        dt = torch.bfloat16 if kind == 0 else torch.float32
        cursor = [0]

        def carve(rows, kp):
            n = rows * kp * (2 if kind == 0 else 4)
            v = self._arena.narrow(0, cursor[0], n).view(dt).view(rows, kp)
            cursor[0] += (n + 255) // 256 * 256
            return v

        off, out_t = 0, {}
        for name, n in outs:
            out_t[name] = self._pool.narrow(0, off, n)
            off += (n + 63) // 64 * 64
        phases = [dict(split=[], src=[], gemm=[], alpha=[]) for _ in range(2)]
        for pr in probs:
            # operands keep only their K columns (rounded up to 8): the GEMM's tensor maps
            # end there and read the padding up to the k-block as zeros
            k, kp, k8 = pr["k"], contract.padded_k(pr["k"], kind), (pr["k"] + 7) // 8 * 8
            bufs = {}
            P = phases[pr["phase"]]
            for side, rows in (("A", pr["m"]), ("B", pr["n"])):
                op = pr[side]
                hi, lo = carve(rows, k8), carve(rows, k8)
                bufs[side] = (hi, lo)
                P["split"].append([hi.data_ptr(), lo.data_ptr(), rows, k, k8, k8, 0] +
                                  list(contract.as4(op["fm"])) + list(contract.as4(op["fk"])) +
                                  [1 if op["src"] in out_t else 0])
                P["src"].append((op["src"], op["coef"], op["off"]))
            (ah, al), (bh, bl) = bufs["A"], bufs["B"]
            P["gemm"].append([ah.data_ptr(), al.data_ptr(), k8, bh.data_ptr(), bl.data_ptr(), k8,
                              pr["m"], pr["n"], kp, out_t[pr["out"]].data_ptr() + 4 * pr["ooff"], 1] +
                             list(contract.as4(pr["orow"])) + list(contract.as4(pr["ocol"])))
            P["alpha"].append(pr["alpha"])
        plan = {"zero": self._pool.narrow(0, 0, off), "out": out_t, "phases": []}
        for P in phases:
            plan["phases"].append({
                "split": contract.GroupedSplit(np.asarray(P["split"], dtype=np.int64), kind, dev),
                "gemm": contract.GroupedGemm(np.asarray(P["gemm"], dtype=np.int64),
                                             np.asarray(P["alpha"], dtype=np.float64), kind, dev),
                "src_names": [x[0] for x in P["src"]],
                "src_coef": np.stack([x[1] for x in P["src"]]),
                "src_off": np.array([x[2] for x in P["src"]], dtype=np.int64),
            })
        return plan

    def prepare(self, group_list=None, d_ranges=None):
        """Build the grouped tables of every group shape in group_list (default: all
        groups; d_ranges as in run) ahead of run(), so no planning happens inside a timed
        region."""
        if self.kind is None:
            return
        for (a0, a1, b0, b1, c0, c1), dlo, dhi in self._work(group_list, d_ranges):
            for d0, d1 in self._chunks(dlo, dhi):
                sig = (a1 - a0, b1 - b0, c1 - c0, d1 - d0)
                if sig not in self._plans:
                    self._plans[sig] = self._plan(sig)

    def _run_split(self, er, t2, slabs, r):
        no, nv = self.no, self.nv
        a0, a1, b0, b1, c0, c1, d0, d1 = r
        sig = (a1 - a0, b1 - b0, c1 - c0, d1 - d0)
        plan = self._plans.get(sig)
        if plan is None:
            plan = self._plans[sig] = self._plan(sig)
        plan["zero"].zero_()
        base = dict(er)
        base["t2"] = t2
        base.update(slabs)
        base.update(plan["out"])
        org = np.array([a0, b0, c0, d0], dtype=np.int64)
        for ph in plan["phases"]:
            offs = ph["src_coef"] @ org + ph["src_off"]
            ptrs = [base[nm].data_ptr() + int(o) * base[nm].element_size() for nm, o in zip(ph["src_names"], offs)]
            ph["split"].run(ptrs)
            ph["gemm"].run(self.status)
        return plan["out"]["z"], plan["out"]["x"]

    def run(self, er, t2, t3_abc, e_occ, e_vir, group_list=None, d_ranges=None):
        """Accumulate [Q] and (Q) over the tasks of `group_list` (default: all groups), or,
        with d_ranges ({group: (d0, d1)}, job_d_ranges), over the listed groups' d ranges
        only.  Returns the device tensor [e_bracket, e_paren]."""
        nv, no = self.nv, self.no
        er = {k: v.contiguous() for k, v in er.items()}
        t2 = t2.contiguous()
        vvooT, t2T = self._transposed(er, t2)
        for (a0, a1, b0, b1, c0, c1), dlo, dhi in self._work(group_list, d_ranges):
            slabs = self._slabs(t3_abc, (a0, a1, b0, b1, c0, c1, c0, nv), which=("Sab", "Sac", "Sbc"))
            for d0, d1 in self._chunks(dlo, dhi):
                r = (a0, a1, b0, b1, c0, c1, d0, d1)
                self._slabs(t3_abc, r, which=("Sad", "Sbd", "Scd"), out=slabs)
                if self.kind is None:
                    z, x = self._run_fp64(er, t2, slabs, r)
                else:
                    z, x = self._run_split(er, t2, slabs, r)
                _c_rccsdt_q.q_group_epilogue(x, z, vvooT, t2T, e_occ, e_vir, r, no, nv, self.out, workspace=self.ws)
        return self.out


def q_energy(er, t2, t3_ijk, e_occ, e_vir, nocc, nvir, blksize=4, precision="fp64", group_list=None, job_idx=0,
             n_jobs=1, t3_abc=None):
    """(e_bracket, e_paren) from canonical IJK-ordered T3 on the device (or from T3 already in
    the ABC layout, `t3_abc` [a<=b<=c][i][j][k], as prepare_tamps_for_q leaves it on one rank,
    distr_cc/rccsdt_q.py:82-96; t3_ijk is then unused); with n_jobs > 1, the share of job
    `job_idx` (the energies of all jobs add up to the full ones)."""
    if t3_abc is None:
        t3_abc = _c_rccsdt.redistribute_ijk_to_abc(t3_ijk, nocc, nvir)
    elif tuple(t3_abc.shape) != (nvir * (nvir + 1) * (nvir + 2) // 6, nocc, nocc, nocc):
        raise ValueError("t3_abc must have shape (nvir(nvir+1)(nvir+2)/6, nocc, nocc, nocc)")
    q = QEnergy(nocc, nvir, blksize, precision, device=t3_abc.device)
    d_ranges = None if n_jobs == 1 else job_d_ranges(nvir, blksize, job_idx, n_jobs)
    out = q.run(er, t2, t3_abc, e_occ, e_vir, group_list, d_ranges)
    eb, ep = float(out[0]), float(out[1])
    if not q.status_ok():
        raise RuntimeError("split GEMM reported a timeout")
    return eb, ep
