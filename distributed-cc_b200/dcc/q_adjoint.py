"""Hand-written adjoint (VJP) of the (Q) energies behind torch.autograd.Function.

Forward: (e_bracket, e_paren) = rccsdt_q.q_energy(integrals, t2, canonical t3)
(distr_cc/rccsdt_q.py:227-1175, the task loop of :976-1160).  For cotangents
(g_b, g_p) the backward returns the gradients of g_b [Q] + g_p (Q) with respect
to t2, t3 and the seven integral slices (vvvo, vooo, vvoo, ovvo, ovov, vvvv,
oooo); the orbital energies are not differentiated.

Per task group (the tasks sharing a-, b- and c-blocks, d over [c0, nvir)):

  1. recompute the group's blocks instead of storing them: the T3 slabs
     T[X, Y, :, i, j, k] from U = unpack(t3), the W_vvvvoo / W_vvoooo
     intermediates, z4 and t4 (the einsum table rccsdt_q.group_terms, FP64);
  2. dcc_q_group_epilogue_adjoint: with X = (t4 + z4) / D and Y = f P4_444(X),
       dX = P4_444^T(f (g_p z4 + (g_b + g_p) z4sq) / 12),
       g t4 = dX / D,  g z4 = dX / D + g_p Y / 12,  g z4sq = (g_b + g_p) Y / 12;
  3. back through every einsum of the table in reverse order (t4 strings, then
     the z4 strings and the intermediates' builds): for out += alpha X.Y,
     gX += alpha gout.Y and gY += alpha X.gout over the operand's range, and
     through the six disconnected vvoo x t2 products of z4sq (:1143-1150);
  4. the slab gradients go back into the full T3, and unpack^T takes them to
     the canonical blocks.

Gradients with respect to t3 are returned projected onto blocks symmetric under
their stabilizer (i = j, j = k), the subspace canonical T3 lives in.  Every
contraction of the backward is FP64 (torch / cuBLAS).
"""
from __future__ import annotations

import torch

from . import _lib as L
from . import _c_rccsdt, rccsdt_q, t3_residual
from .adjoint import _stab_masks
from .synthetic import canonical_ijk

f64 = torch.float64

ER_NAMES = ("vvvo", "vooo", "vvoo", "ovvo", "ovov", "vvvv", "oooo")

# the disconnected z4sq = sum of vvoo[x, y, p, q] t2[z, w, r, s] (distr_cc/rccsdt_q.py:1143-1150),
# as (vvoo indices, t2 indices) over the output 'abcdijkl'
_ZSQ = [("abij", "cdkl"), ("acik", "bdjl"), ("adil", "bcjk"), ("bcjk", "adil"), ("bdjl", "acik"), ("cdkl", "abij")]


def _epilogue_adjoint(x, z, vvooT, t2T, e_occ, e_vir, r, nocc, nvir, g_b, g_p):
    gx, gz, gzsq = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    for t, n in ((x, "t4"), (z, "z4"), (vvooT, "vvooT"), (t2T, "t2T"), (e_occ, "e_occ"), (e_vir, "e_vir")):
        L.as_tensor(t, f64, n)
    a0, a1, b0, b1, c0, c1, d0, d1 = r
    L.call("dcc_q_group_epilogue_adjoint", L.ptr(x), L.ptr(z), L.ptr(vvooT), L.ptr(t2T), L.ptr(e_occ), L.ptr(e_vir),
           a0, a1, b0, b1, c0, c1, d0, d1, nocc, nvir, L.c_dbl(g_b), L.c_dbl(g_p), L.ptr(gx), L.ptr(gz), L.ptr(gzsq),
           L.stream_ptr())
    return gx, gz, gzsq


L.bind("dcc_q_group_epilogue_adjoint", [L.c_vp] * 6 + [L.c_i64] * 10 + [L.c_dbl, L.c_dbl] + [L.c_vp] * 4)


def q_energy_vjp(g, er, t2, t3, e_occ, e_vir, nocc, nvir, blksize=4):
    """Gradients of g[0] [Q] + g[1] (Q) with respect to (t2, t3, {integral name: tensor}).

    er: dict of the seven FP64 integral slices; t2 [a,b,i,j] (vvoo order); t3 the
    canonical IJK-ordered blocks [n3][nvir]^3; all on one CUDA device."""
    g_b, g_p = float(g[0]), float(g[1])
    dev = t3.device
    er = {k: er[k].contiguous() for k in ER_NAMES}
    t2 = t2.contiguous()
    no, nv = int(nocc), int(nvir)
    q = rccsdt_q.QEnergy(no, nv, blksize, "fp64", device=dev)
    vvooT, t2T = q._transposed(er, t2)
    U = torch.empty((no,) * 3 + (nv,) * 3, dtype=f64, device=dev)
    t3_residual.unpack_all_(t3.contiguous(), U.view(no ** 3, nv, nv, nv), no, nv)
    T = U.permute(3, 4, 5, 0, 1, 2)  # T[a,b,c,i,j,k]
    gU = torch.zeros_like(U)
    gT = gU.permute(3, 4, 5, 0, 1, 2)
    ger = {k: torch.zeros_like(v) for k, v in er.items()}
    gt2 = torch.zeros_like(t2)
    terms = q.terms
    for (a0, a1, b0, b1, c0, c1) in rccsdt_q.groups(nv, blksize):
        r = (a0, a1, b0, b1, c0, c1, c0, nv)
        rng = {"a": (a0, a1), "b": (b0, b1), "c": (c0, c1), "d": (c0, nv)}
        sh = rccsdt_q._Shapes(no, nv, a1 - a0, b1 - b0, c1 - c0, nv - c0)
        origin = {"A": a0, "B": b0, "C": c0, "D": c0}
        bufs, gbufs = dict(er), dict(ger)
        bufs["t2"], gbufs["t2"] = t2, gt2
        for s in rccsdt_q._SLABS:
            (x0, x1), (y0, y1) = rng[s[1]], rng[s[2]]
            bufs[s] = T[x0:x1, y0:y1].contiguous()
            gbufs[s] = torch.zeros_like(bufs[s])
        # 1. recompute z4, t4 and the intermediates (FP64)
        grp = (no,) * 4 + (sh.len["A"], sh.len["B"], sh.len["C"], sh.len["D"])
        bufs["z"], bufs["x"] = torch.zeros(grp, dtype=f64, device=dev), torch.zeros(grp, dtype=f64, device=dev)

        def view(base, name, ranges):
            t = base[name]
            if ranges is None or name in ("z", "x"):
                return t
            for dim, (s0, n) in enumerate(zip(rccsdt_q._starts(ranges, origin), sh.lengths(name, ranges))):
                if s0 != 0 or n != t.shape[dim]:
                    t = t.narrow(dim, s0, n)
            return t

        def store(subs):
            ins, o = subs.split("->")
            return ins, o, (o[4:] + o[:4] if len(o) == 8 else o)

        for phase, subs, (xn, xr), (yn, yr), on, al in terms:
            ins, o, os_ = store(subs)
            if on not in bufs:
                bufs[on] = torch.zeros(sh.shape[on], dtype=f64, device=dev)
                gbufs[on] = torch.zeros(sh.shape[on], dtype=f64, device=dev)
            bufs[on].add_(torch.einsum(ins + "->" + os_, view(bufs, xn, xr), view(bufs, yn, yr)), alpha=al)
        # 2. the epilogue's adjoint
        gbufs["x"], gbufs["z"], gzsq = _epilogue_adjoint(bufs["x"], bufs["z"], vvooT, t2T, e_occ, e_vir, r, no, nv,
                                                         g_b, g_p)
        # z4sq = sum vvoo . t2 over the group's ranges
        for vi, ti in _ZSQ:
            V = er["vvoo"][slice(*rng[vi[0]]), slice(*rng[vi[1]])]
            W2 = t2[slice(*rng[ti[0]]), slice(*rng[ti[1]])]
            ger["vvoo"][slice(*rng[vi[0]]), slice(*rng[vi[1]])].add_(
                torch.einsum("ijklabcd," + ti + "->" + vi, gzsq, W2))
            gt2[slice(*rng[ti[0]]), slice(*rng[ti[1]])].add_(torch.einsum("ijklabcd," + vi + "->" + ti, gzsq, V))
        # 3. every einsum of the table in reverse order
        for phase, subs, (xn, xr), (yn, yr), on, al in reversed(terms):
            ins, o, os_ = store(subs)
            xs, ys = ins.split(",")
            gout = gbufs[on]
            view(gbufs, xn, xr).add_(torch.einsum(os_ + "," + ys + "->" + xs, gout, view(bufs, yn, yr)), alpha=al)
            view(gbufs, yn, yr).add_(torch.einsum(xs + "," + os_ + "->" + ys, view(bufs, xn, xr), gout), alpha=al)
        # 4. slabs back into the full T3
        for s in rccsdt_q._SLABS:
            (x0, x1), (y0, y1) = rng[s[1]], rng[s[2]]
            gT[x0:x1, y0:y1].add_(gbufs[s])
        del bufs, gbufs
    # unpack^T, then the projection onto stabilizer-symmetric blocks
    ijk = torch.tensor(canonical_ijk(no), dtype=torch.int32, device=dev)
    gt3 = torch.empty_like(t3)
    t3_residual.perm_gather_(gt3, ijk, nv, 0.0, [(gU.view(no ** 3, nv, nv, nv), 1.0,
                                                  t3_residual.full_strides(no, nv), t3_residual.ALL_S3)])
    ab, bc, al3 = _stab_masks(ijk)
    gt3.div_(1.0 + ab + bc + 3.0 * al3)
    return gt2, gt3, ger


class QEnergyFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, t2, t3, vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo, e_occ, e_vir, blksize, precision):
        nocc, nvir = t2.shape[2], t2.shape[0]
        er = dict(zip(ER_NAMES, (vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo)))
        er = {k: v.contiguous() for k, v in er.items()}
        t3_abc = _c_rccsdt.redistribute_ijk_to_abc(t3.contiguous(), nocc, nvir)
        q = rccsdt_q.QEnergy(nocc, nvir, blksize, precision, device=t3.device)
        out = q.run(er, t2.contiguous(), t3_abc, e_occ.contiguous(), e_vir.contiguous()).clone()
        if not q.status_ok():
            raise RuntimeError("a bounded wait in a GPU kernel gave up (timeout)")
        ctx.blksize = blksize
        ctx.save_for_backward(t2, t3, vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo, e_occ, e_vir)
        return out

    @staticmethod
    def backward(ctx, g):
        t2, t3, vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo, e_occ, e_vir = ctx.saved_tensors
        er = dict(zip(ER_NAMES, (vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo)))
        gt2, gt3, ger = q_energy_vjp(g.detach().cpu().tolist(), er, t2, t3, e_occ, e_vir, t2.shape[2], t2.shape[0],
                                     ctx.blksize)
        return (gt2, gt3) + tuple(ger[k] for k in ER_NAMES) + (None, None, None, None)


def q_energy_fn(t2, t3, vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo, e_occ, e_vir, blksize=4, precision="fp64"):
    """Differentiable [e_bracket, e_paren] (device tensor) with the hand-written backward above.

    t2 [a,b,i,j] (vvoo order), t3 canonical IJK blocks; the forward runs in `precision`,
    the backward in FP64."""
    return QEnergyFunction.apply(t2, t3, vvvo, vooo, vvoo, ovvo, ovov, vvvv, oooo, e_occ, e_vir, blksize, precision)
