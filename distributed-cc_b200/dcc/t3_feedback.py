"""T3 -> lower-order feedback on the GPU (distr_cc/rccsdt.py:253-366).

The reference loops over canonical blocks and every distinct ordering of
each, taking the block (take_t3), symmetrizing it (P3_422 / P3_201) and
issuing small einsums into r1, r2, W_vooo and W_vvvo.  Here:

* r1 (distr_cc/rccsdt.py:270-293): with V = P3_422 of every canonical block
  the paired strings of each case collapse to
      r1[i] += c1 <E[j,k], V[a,b,c]>,  r1[j] += c2 <E[i,k], V[b,a,c]>,
      r1[k] += c3 <E[i,j], V[b,c,a]>       (sums over b, c; E = t1_eris[o,o,v,v])
  with (c1, c2, c3) = (1, 1, 1) for i<j<k, (1, 0, 1/2) for i=j<k,
  (1/2, 1, 0) for i<j=k (the 'cb,acb' partner of a 'bc,abc' string is the same
  sum); the permutations of V move onto E, so three batched GEMMs over t3 itself
  give all three (no V pass), scattered to r1 by a one-hot product
  (deterministic).
* r2, W_vooo, W_vvvo (distr_cc/rccsdt.py:300-316, 340-358): the distinct
  orderings of all canonical blocks are all ordered (x,y,z) once, so with X =
  P3_201 applied to every block of the unpacked U (dcc_t3_unpack_all), each
  string is one contraction over x (and z) for all blocks at once.

All in FP64 (bandwidth-bound: K = nvir or nocc*nvir against 1-6 GB of T3)."""
from __future__ import annotations

import torch

from . import _c_rccsdt
from .t3_residual import unpack_all_

f64 = torch.float64


def _case_coefficients(ijk):
    i, j, k = ijk[:, 0], ijk[:, 1], ijk[:, 2]
    lt_lt = (i < j) & (j < k)
    eq_lt = (i == j) & (j < k)
    lt_eq = (i < j) & (j == k)
    z = torch.zeros(ijk.shape[0], dtype=f64, device=ijk.device)
    c1 = torch.where(lt_lt | eq_lt, 1.0, torch.where(lt_eq, 0.5, 0.0)).to(f64) + z
    c2 = torch.where(lt_lt | lt_eq, 1.0, 0.0).to(f64) + z
    c3 = torch.where(lt_lt, 1.0, torch.where(eq_lt, 0.5, 0.0)).to(f64) + z
    return c1, c2, c3


def r1_add_t3_(r1, t1_eris, t3, ijk, nocc, oovv=None, V=None):
    """r1 += T3 part of r1 (distr_cc/rccsdt.py:262-296); t3 canonical blocks.  oovv: the
    [o,o,v,v] slice of t1_eris when the caller passes the slice alone (t1_eris None).

    The reference contracts V = P3_422(t3) of each block with E = oovv slices:
      Ra[a] = sum_bc E[j,k][b,c] V[a,b,c], Rb[a] = sum_bc E[i,k][b,c] V[b,a,c],
      Rc[a] = sum_bc E[i,j][b,c] V[b,c,a],
    with V[x,y,z] = 4 t[x,y,z] - 2 (t[z,y,x] + t[y,x,z] + t[x,z,y]) + t[y,z,x] + t[z,x,y].
    Moving the permutations onto E, each R is a sum over the free position f of t3 of
    y_f(M)[.] = t3 contracted with a matrix M over its other two positions, where M is
    alpha E + beta E^T:
      Ra = y0(4E1 - 2E1^T) + y1(-2E1 + E1^T) + y2(E1 - 2E1^T)
      Rb = y0(-2E2 + E2^T) + y1(4E2 - 2E2^T) + y2(-2E2 + E2^T)
      Rc = y0(E3 - 2E3^T) + y1(-2E3 + E3^T) + y2(4E3 - 2E3^T)
    (E1 = E[j,k], E2 = E[i,k], E3 = E[i,j]), so three batched GEMMs with three right-hand sides
    read t3 once each and V is never formed.  V: unused (kept for the callers' signature)."""
    n, nvir = t3.shape[0], t3.shape[1]
    E = oovv if oovv is not None else eris_slices(t1_eris, None, nocc)["oovv"]
    il, jl, kl = ijk[:, 0].long(), ijk[:, 1].long(), ijk[:, 2].long()
    c1, c2, c3 = _case_coefficients(ijk)
    E1, E2, E3 = E[jl, kl], E[il, kl], E[il, jl]  # [n][nvir][nvir]

    def mix(a, b, M):
        return a * M + b * M.transpose(1, 2)

    # the matrices of the three free positions, one column per output (Ra, Rb, Rc)
    G0 = torch.stack([mix(4.0, -2.0, E1), mix(-2.0, 1.0, E2), mix(1.0, -2.0, E3)], -1)  # over (y, z)
    G1 = torch.stack([mix(-2.0, 1.0, E1), mix(4.0, -2.0, E2), mix(-2.0, 1.0, E3)], -1)  # over (x, z)
    G2 = torch.stack([mix(1.0, -2.0, E1), mix(-2.0, 1.0, E2), mix(4.0, -2.0, E3)], -1)  # over (x, y)
    nv2 = nvir * nvir
    R = torch.bmm(t3.view(n, nvir, nv2), G0.reshape(n, nv2, 3))
    R += torch.bmm(t3.view(n * nvir, nvir, nvir), G1.reshape(n * nvir, nvir, 3)).view(n, nvir, nvir, 3).sum(1)
    R += torch.bmm(t3.view(n, nv2, nvir).transpose(1, 2), G2.reshape(n, nv2, 3))
    Ra, Rb, Rc = R[..., 0] * c1[:, None], R[..., 1] * c2[:, None], R[..., 2] * c3[:, None]
    eye = torch.eye(nocc, dtype=f64, device=t3.device)
    r1 += eye[il].t() @ Ra + eye[jl].t() @ Rb + eye[kl].t() @ Rc
    return r1


def p3_201_all(t3, nocc, U=None, out=None, unpack_into=None):
    """X = P3_201 of every ordered block of the unpacked T3 [x][y][z][a][b][c].

    U: the unpacked T3 when the caller has it already (unpacked here otherwise), FP64 or FP32
    (X then FP32 too); out: a buffer of at least U's bytes to hold X (a fresh one otherwise); unpack_into: a buffer that
    receives the unpacked T3 in the same pass that writes X (one launch, dcc_t3_unpack_p3: X
    costs no read of U; used where the rows are not 16-byte aligned and the separate passes
    cannot use TMA)."""
    nvir = t3.shape[1]
    if unpack_into is not None:
        X = torch.empty_like(unpack_into) if out is None else out.view(unpack_into.shape)
        _c_rccsdt.t3_unpack_p3(t3, unpack_into, X, nocc, nvir, "P3_201", 1.0, 0.0)
        return X.view(nocc, nocc, nocc, nvir, nvir, nvir)
    if U is None:
        U = torch.empty((nocc ** 3, nvir, nvir, nvir), dtype=f64, device=t3.device)
        unpack_all_(t3, U, nocc, nvir)
    if out is None:
        X = torch.empty_like(U)
    else:  # X in the leading bytes of out (an FP32 X takes half of an FP64 buffer)
        X = out.view(-1).view(torch.uint8)[:U.numel() * U.element_size()].view(U.dtype).view(U.shape)
    if U.dtype == torch.float32:
        _c_rccsdt.t3_spin_summation_f32(U, X, U.shape[0], nvir, "P3_201", 1.0, 0.0)
    else:
        _c_rccsdt.t3_spin_summation(U, X, U.shape[0], nvir, "P3_201", 1.0, 0.0)
    return X.view(nocc, nocc, nocc, nvir, nvir, nvir)


def eris_slices(t1_eris, t1_fock, nocc):
    """The pieces of the dressed Fock matrix and ERIs the feedback reads (so a caller can
    upload these instead of the whole [nmo]^4 tensor): fock_ov [o,v], oovv, vovv, ooov."""
    o, v = slice(0, nocc), slice(nocc, None)
    sl = {"oovv": t1_eris[o, o, v, v], "vovv": t1_eris[v, o, v, v], "ooov": t1_eris[o, o, o, v]}
    if t1_fock is not None:
        sl["fock_ov"] = t1_fock[o, v]
    return sl


def r2_add_t3_x_(r2, fock_ov, vovv, ooov, X):
    """r2 += T3 part of r2 (distr_cc/rccsdt.py:300-316) from X = p3_201_all(t3), one leading
    occupied index x at a time (the temporaries stay one 1/nocc slice of X):
        r2[y,z,b,c] += 1/2 f[x,a] X[x,y,z,a,b,c] + E[c,x,a,d] X[x,y,z,d,b,a]
        r2[y,l,b,c] -= E[z,x,l,a] X[x,y,z,a,b,c]."""
    no, nv = X.shape[0], X.shape[3]
    e = torch.einsum
    for x in range(no):
        Xx = X[x]
        r2.view(no * no, nv * nv).add_(
            torch.matmul(fock_ov[x].view(1, 1, nv), Xx.reshape(no * no, nv, nv * nv)).view(no * no, nv * nv),
            alpha=0.5)
        r2 += e('cad,yzdba->yzbc', vovv[:, x], Xx)
        r2 -= e('zla,yzabc->ylbc', ooov[:, x], Xx)
    return r2


def r2_add_t3_(r2, t1_fock, t1_eris, X, nocc):
    """r2 += T3 part of r2 (distr_cc/rccsdt.py:300-316) from X = p3_201_all(t3)."""
    sl = eris_slices(t1_eris, t1_fock, nocc)
    return r2_add_t3_x_(r2, sl["fock_ov"], sl["vovv"], sl["ooov"], X)


def intermediates_t3_add_x_(W_vooo, W_vvvo, oovv, X):
    """W_vooo, W_vvvo += T3 parts (distr_cc/rccsdt.py:323-366) from X = p3_201_all(t3), one
    leading occupied index x at a time:
        W_vooo[a,m,y,z] += E[m,x,d,e] X[x,y,z,e,a,d],  W_vvvo[a,b,d,y] -= E[z,x,d,e] X[x,y,z,e,b,a]."""
    no = X.shape[0]
    e = torch.einsum
    for x in range(no):
        W_vooo += e('mde,yzead->amyz', oovv[:, x], X[x])
        W_vvvo -= e('zde,yzeba->abdy', oovv[:, x], X[x])
    return W_vooo, W_vvvo


def intermediates_t3_add_(W_vooo, W_vvvo, t1_eris, X, nocc):
    """W_vooo, W_vvvo += T3 parts (distr_cc/rccsdt.py:323-366) from X = p3_201_all(t3)."""
    return intermediates_t3_add_x_(W_vooo, W_vvvo, eris_slices(t1_eris, None, nocc)["oovv"], X)


class SplitFeedback:
    """The four T3 -> lower-order strings of the split-precision path as tcgen05 GEMMs on
    split operands (r1r2_add_t3_tri_ and intermediates_t3_add_t3_tri, distr_cc/rccsdt.py:
    300-316, 340-358), from X = p3_201_all(t3) read in place through address maps:

        r2[y,z,b,c]     += sum_{x,d,a} E_vovv[c,x,a,d] X[x,y,z,d,b,a]
        r2[y,l,b,c]     -= sum_{x,z,a} E_ooov[z,x,l,a] X[x,y,z,a,b,c]
        W_vooo[a,m,y,z] += sum_{x,e,d} E_oovv[m,x,d,e] X[x,y,z,e,a,d]
        W_vvvo[a,b,d,y] -= sum_{x,z,e} E_oovv[z,x,d,e] X[x,y,z,e,b,a]

    The small E slices are the GEMM's row operand (permuted once so that the contraction index
    is contiguous) and X the column operand; each contraction runs over (x, two more indices) in
    the order that keeps X's contiguous index innermost.  The strings that read X the same way
    (vovv with W_vooo, ooov with W_vvvo: the same columns and contraction over X's axes) are one
    GEMM: their E slices stacked as the rows (nvir + nocc rows, one 128-row tile, so the padded
    MMA rows and the reads of X are paid once for both).  Every value of x is its own piece of
    the split operands (starting on a k-block) and its own GEMM: the tensor cores accumulate in
    FP32 over the other two indices only, and the epilogue sums the nocc partial results in FP64
    -- one FP32 accumulation over the whole contraction (nocc nvir^2 terms at nvir ~ 90) lost
    four digits to cancellation.  The partial results accumulate in an FP64 scratch T[row][column]
    (contiguous, so the epilogue writes whole rows; W_vvvo's own layout puts every element of an
    epilogue row in its own sector), and each string's rows are added to its output once, with a
    permutation.  One split buffer of X (nocc^2 nvir x nocc nvir^2 elements, two 2-byte pieces
    each in bf16x3) serves the two GEMMs in turn.  The f_ov term of r2 (K = nvir) stays an FP64
    product."""

    def __init__(self, nocc, nvir, precision, device="cuda"):
        from . import contract
        self.c = contract
        self.no, self.nv, self.kind, self.dev = nocc, nvir, contract.KIND[precision], device
        no, nv = nocc, nvir
        Sz = nv ** 3
        Sy, Sx, Sp, Sq = no * Sz, no * no * Sz, nv * nv, nv
        self.Sx = Sx
        c = contract
        # N, X column map, inner contraction digits of X (R1, R2, S1, S2) after x, E slice and
        # the permutation that puts it in [row][x][k1][k2] order, the string's block of the
        # scratch as [row][column digits] and its permutation to the output's index order,
        # alpha, output
        self.terms = {
            # r2 vovv: rows c, columns (y,z,b); K = (x, d, a); E_vovv[c,x,a,d] -> [c][x][d][a]
            "vovv": dict(N=no * no * nv, fn=c.three(no, nv, Sy, Sz, Sq), kin=(nv, nv, Sp, 1), M=nv,
                         src="vovv", perm=(0, 1, 3, 2), tview=(nv, no, no, nv), tperm=(1, 2, 3, 0),
                         alpha=1.0, out="r2"),
            # r2 ooov: rows l, columns (y,b,c); K = (x, z, a); E_ooov[z,x,l,a] -> [l][x][z][a]
            "ooov": dict(N=no * nv * nv, fn=c.three(nv, nv, Sy, Sq, 1), kin=(no, nv, Sz, Sp), M=no,
                         src="ooov", perm=(2, 1, 0, 3), tview=(no, no, nv, nv), tperm=(1, 0, 2, 3),
                         alpha=-1.0, out="r2"),
            # W_vooo: rows m, columns (y,z,a); K = (x, e, d); E_oovv[m,x,d,e] -> [m][x][e][d]
            "wvooo": dict(N=no * no * nv, fn=c.three(no, nv, Sy, Sz, Sq), kin=(nv, nv, Sp, 1), M=no,
                          src="oovv", perm=(0, 1, 3, 2), tview=(no, no, no, nv), tperm=(3, 0, 1, 2),
                          alpha=1.0, out="W_vooo"),
            # W_vvvo: rows d, columns (y,b,a); K = (x, z, e); E_oovv[z,x,d,e] -> [d][x][z][e]
            "wvvvo": dict(N=no * nv * nv, fn=c.three(nv, nv, Sy, Sq, 1), kin=(no, nv, Sz, Sp), M=nv,
                          src="oovv", perm=(2, 1, 0, 3), tview=(nv, no, nv, nv), tperm=(3, 2, 0, 1),
                          alpha=-1.0, out="W_vvvo"),
        }
        dt = torch.bfloat16 if self.kind == 0 else torch.float32
        self.blk = contract._KBLK[self.kind]
        self.plans = {}
        xmax = 0
        for name, tm in self.terms.items():
            R1, R2, S1, S2 = tm["kin"]
            pieces = [(x, 1) for x in range(no)]  # one piece (and one GEMM) per value of x
            ks = [R1 * R2] * no
            w = contract.padded_k(R1 * R2, self.kind)
            Kp = w * no
            self.plans[name] = (pieces, ks, Kp)
            xmax = max(xmax, tm["N"] * Kp)
        # the row operand and the scratch hold both strings of a group: at most nvir + nocc rows
        emax = (nv + no) * max(p[2] for p in self.plans.values())
        tmax = (nv + no) * max(tm["N"] for tm in self.terms.values())
        self._xhi = torch.empty(xmax, dtype=dt, device=device)
        self._xlo = torch.empty(xmax, dtype=dt, device=device)
        self._ehi = torch.empty(emax, dtype=dt, device=device)
        self._elo = torch.empty(emax, dtype=dt, device=device)
        self._scratch = torch.empty(tmax, dtype=f64, device=device)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)

    def _operand(self, rows, ks, Kp, hi, lo):
        n = rows * Kp
        buf = (hi[:n].view(rows, Kp), lo[:n].view(rows, Kp))
        return self.c.Split(rows, kind=self.kind, buffers=buf, pieces=ks, align=self.blk)

    def run(self, X, E, outs, names=("vovv", "ooov", "wvooo", "wvvvo")):
        """outs[...] += the strings above.  X: [no,no,no,nv,nv,nv] FP64, contiguous; E: the
        slices {'vovv', 'ooov', 'oovv'} of eris_slices on the device; outs: {'r2', 'W_vooo',
        'W_vvvo'} FP64 device tensors.  Strings that read X the same way share one split of X
        and one GEMM per piece."""
        c = self.c
        Xf = X.reshape(-1)
        done = set()
        for name in names:
            if name in done:
                continue
            tm = self.terms[name]
            group = [n for n in names if n not in done and self.terms[n]["fn"] == tm["fn"]
                     and self.terms[n]["kin"] == tm["kin"] and self.terms[n]["N"] == tm["N"]]
            pieces, ks, Kp = self.plans[name]
            R1, R2, S1, S2 = tm["kin"]
            N = tm["N"]
            B = self._operand(N, ks, Kp, self._xhi, self._xlo)
            for i, (x0, xc) in enumerate(pieces):
                B.fill_piece(i, Xf[x0 * self.Sx:], tm["fn"], c.three(R1, R2, self.Sx, S1, S2))
            # the strings' E slices stacked: [row][x][k1][k2]
            Ep = torch.cat([E[self.terms[n]["src"]].permute(*self.terms[n]["perm"]) for n in group]).contiguous()
            M = Ep.shape[0]
            A = self._operand(M, ks, Kp, self._ehi, self._elo)
            row = self.no * R1 * R2
            for i, (x0, xc) in enumerate(pieces):
                A.fill_piece(i, Ep[:, x0:], c.lin(row), c.lin(1))
            T = self._scratch[:M * N].view(M, N)
            for i, (off, _, w) in enumerate(A.pieces):
                c.gemm_range_(A, B, T, c.lin(N), c.lin(1), 1.0, 0.0 if i == 0 else 1.0, self.status, off, w)
            r0 = 0
            for n in group:
                tn = self.terms[n]
                outs[tn["out"]].add_(T[r0:r0 + tn["M"]].view(tn["tview"]).permute(*tn["tperm"]), alpha=tn["alpha"])
                r0 += tn["M"]
                done.add(n)
        return outs
