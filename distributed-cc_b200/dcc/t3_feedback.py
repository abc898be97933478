"""T3 -> lower-order feedback on the GPU (distr_cc/rccsdt.py:253-366).

The reference loops over canonical blocks and every distinct ordering of
each, taking the block (take_t3), symmetrizing it (P3_422 / P3_201) and
issuing small einsums into r1, r2, W_vooo and W_vvvo.  Here:

* r1 (distr_cc/rccsdt.py:270-293): V = P3_422 of every canonical block
  (one batched kernel); the paired strings of each case collapse to
      r1[i] += c1 <E[j,k], V[a,b,c]>,  r1[j] += c2 <E[i,k], V[b,a,c]>,
      r1[k] += c3 <E[i,j], V[b,c,a]>       (sums over b, c; E = t1_eris[o,o,v,v])
  with (c1, c2, c3) = (1, 1, 1) for i<j<k, (1, 0, 1/2) for i=j<k,
  (1/2, 1, 0) for i<j=k (the 'cb,acb' partner of a 'bc,abc' string is the same
  sum); three batched contractions, scattered to r1 by a one-hot product
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
    [o,o,v,v] slice of t1_eris when the caller passes the slice alone (t1_eris None);
    V: a scratch buffer of t3's size."""
    nvir = t3.shape[1]
    V = t3.clone() if V is None else V.copy_(t3)
    _c_rccsdt.t3_spin_summation_inplace_(V, V.shape[0], nvir, "P3_422", 1.0, 0.0)
    E = oovv if oovv is not None else eris_slices(t1_eris, None, nocc)["oovv"]
    il, jl, kl = ijk[:, 0].long(), ijk[:, 1].long(), ijk[:, 2].long()
    c1, c2, c3 = _case_coefficients(ijk)
    Ra = torch.einsum('qbc,qabc->qa', E[jl, kl], V) * c1[:, None]
    Rb = torch.einsum('qbc,qbac->qa', E[il, kl], V) * c2[:, None]
    Rc = torch.einsum('qbc,qbca->qa', E[il, jl], V) * c3[:, None]
    eye = torch.eye(nocc, dtype=f64, device=t3.device)
    r1 += eye[il].t() @ Ra + eye[jl].t() @ Rb + eye[kl].t() @ Rc
    return r1


def p3_201_all(t3, nocc, U=None, out=None):
    """X = P3_201 of every ordered block of the unpacked T3 [x][y][z][a][b][c].

    U: the unpacked T3 when the caller has it already (unpacked here otherwise);
    out: a buffer of U's size to hold X (a fresh one otherwise)."""
    nvir = t3.shape[1]
    if U is None:
        U = torch.empty((nocc ** 3, nvir, nvir, nvir), dtype=f64, device=t3.device)
        unpack_all_(t3, U, nocc, nvir)
    X = U.clone() if out is None else out.view(U.shape).copy_(U)
    _c_rccsdt.t3_spin_summation_inplace_(X, X.shape[0], nvir, "P3_201", 1.0, 0.0)
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
