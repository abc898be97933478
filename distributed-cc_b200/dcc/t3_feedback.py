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


def r1_add_t3_(r1, t1_eris, t3, ijk, nocc):
    """r1 += T3 part of r1 (distr_cc/rccsdt.py:262-296); t3 canonical blocks."""
    nvir = t3.shape[1]
    o, v = slice(0, nocc), slice(nocc, None)
    V = t3.clone()
    _c_rccsdt.t3_spin_summation_inplace_(V, V.shape[0], nvir, "P3_422", 1.0, 0.0)
    E = t1_eris[o, o, v, v]
    il, jl, kl = ijk[:, 0].long(), ijk[:, 1].long(), ijk[:, 2].long()
    c1, c2, c3 = _case_coefficients(ijk)
    Ra = torch.einsum('qbc,qabc->qa', E[jl, kl], V) * c1[:, None]
    Rb = torch.einsum('qbc,qbac->qa', E[il, kl], V) * c2[:, None]
    Rc = torch.einsum('qbc,qbca->qa', E[il, jl], V) * c3[:, None]
    eye = torch.eye(nocc, dtype=f64, device=t3.device)
    r1 += eye[il].t() @ Ra + eye[jl].t() @ Rb + eye[kl].t() @ Rc
    return r1


def p3_201_all(t3, nocc, U=None):
    """X = P3_201 of every ordered block of the unpacked T3 [x][y][z][a][b][c]."""
    nvir = t3.shape[1]
    if U is None:
        U = torch.empty((nocc ** 3, nvir, nvir, nvir), dtype=f64, device=t3.device)
        unpack_all_(t3, U, nocc, nvir)
    X = U.clone()
    _c_rccsdt.t3_spin_summation_inplace_(X, X.shape[0], nvir, "P3_201", 1.0, 0.0)
    return X.view(nocc, nocc, nocc, nvir, nvir, nvir)


def r2_add_t3_(r2, t1_fock, t1_eris, X, nocc):
    """r2 += T3 part of r2 (distr_cc/rccsdt.py:300-316) from X = p3_201_all(t3)."""
    o, v = slice(0, nocc), slice(nocc, None)
    e = torch.einsum
    r2 += 0.5 * e('xa,xyzabc->yzbc', t1_fock[o, v], X)
    r2 += e('cxad,xyzdba->yzbc', t1_eris[v, o, v, v], X)
    r2 -= e('zxla,xyzabc->ylbc', t1_eris[o, o, o, v], X)
    return r2


def intermediates_t3_add_(W_vooo, W_vvvo, t1_eris, X, nocc):
    """W_vooo, W_vvvo += T3 parts (distr_cc/rccsdt.py:323-366) from X = p3_201_all(t3)."""
    o, v = slice(0, nocc), slice(nocc, None)
    E = t1_eris[o, o, v, v]
    W_vooo += torch.einsum('mxde,xyzead->amyz', E, X)
    W_vvvo -= torch.einsum('zxde,xyzeba->abdy', E, X)
    return W_vooo, W_vvvo
