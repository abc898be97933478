"""Generate tests/golden/ref_helpers.npz from the reference's own C helpers.

The reference library is compiled from the reference sources by oracle/Makefile
(oracle/_ref/libdistr_cc_ref.so).  Run from the repository root:

    make -C oracle && python tests/golden/make_golden.py

Every case stores its seeded input and the reference output; the fixtures are
small so the whole file stays well under a megabyte.
"""
import ctypes
import itertools
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Reference  # noqa: E402


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def main():
    ref = Reference()
    rng = np.random.default_rng(20261203)
    out = {}
    nvir = 7
    # P3 symmetrizers
    for pat in ("P3_full", "P3_422", "P3_201"):
        A = rng.standard_normal((nvir,) * 3)
        B = A.copy()
        ref.t3_single_spin_summation_inplace_(_p(B), nvir, pat.encode(), -1.0 / 6.0, 1.0)
        out["p3_%s_in" % pat], out["p3_%s_out" % pat] = A, B
    A = rng.standard_normal((nvir,) * 3)
    B = [np.empty_like(A) for _ in range(3)]
    ref.t3_spin_summation_triple_sym_(_p(A), _p(B[0]), _p(B[1]), _p(B[2]), nvir)
    T = np.empty_like(A)
    ref.t3_transpose_add_(_p(A), _p(T), nvir)
    out.update(tsym_in=A, tsym_b0=B[0], tsym_b1=B[1], tsym_b2=B[2], tadd_out=T)
    # take_t3 for every ordering of a nocc=3 set of blocks
    nocc = 3
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = rng.standard_normal((n3, 4, 4, 4))
    loc = np.arange(n3, dtype=np.int64)
    takes = np.zeros((nocc ** 3, 4, 4, 4))
    for q, (i, j, k) in enumerate(itertools.product(range(nocc), repeat=3)):
        ref.take_t3_ijk_single_(_p(t3), _p(takes[q]), _p(loc), i, j, k, nocc, 4)
    out.update(take_in=t3, take_out=takes)
    # T4: projector, P4 patterns, transpose-add, quadruple sym
    nv4 = 5
    A = rng.standard_normal((2,) + (nv4,) * 4)
    B = A.copy()
    ref.t4_project_1_minus_p4_p31_inplace_(_p(B), 2, nv4, 1.0, 0.0)
    out.update(proj_in=A, proj_out=B)
    for pat in ("P4_full", "P4_444", "P4_442", "P4_201"):
        A = rng.standard_normal((2,) + (nv4,) * 4)
        B = A.copy()
        ref.t4_spin_summation_inplace_(_p(B), 2, nv4, pat.encode(), 1.0, 0.0)
        out["p4_%s_in" % pat], out["p4_%s_out" % pat] = A, B
    A = rng.standard_normal((nv4,) * 4)
    D = np.empty_like(A)
    ref.t4_transpose_add_(_p(A), _p(D), nv4)
    Q = [np.empty_like(A) for _ in range(4)]
    ref.t4_spin_summation_quadruple_sym_(_p(A), *[_p(q) for q in Q], nv4)
    out.update(t4sym_in=A, t4tadd_out=D, t4qs_b0=Q[0], t4qs_b1=Q[1], t4qs_b2=Q[2], t4qs_b3=Q[3])
    # (Q) denominator + factor on one task block
    nq, nvq, blk = 3, 6, 3
    e_occ = rng.uniform(-1.5, -0.3, nq)
    e_vir = rng.uniform(0.1, 3.0, nvq)
    r4 = rng.standard_normal((blk,) * 4 + (nq,) * 4)
    R = r4.copy()
    ref.e_abcdijkl_division_(_p(R), _p(e_occ), _p(e_vir), 0, 3, 0, 3, 3, 6, 3, 6, blk, blk, blk, blk, nq)
    out.update(qdiv_in=r4, qdiv_out=R, q_eocc=e_occ, q_evir=e_vir)
    # IJK -> ABC through the reference record pack/unpack (one rank)
    no, nv = 3, 4
    t3 = rng.standard_normal((no * (no + 1) * (no + 2) // 6, nv, nv, nv))
    out.update(i2a_in=t3, i2a_out=ref.ijk_to_abc_records(t3, no, nv))
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_helpers.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
