"""Pin the C restatement oracle against the reference's own C helpers (compiled
from the reference sources into oracle/_ref).  Float kernels must agree bit for
bit (numerical equality, +0 == -0); index maps exactly."""
import ctypes
import itertools

import numpy as np
import pytest

from oracle.oracle import P3_PATTERNS, P4_PATTERNS


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _ijk_list(nocc):
    return [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]


@pytest.mark.parametrize("nvir", [1, 2, 3, 5, 8, 13])
@pytest.mark.parametrize("pattern", list(P3_PATTERNS))
def test_t3_spin_sum(oracle, reference, nvir, pattern):
    rng = np.random.default_rng(nvir)
    for alpha, beta in [(1.0, 0.0), (-1.0 / 6.0, 1.0), (0.5, -0.25)]:
        A = rng.standard_normal((nvir,) * 3)
        ref = A.copy()
        reference.t3_single_spin_summation_inplace_(_p(ref), nvir, pattern.encode(), alpha, beta)
        got = oracle.t3_spin_sum(A.copy(), nvir, pattern, alpha, beta)
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("nvir", [1, 2, 5, 9])
def test_t3_triple_sym_transpose_add(oracle, reference, nvir):
    rng = np.random.default_rng(1)
    A = rng.standard_normal((nvir,) * 3)
    B = [np.empty_like(A) for _ in range(3)]
    reference.t3_spin_summation_triple_sym_(_p(A), _p(B[0]), _p(B[1]), _p(B[2]), nvir)
    for got, ref in zip(oracle.t3_triple_sym(A, nvir), B):
        assert np.array_equal(got, ref)
    T = np.empty_like(A)
    reference.t3_transpose_add_(_p(A), _p(T), nvir)
    assert np.array_equal(oracle.t3_transpose_add(A, nvir), T)


@pytest.mark.parametrize("nocc,nvir", [(1, 3), (3, 4), (4, 2)])
def test_take_t3_all_orderings(oracle, reference, nocc, nvir):
    rng = np.random.default_rng(2)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = rng.standard_normal((n3, nvir, nvir, nvir))
    loc = np.arange(n3, dtype=np.int64)
    for i, j, k in itertools.product(range(nocc), repeat=3):
        ref = np.zeros((nvir,) * 3)
        reference.take_t3_ijk_single_(_p(t3), _p(ref), _p(loc), i, j, k, nocc, nvir)
        got, rc = oracle.take_t3(t3, loc, i, j, k, nocc, nvir)
        assert rc == 0 and np.array_equal(got, ref)


def test_ijk_maps(oracle):
    for nocc in range(1, 9):
        for idx, (i, j, k) in enumerate(_ijk_list(nocc)):
            assert oracle.ijk_to_linear(i, j, k, nocc) == idx
        idx = 0
        for i in range(nocc):
            for j in range(i, nocc):
                for k in range(j, nocc):
                    for l in range(k, nocc):
                        assert oracle.ijkl_to_linear(i, j, k, l, nocc) == idx
                        idx += 1


@pytest.mark.parametrize("nvir", [1, 2, 3, 5, 6])
@pytest.mark.parametrize("pattern", list(P4_PATTERNS))
def test_t4_spin_sum(oracle, reference, nvir, pattern):
    rng = np.random.default_rng(3)
    nouter = 3
    for alpha, beta in [(1.0, 0.0), (0.75, 1.0)]:
        A = rng.standard_normal((nouter,) + (nvir,) * 4)
        ref = A.copy()
        reference.t4_spin_summation_inplace_(_p(ref), nouter, nvir, pattern.encode(), alpha, beta)
        got = oracle.t4_spin_sum(A.copy(), nouter, nvir, pattern, alpha, beta)
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("nvir", [1, 2, 4, 5, 9])
@pytest.mark.parametrize("pattern", ["P4_full", "P4_442", "P4_201"])
def test_t4_single_spin_sum(oracle, reference, nvir, pattern):
    rng = np.random.default_rng(4)
    A = rng.standard_normal((nvir,) * 4)
    ref = A.copy()
    reference.t4_single_spin_summation_inplace_(_p(ref), nvir, pattern.encode(), 1.0, 0.5)
    got = oracle.t4_spin_sum(A.copy(), 1, nvir, pattern, 1.0, 0.5)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("nvir", [1, 2, 3, 4, 6, 11])
def test_t4_project(oracle, reference, nvir):
    rng = np.random.default_rng(5)
    A = rng.standard_normal((2,) + (nvir,) * 4)
    for alpha, beta in [(1.0, 0.0), (-1.0, 1.0)]:
        ref = A.copy()
        reference.t4_project_1_minus_p4_p31_inplace_(_p(ref), 2, nvir, alpha, beta)
        got = oracle.t4_project(A.copy(), 2, nvir, alpha, beta)
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("nvir", [1, 3, 5])
def test_t4_transpose_add_quadruple_sym(oracle, reference, nvir):
    rng = np.random.default_rng(6)
    A = rng.standard_normal((nvir,) * 4)
    D = np.empty_like(A)
    reference.t4_transpose_add_(_p(A), _p(D), nvir)
    assert np.array_equal(oracle.t4_transpose_add(A, nvir), D)
    B = [np.empty_like(A) for _ in range(4)]
    reference.t4_spin_summation_quadruple_sym_(_p(A), *[_p(b) for b in B], nvir)
    for got, ref in zip(oracle.t4_quadruple_sym(A, nvir), B):
        assert np.array_equal(got, ref)


def _stored_ijkl(nocc):
    out = []
    for i in range(nocc):
        for j in range(i, nocc):
            for k in range(j, nocc):
                for l in range(k, nocc):
                    if (i == j == k) or (j == k == l):
                        continue
                    out.append((i, j, k, l))
    return out


def test_r4_divide_and_unpack(oracle, reference):
    rng = np.random.default_rng(7)
    nocc, nvir = 4, 3
    stored = _stored_ijkl(nocc)
    nfull = nocc * (nocc + 1) * (nocc + 2) * (nocc + 3) // 24
    full_to_local = np.full(nfull, -1, dtype=np.int64)
    for q, (i, j, k, l) in enumerate(stored):
        full_to_local[oracle.ijkl_to_linear(i, j, k, l, nocc)] = q
    r4 = rng.standard_normal((len(stored),) + (nvir,) * 4)
    eia = rng.uniform(-3, -0.5, (nocc, nvir))
    ijkl = np.asarray(stored, dtype=np.int32)
    ref = r4.copy()
    reference.r4_local_tri_divide_e_(_p(ref), _p(eia), _p(ijkl), len(stored), nvir)
    assert np.array_equal(oracle.r4_divide(r4.copy(), eia, ijkl), ref)
    for i, j, k, l in itertools.product(range(nocc), repeat=4):
        want = np.full((nvir,) * 4, 7.0)
        reference.unpack_t4_ijkl_single_(_p(r4), _p(want), _p(full_to_local), i, j, k, l, nocc, nvir)
        got, _ = oracle.unpack_t4(r4, full_to_local, i, j, k, l, nocc, nvir, out=np.full((nvir,) * 4, 7.0))
        assert np.array_equal(got, want)


def test_q_division_and_factor(oracle, reference):
    rng = np.random.default_rng(8)
    nocc, nvir, blk = 3, 7, 3
    e_occ = rng.uniform(-1.5, -0.3, nocc)
    e_vir = rng.uniform(0.1, 3.0, nvir)
    for (a0, a1), (b0, b1), (c0, c1), (d0, d1) in [((0, 3), (0, 3), (3, 6), (6, 7)), ((3, 6), (3, 6), (3, 6), (6, 7))]:
        r4 = rng.standard_normal((blk,) * 4 + (nocc,) * 4)
        ref = r4.copy()
        reference.e_abcdijkl_division_(_p(ref), _p(e_occ), _p(e_vir), a0, a1, b0, b1, c0, c1, d0, d1,
                                       blk, blk, blk, blk, nocc)
        got = oracle.e_abcdijkl_division(r4.copy(), e_occ, e_vir, a0, a1, b0, b1, c0, c1, d0, d1,
                                         blk, blk, blk, nocc)
        assert np.array_equal(got, ref)
        factor = np.zeros((blk,) * 4)
        for ia, ib, ic, id_ in itertools.product(range(blk), repeat=4):
            a, b, c, d = a0 + ia, b0 + ib, c0 + ic, d0 + id_
            if a < a1 and b < b1 and c < c1 and d < d1:
                factor[ia, ib, ic, id_] = oracle.q_factor(a, b, c, d)
        ref2 = ref.copy()
        reference.t4_multiply_factor_(_p(ref2), _p(factor), blk, blk, blk, blk, nocc)
        assert np.array_equal(oracle.t4_multiply_factor(ref.copy(), factor, blk, blk, blk, blk, nocc), ref2)


def _abc_storage(nvir, nocc, rng):
    nabc = nvir * (nvir + 1) * (nvir + 2) // 6
    return rng.standard_normal((nabc, nocc, nocc, nocc))


@pytest.mark.parametrize("nocc,nvir,blk", [(2, 5, 2), (3, 7, 3), (1, 4, 4)])
def test_fill_t3_abc(oracle, reference, nocc, nvir, blk):
    rng = np.random.default_rng(9)
    t3_abc = _abc_storage(nvir, nocc, rng)
    ptr = np.array([t3_abc[g].ctypes.data for g in range(len(t3_abc))], dtype=np.uintp)
    for a0 in range(0, nvir, blk):
        for b0 in range(0, nvir, blk):
            a1, b1 = min(a0 + blk, nvir), min(b0 + blk, nvir)
            size = blk * blk * nvir * nocc ** 3
            ref = np.zeros((blk, blk, nvir, nocc, nocc, nocc))
            reference.fill_t3_from_ptr_array(_p(ref), a0, a1, b0, b1, nvir, nocc, _p(ptr), blk, size, len(ptr))
            got = np.zeros_like(ref)
            miss = oracle.fill_t3_abc(got, a0, a1, b0, b1, nvir, nocc, t3_abc, None, blk)
            assert miss == 0 and np.array_equal(got, ref)


@pytest.mark.parametrize("nocc,nvir", [(1, 2), (2, 3), (3, 4), (4, 3)])
def test_ijk_to_abc_matches_reference_records(oracle, reference, nocc, nvir):
    rng = np.random.default_rng(10)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = rng.standard_normal((n3, nvir, nvir, nvir))  # deliberately not permutation-symmetric
    ref = reference.ijk_to_abc_records(t3, nocc, nvir)
    got = oracle.ijk_to_abc(t3, nocc, nvir)
    assert np.array_equal(got, ref)
