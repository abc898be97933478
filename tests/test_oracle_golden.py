"""The C restatement oracle against the committed reference fixtures
(tests/golden/ref_helpers.npz, made by tests/golden/make_golden.py from the
reference's own C helpers).  Runs without the reference present."""
import itertools
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_helpers.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


@pytest.mark.parametrize("pat", ["P3_full", "P3_422", "P3_201"])
def test_p3(oracle, g, pat):
    A = g["p3_%s_in" % pat].copy()
    assert np.array_equal(oracle.t3_spin_sum(A, A.shape[0], pat, -1.0 / 6.0, 1.0), g["p3_%s_out" % pat])


def test_triple_sym_transpose_add(oracle, g):
    A = g["tsym_in"]
    B = oracle.t3_triple_sym(A, A.shape[0])
    for m in range(3):
        assert np.array_equal(B[m], g["tsym_b%d" % m])
    assert np.array_equal(oracle.t3_transpose_add(A, A.shape[0]), g["tadd_out"])


def test_take_t3(oracle, g):
    t3 = g["take_in"]
    loc = np.arange(t3.shape[0], dtype=np.int64)
    for q, (i, j, k) in enumerate(itertools.product(range(3), repeat=3)):
        got, rc = oracle.take_t3(t3, loc, i, j, k, 3, t3.shape[1])
        assert rc == 0 and np.array_equal(got, g["take_out"][q])


def test_t4_family(oracle, g):
    A = g["proj_in"].copy()
    assert np.array_equal(oracle.t4_project(A, 2, A.shape[1], 1.0, 0.0), g["proj_out"])
    for pat in ("P4_full", "P4_444", "P4_442", "P4_201"):
        A = g["p4_%s_in" % pat].copy()
        assert np.array_equal(oracle.t4_spin_sum(A, 2, A.shape[1], pat, 1.0, 0.0), g["p4_%s_out" % pat])
    A = g["t4sym_in"]
    assert np.array_equal(oracle.t4_transpose_add(A, A.shape[0]), g["t4tadd_out"])
    for m, b in enumerate(oracle.t4_quadruple_sym(A, A.shape[0])):
        assert np.array_equal(b, g["t4qs_b%d" % m])


def test_q_division(oracle, g):
    r4 = g["qdiv_in"].copy()
    got = oracle.e_abcdijkl_division(r4, g["q_eocc"], g["q_evir"], 0, 3, 0, 3, 3, 6, 3, 6, 3, 3, 3, 3)
    assert np.array_equal(got, g["qdiv_out"])


def test_ijk_to_abc(oracle, g):
    assert np.array_equal(oracle.ijk_to_abc(g["i2a_in"], 3, 4), g["i2a_out"])
