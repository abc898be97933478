"""CPU checks of the C ABI: the library loads, exports every symbol that
include/*.h declares, and rejects bad arguments on the host (these paths
return before any CUDA call, so they run without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        names.update(re.findall(r"^DCC_API\s+[^;(]*?\b(dcc_\w+)\s*\(", src, flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def L():
    from dcc import _lib
    return _lib


def test_every_declared_symbol_is_exported(L):
    names = _declared()
    assert len(names) >= 26
    missing = [n for n in names if not hasattr(L.lib(), n)]
    assert not missing, missing


def test_version(L):
    assert L.lib().dcc_version() >= 100


def test_bad_pattern_is_reported(L):
    rc = L.lib().dcc_t3_spin_summation_inplace(None, 0, 4, b"P3_bogus", 1.0, 0.0, None)
    assert rc == 1 and "P3_bogus" in L.last_error()
    rc = L.lib().dcc_t4_spin_summation_inplace(None, 1, 3, b"P4_422", 1.0, 0.0, None)
    assert rc == 1  # the reference accepts only P4_full/P4_444/P4_442/P4_201
    rc = L.lib().dcc_t3_spin_summation_inplace(None, 0, 4, None, 1.0, 0.0, None)
    assert rc == 1


def test_null_and_shape_errors(L):
    lib = L.lib()
    assert lib.dcc_t3_spin_summation_inplace(None, 2, 4, b"P3_full", 1.0, 0.0, None) == 3
    assert lib.dcc_t3_transpose_add(None, None, 1, 3, None) == 3
    assert lib.dcc_t4_transpose_add(None, None, 3, None) == 3
    assert lib.dcc_t3_spin_summation_inplace(None, -1, 4, b"P3_full", 1.0, 0.0, None) == 2
    m = (ctypes.c_int64 * 4)(0, 1, 2, 3)
    assert lib.dcc_take_t3_ijk_single(None, None, m, 0, 0, 5, 2, 4, None) == 2
    assert lib.dcc_fill_t3_from_abc(None, 0, 5, 0, 1, 4, 2, None, 1, None) == 2
    assert lib.dcc_e_abcdijkl_division(None, None, None, 0, 5, 0, 1, 0, 1, 0, 1, 4, 4, 4, 4, 2, None) == 2


def test_not_local_block(L):
    m = (ctypes.c_int64 * 4)(-1, -1, -1, -1)
    rc = L.lib().dcc_take_t3_ijk_single(ctypes.c_void_p(8), ctypes.c_void_p(8), m, 0, 1, 0, 2, 3, None)
    assert rc == 7 and "not stored" in L.last_error()


def test_zero_sizes_are_noops(L):
    lib = L.lib()
    assert lib.dcc_t3_spin_summation_inplace(None, 0, 5, b"P3_422", 1.0, 0.0, None) == 0
    assert lib.dcc_t4_project_1_minus_p4_p31_inplace(None, 0, 5, 1.0, 0.0, None) == 0
    assert lib.dcc_t4_add(None, None, 0, None) == 0


def test_workspace_sizes(L):
    lib = L.lib()
    assert lib.dcc_t3_update_workspace_bytes(220, 90) >= 16
    assert lib.dcc_q_epilogue_workspace_bytes(4, 10) >= 16


def test_python_mirrors_validate_like_reference():
    import torch
    from dcc import _c_rccsdt
    with pytest.raises(TypeError):
        _c_rccsdt.t3_single_spin_summation_inplace_(torch.zeros(8, dtype=torch.float32), 2, "P3_full")
    with pytest.raises(ValueError):
        _c_rccsdt.t3_single_spin_summation_inplace_(torch.zeros(4, 2, dtype=torch.float64).t(), 2, "P3_full")
    with pytest.raises(ValueError):  # host tensor: this library computes on the GPU only
        _c_rccsdt.t3_single_spin_summation_inplace_(torch.zeros(8, dtype=torch.float64), 2, "P3_full")


def test_split_gemm_host_validation_accepts_our_maps(L):
    """The maps the drivers pass must clear the host-side checks: on a box
    without a GPU a valid call gets as far as the launch (DCC_ERR_CUDA), an
    invalid one stops at DCC_ERR_SHAPE."""
    import torch
    from dcc import contract as c
    if torch.cuda.is_available():
        pytest.skip("checks the no-device fall-through")
    from dcc import t3_residual as tr
    fake = ctypes.c_void_p(4096)
    nv, n, no = 90, 220, 10
    K = no * nv
    plan = tr.s_plan(no, nv)
    # (M, K, kw, ld, k0, row map, k map) of every split the drivers issue
    splits = [(n * nv, nv * nv, 8128, 8128, 0, am, ak) for am, ak, _, _ in c.wvvvv_maps(nv)]
    splits += [(no * nv * nv, nv, 128, 128, 0) + plan["x"]["a"][0][1:],
               (no * no * nv, nv, 128, 128, 0) + plan["x"]["b"][0][1:],
               (no * nv, K, 960, 960, 0) + plan["t1"]["a"][0][1:]]
    for rows, ent in ((no * nv, plan["oo"]["a"]), (no * no * nv * nv, plan["oo"]["b"])):
        sp = c.Split(rows, kind=0, device="cpu", pieces=[K, K])
        splits += [(rows, k, w, sp.Kp, off, fm, fk) for (off, k, w), (_, fm, fk) in zip(sp.pieces, ent)]
    for M, Kk, kw, ld, k0, fm, fk in splits:
        rc = c._split(fake, fake, fake, M, Kk, kw, ld, k0, c._i64x14(fm, fk), 0, None)
        assert rc == 4, L.last_error()
    # (M, N, Kp, lda, ldb, out maps) of every GEMM
    epis = [(n * nv, nv * nv, 8128, 8128, 8128, er, ec) for _, _, er, ec in c.wvvvv_maps(nv)]
    epis += [(no * nv * nv, no * no * nv, 128, 128, 128) + plan["x"]["out"],
             (no * nv, no * no * nv * nv, 1856, 1856, 1856) + plan["oo"]["out"],
             (no * nv, no * no * nv * nv, 960, 960, 1856) + plan["t1"]["out"]]
    for M, Nn, Kp, lda, ldb, fr, fc in epis:
        rc = c._gemm(fake, fake, lda, fake, fake, ldb, M, Nn, Kp, fake, c._i64x14(fr, fc), 1.0, 1.0, 0, fake, None)
        assert rc == 4, L.last_error()
    rc = c._gemm(fake, fake, 100, fake, fake, 100, 10, 10, 100, fake, c._i64x14(c.lin(10), c.lin(1)), 1.0, 0.0, 0,
                 fake, None)
    assert rc == 2  # Kp not a multiple of 64
    rc = c._gemm(fake, fake, 64, fake, fake, 60, 10, 10, 64, fake, c._i64x14(c.lin(10), c.lin(1)), 1.0, 0.0, 0,
                 fake, None)
    assert rc == 2  # ldb < Kp
    rc = c._split(fake, fake, fake, 10, 10, 64, 64, 0, c._i64x14((0, 1, 0, 0, 1), c.lin(1)), 0, None)
    assert rc == 2  # radix 0
    rc = c._split(fake, fake, fake, 10, 10, 64, 100, 64, c._i64x14(c.lin(10), c.lin(1)), 0, None)
    assert rc == 2  # piece runs past the row pitch


def test_three_digit_map_helpers():
    from dcc import contract as c
    f = lambda m, R1, R2, S0, S1, S2: (m // (R1 * R2)) * S0 + ((m // R2) % R1) * S1 + (m % R2) * S2  # noqa: E731
    for m in [0, 1, 7, 89, 90, 8099, 8100, 19799]:
        assert f(m, *c.lin(3)) == 3 * m
        assert f(m, *c.two(90, 1000, 7)) == (m // 90) * 1000 + (m % 90) * 7


def test_diis_vector_layout(L):
    """dcc_diis_vector_length: segments start on multiples of 32 elements (host-only call)."""
    lib = L.lib()
    lib.dcc_diis_vector_length.restype = ctypes.c_int64
    lib.dcc_diis_vector_length.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    n = (ctypes.c_int64 * 3)(5, 40, 0)
    off = (ctypes.c_int64 * 3)()
    assert lib.dcc_diis_vector_length(n, 3, off) == 32 + 64 + 0
    assert list(off) == [0, 32, 96]
    assert lib.dcc_diis_vector_length(n, 0, None) == -1
