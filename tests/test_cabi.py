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
    from dcc import contract
    if torch.cuda.is_available():
        pytest.skip("checks the no-device fall-through")
    fake = ctypes.c_void_p(4096)
    nv, n = 90, 220
    for amap, emap in contract.wvvvv_maps(nv):
        rc = contract._split(fake, fake, fake, n * nv, nv * nv, contract.padded_k(nv * nv, 0),
                             contract._i64x6(amap), 0, None)
        assert rc == 4, L.last_error()
        rc = contract._gemm(fake, fake, fake, fake, n * nv, nv * nv, contract.padded_k(nv * nv, 0), fake,
                            contract._i64x6(emap), 1.0, 1.0, 0, fake, None)
        assert rc == 4, L.last_error()
    rc = contract._gemm(fake, fake, fake, fake, 10, 10, 100, fake, contract._i64x6((1, 0, 1, 1, 0, 1)), 1.0, 0.0, 0,
                        fake, None)
    assert rc == 2  # Kp not a multiple of 64


def test_residual_split_maps_clear_host_checks(L):
    import torch
    from dcc import contract
    if torch.cuda.is_available():
        pytest.skip("checks the no-device fall-through")
    fake = ctypes.c_void_p(4096)
    no, nv, B = 10, 90, contract.BIG
    for M, K, m6 in [(no * nv * nv, nv, (nv * nv, 1, nv * no, B, 0, no)), (no * no * nv, nv, (nv, nv * nv, 1, B, 0, nv))]:
        rc = contract._split(fake, fake, fake, M, K, contract.padded_k(K, 0), contract._i64x6(m6), 0, None)
        assert rc == 4, L.last_error()
