"""GPU parity of the bandwidth-bound T3/T4/(Q) kernels against the oracle.

Index work and the FP64 symmetrizers are compared bit for bit (numerical
equality, so +0 == -0): the kernels use the reference's operation order with
no FMA contraction.  Energy dot products use a relative tolerance of 1e-12
because the summation order differs from numpy's."""
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P3 = ["P3_full", "P3_422", "P3_201"]
P4 = ["P4_full", "P4_444", "P4_442", "P4_201"]


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


@pytest.fixture(scope="module")
def C():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import _c_rccsdt, _c_rccsdt_q, _c_rccsdtq
    return _c_rccsdt, _c_rccsdt_q, _c_rccsdtq


@pytest.mark.parametrize("nvir", [1, 2, 5, 8, 10, 13, 17, 18, 30, 50, 90])
@pytest.mark.parametrize("pattern", P3)
def test_t3_spin_sum(C, oracle, nvir, pattern):
    c3 = C[0]
    rng = np.random.default_rng(nvir)
    nblk = 2 if nvir == 90 else 5
    for alpha, beta in [(1.0, 0.0), (-1.0 / 6.0, 1.0)]:
        A = rng.standard_normal((nblk,) + (nvir,) * 3)
        want = oracle.t3_spin_sum(A.copy(), nvir, pattern, alpha, beta)
        d = dev(A)
        c3.t3_spin_summation_inplace_(d, nblk, nvir, pattern, alpha, beta)
        assert np.array_equal(host(d), want)
        d1 = dev(A[0])
        c3.t3_single_spin_summation_inplace_(d1, nvir, pattern, alpha, beta)
        assert np.array_equal(host(d1), want[0])
        # an 8-byte aligned view: the copy-engine kernel needs 16-byte alignment, the other path serves it
        buf = torch.zeros(A.size + 1, dtype=torch.float64, device="cuda")
        view = buf[1:].view(A.shape)
        view.copy_(dev(A))
        c3.t3_spin_summation_inplace_(view, nblk, nvir, pattern, alpha, beta)
        assert np.array_equal(host(view), want)
    assert c3.symmetrize_status() == 0


@pytest.mark.parametrize("nvir", [1, 2, 5, 10, 13, 30, 93, 104, 105])
@pytest.mark.parametrize("kernel", [1, 2])
def test_t3_spin_sum_kernels(C, oracle, nvir, kernel):
    """Each kernel of the out-of-place P3_201 (1 strips, 2 orbit tiles) bit-exact with the oracle
    where it applies; the strip kernel refuses larger nvir and the patterns with a p4 term and
    launches nothing."""
    c3 = C[0]
    rng = np.random.default_rng(200 + nvir)
    nblk = 2 if nvir >= 90 else 3
    applies = kernel == 2 or nvir <= 104
    for alpha, beta in [(1.0, 0.0), (-1.0 / 6.0, 1.0)]:
        A = rng.standard_normal((nblk,) + (nvir,) * 3)
        want = oracle.t3_spin_sum(A.copy(), nvir, "P3_201", alpha, beta)
        d, out = dev(A), torch.full(A.shape, float("nan"), dtype=torch.float64, device="cuda")
        if not applies:
            with pytest.raises(RuntimeError, match="does not apply"):
                c3.t3_spin_summation(d, out, nblk, nvir, "P3_201", alpha, beta, kernel=kernel)
            assert torch.isnan(out).all()
            continue
        c3.t3_spin_summation(d, out, nblk, nvir, "P3_201", alpha, beta, kernel=kernel)
        assert np.array_equal(host(out), want)
        assert np.array_equal(host(d), A)
    # the patterns with a p4 term run through the orbit kernel alone
    A = rng.standard_normal((nblk,) + (nvir,) * 3)
    d, out = dev(A), torch.empty(A.shape, dtype=torch.float64, device="cuda")
    if kernel == 2:
        c3.t3_spin_summation(d, out, nblk, nvir, "P3_422", 1.0, 0.0, kernel=kernel)
        assert np.array_equal(host(out), oracle.t3_spin_sum(A.copy(), nvir, "P3_422", 1.0, 0.0))
    else:
        with pytest.raises(RuntimeError, match="does not apply"):
            c3.t3_spin_summation(d, out, nblk, nvir, "P3_422", 1.0, 0.0, kernel=kernel)
    assert c3.symmetrize_status() == 0


@pytest.mark.parametrize("nvir", [1, 2, 5, 13, 30, 93, 104])
def test_t3_spin_sum_f32(C, oracle, nvir):
    """The FP32 P3_201 (X of the split precisions): FP64 arithmetic on the FP32 values, rounded
    once, so bit-exact with the oracle on the same values cast to FP64, the result cast back;
    A untouched; other patterns and larger nvir refused."""
    c3 = C[0]
    rng = np.random.default_rng(300 + nvir)
    nblk = 2 if nvir >= 90 else 3
    for alpha, beta in [(1.0, 0.0), (-1.0 / 6.0, 1.0)]:
        A = rng.standard_normal((nblk,) + (nvir,) * 3).astype(np.float32)
        want = oracle.t3_spin_sum(A.astype(np.float64), nvir, "P3_201", alpha, beta).astype(np.float32)
        d, out = dev(A), torch.full(A.shape, float("nan"), dtype=torch.float32, device="cuda")
        c3.t3_spin_summation_f32(d, out, nblk, nvir, "P3_201", alpha, beta)
        assert np.array_equal(host(out), want)
        assert np.array_equal(host(d), A)
    with pytest.raises(RuntimeError, match="p4 term"):
        c3.t3_spin_summation_f32(d, out, nblk, nvir, "P3_422")
    big = torch.zeros((1,) + (105,) * 3, dtype=torch.float32, device="cuda")
    with pytest.raises(RuntimeError, match="p4 term"):
        c3.t3_spin_summation_f32(big, big.clone(), 1, 105, "P3_201")


@pytest.mark.parametrize("nocc,nvir", [(1, 5), (2, 13), (3, 17), (2, 93), (2, 104)])
def test_unpack_all_f32(C, nocc, nvir):
    """The FP32 unpack equals the FP64 unpack rounded to FP32, element for element."""
    from dcc import t3_residual
    rng = np.random.default_rng(17)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = dev(rng.standard_normal((n3,) + (nvir,) * 3))
    shape = (nocc ** 3,) + (nvir,) * 3
    U64 = torch.empty(shape, dtype=torch.float64, device="cuda")
    U32 = torch.full(shape, 7.0, dtype=torch.float32, device="cuda")
    t3_residual.unpack_all_(t3, U64, nocc, nvir)
    t3_residual.unpack_all_(t3, U32, nocc, nvir)
    assert torch.equal(U32, U64.float())
    with pytest.raises(RuntimeError, match="nvir <= 104"):
        t3_residual.unpack_all_(torch.zeros((1,) + (105,) * 3, dtype=torch.float64, device="cuda"),
                                torch.empty((1,) + (105,) * 3, dtype=torch.float32, device="cuda"), 1, 105)
    assert C[0].symmetrize_status() == 0


@pytest.mark.parametrize("nvir", [1, 5, 10, 13, 30, 90, 93, 106])
@pytest.mark.parametrize("pattern", P3)
def test_t3_spin_sum_out_of_place(C, oracle, nvir, pattern):
    """B = beta*A + alpha*P(A) out of place (the library's choice of kernel: strips for P3_201 up
    to nvir = 104, orbit tiles otherwise): bit-exact with the oracle, and A untouched."""
    c3 = C[0]
    rng = np.random.default_rng(100 + nvir)
    nblk = 2 if nvir >= 90 else 4
    for alpha, beta in [(1.0, 0.0), (-1.0 / 6.0, 1.0)]:
        A = rng.standard_normal((nblk,) + (nvir,) * 3)
        want = oracle.t3_spin_sum(A.copy(), nvir, pattern, alpha, beta)
        d, out = dev(A), torch.full(A.shape, float("nan"), dtype=torch.float64, device="cuda")
        c3.t3_spin_summation(d, out, nblk, nvir, pattern, alpha, beta)
        assert np.array_equal(host(out), want)
        assert np.array_equal(host(d), A)
    assert c3.symmetrize_status() == 0


@pytest.mark.parametrize("nocc,nvir", [(1, 5), (2, 1), (3, 8), (4, 13), (3, 17), (2, 93)])
@pytest.mark.parametrize("pattern", P3)
def test_t3_unpack_p3(C, oracle, nocc, nvir, pattern):
    """U and X = beta U + alpha P(U) of every ordering in one pass (dcc_t3_unpack_p3): U equal to
    the unpack of every ordering, X bit-exact with the oracle's P3 over it (the same values as a
    P3 pass over U), with and without U, t3 untouched."""
    from dcc import t3_residual
    c3 = C[0]
    rng = np.random.default_rng(7 * nocc + nvir)
    trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
    full = rng.standard_normal((nocc,) * 3 + (nvir,) * 3)
    import itertools
    full = sum(full.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3))) / 6
    t3 = np.stack([full[i, j, k] for i, j, k in trip])
    d = dev(t3)
    Uw = torch.empty((nocc ** 3,) + (nvir,) * 3, dtype=torch.float64, device="cuda")
    t3_residual.unpack_all_(d, Uw, nocc, nvir)
    for alpha, beta in [(1.0, 0.0), (-1.0 / 6.0, 1.0)]:
        want = oracle.t3_spin_sum(host(Uw).copy(), nvir, pattern, alpha, beta)
        U = torch.full_like(Uw, float("nan"))
        X = torch.full_like(Uw, float("nan"))
        c3.t3_unpack_p3(d, U, X, nocc, nvir, pattern, alpha, beta)
        assert torch.equal(U, Uw)
        assert np.array_equal(host(X), want)
        X2 = torch.full_like(Uw, float("nan"))
        c3.t3_unpack_p3(d, None, X2, nocc, nvir, pattern, alpha, beta)
        assert torch.equal(X2, X)
    assert np.array_equal(host(d), t3)


@pytest.mark.parametrize("nvir", [2, 10, 30, 90])
def test_orbit_roundtrip_is_identity(C, nvir):
    """The diagnostic tile round trip of the spin-summation kernel leaves every block unchanged."""
    c3 = C[0]
    A = np.random.default_rng(nvir).standard_normal((3,) + (nvir,) * 3)
    d = dev(A)
    c3.t3_orbit_roundtrip_(d, 3, nvir)
    assert np.array_equal(host(d), A)
    assert c3.symmetrize_status() == 0


@pytest.mark.parametrize("nvir", [1, 2, 3, 8, 10, 11, 18, 30, 50, 90])
@pytest.mark.parametrize("aligned", [True, False])
def test_triple_sym_transpose_add(C, oracle, nvir, aligned):
    """Even nvir with 16-byte aligned buffers run the TMA orbit-tile kernel, the rest the cp.async one."""
    c3 = C[0]
    rng = np.random.default_rng(1)
    nblk = 2 if nvir == 90 else 3
    A = rng.standard_normal((nblk,) + (nvir,) * 3)

    def buf():
        if aligned:
            return torch.empty(A.shape, dtype=torch.float64, device="cuda")
        return torch.empty(A.size + 1, dtype=torch.float64, device="cuda")[1:].view(A.shape)

    dA = buf()
    dA.copy_(dev(A))
    B = [buf() for _ in range(3)]
    c3.t3_spin_summation_triple_sym_(dA, *B, nvir)
    T = buf()
    c3.t3_transpose_add_(dA, T, nvir)
    for b in range(nblk):
        want = oracle.t3_triple_sym(np.ascontiguousarray(A[b]), nvir)
        for m in range(3):
            assert np.array_equal(host(B[m])[b], want[m])
        assert np.array_equal(host(T)[b], oracle.t3_transpose_add(np.ascontiguousarray(A[b]), nvir))
    assert np.array_equal(host(dA), A)
    assert c3.symmetrize_status() == 0


@pytest.mark.parametrize("nocc,nvir", [(1, 3), (3, 5), (4, 9), (3, 17)])
def test_take_t3(C, oracle, nocc, nvir):
    c3 = C[0]
    rng = np.random.default_rng(2)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = rng.standard_normal((n3,) + (nvir,) * 3)
    loc = np.arange(n3, dtype=np.int64)
    loc[n3 // 2] = -1  # one block not stored
    trip = list(itertools.product(range(nocc), repeat=3))
    dt3 = dev(t3)
    out = torch.empty((len(trip),) + (nvir,) * 3, dtype=torch.float64, device="cuda")
    c3.take_t3_batched(dt3, out, dev(np.array(trip, dtype=np.int32)), dev(loc), nocc, nvir)
    got = host(out)
    from dcc._lib import DccError
    for q, (i, j, k) in enumerate(trip):
        want, rc = oracle.take_t3(t3, loc, i, j, k, nocc, nvir)
        if rc:
            assert not got[q].any()
            with pytest.raises(DccError):
                c3.take_t3_ijk_single_(dt3, torch.empty(nvir ** 3, dtype=torch.float64, device="cuda"), loc, i, j, k,
                                       nocc, nvir)
            continue
        assert np.array_equal(got[q], want)
        one = torch.empty((nvir,) * 3, dtype=torch.float64, device="cuda")
        c3.take_t3_ijk_single_(dt3, one, loc, i, j, k, nocc, nvir)
        assert np.array_equal(host(one), want)


def test_fill_local_data_ijk(C, oracle):
    c3 = C[0]
    rng = np.random.default_rng(3)
    t3 = rng.standard_normal((10, 6, 6, 6))
    loc = np.arange(10, dtype=np.int64)
    loc[4] = -1
    req = np.array([7, 0, 4, 9, 3], dtype=np.int32)
    want = oracle.gather_t3(t3, req, loc, 6)
    out = torch.zeros((5, 6, 6, 6), dtype=torch.float64, device="cuda")
    c3.fill_local_data_ijk_(dev(t3), out, dev(req), dev(loc), 5, 6)
    assert np.array_equal(host(out), want)


@pytest.mark.parametrize("nocc,nvir,nact", [(3, 7, 7), (4, 13, 9), (10, 90, 60)])
def test_divide_update(C, oracle, nocc, nvir, nact):
    c3 = C[0]
    rng = np.random.default_rng(4)
    trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
    if nvir == 90:
        trip = trip[::37]
    ijk = np.array(trip, dtype=np.int32)
    r3 = rng.standard_normal((len(trip),) + (nvir,) * 3)
    t3 = rng.standard_normal(r3.shape)
    eo, ev = rng.uniform(-1.5, -0.3, nocc), rng.uniform(0.1, 3.0, nvir)
    eia = np.ascontiguousarray(eo[:, None] - ev[None, :])
    want_r = oracle.r3_divide(r3.copy(), eia, ijk)
    d_r = dev(r3)
    c3.r3_tri_divide_e_(d_r, dev(eia), dev(ijk))
    assert np.array_equal(host(d_r), want_r)
    d_r, d_t = dev(r3), dev(t3)
    norms = c3.t3_divide_update_(d_t, d_r, dev(eia), dev(ijk), nvir_active=nact, write_r3=True)
    assert np.array_equal(host(d_r), want_r)
    assert np.array_equal(host(d_t), t3 + want_r)
    n = host(norms)
    np.testing.assert_allclose(n[0], np.sum(want_r ** 2), rtol=1e-12)
    np.testing.assert_allclose(n[1], np.sum(want_r[:, :nact, :nact, :nact] ** 2), rtol=1e-12)


def _symmetric_t3(nocc, nvir, rng):
    """Canonical blocks of a T3 with the physical simultaneous-permutation symmetry."""
    full = rng.standard_normal((nocc,) * 3 + (nvir,) * 3)
    sym = sum(full.transpose(p + tuple(3 + q for q in p)) for p in itertools.permutations(range(3))) / 6
    return np.stack([sym[i, j, k] for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)])


@pytest.mark.parametrize("nocc,nvir", [(1, 3), (3, 4), (4, 7), (5, 10)])
def test_ijk_to_abc(C, oracle, nocc, nvir):
    c3 = C[0]
    rng = np.random.default_rng(5)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    for t3 in (rng.standard_normal((n3,) + (nvir,) * 3), _symmetric_t3(nocc, nvir, rng)):
        want = oracle.ijk_to_abc(np.ascontiguousarray(t3), nocc, nvir)
        assert np.array_equal(host(c3.redistribute_ijk_to_abc(dev(t3), nocc, nvir)), want)


@pytest.mark.parametrize("nocc,nvir,blk", [(2, 5, 2), (3, 10, 4), (4, 9, 4)])
def test_fill_t3_from_abc(C, oracle, nocc, nvir, blk):
    cq = C[1]
    rng = np.random.default_rng(6)
    nabc = nvir * (nvir + 1) * (nvir + 2) // 6
    t3_abc = rng.standard_normal((nabc, nocc, nocc, nocc))
    d_abc = dev(t3_abc)
    for a0 in range(0, nvir, blk):
        for b0 in range(0, nvir, blk):
            a1, b1 = min(a0 + blk, nvir), min(b0 + blk, nvir)
            want = np.zeros((blk, blk, nvir, nocc, nocc, nocc))
            oracle.fill_t3_abc(want, a0, a1, b0, b1, nvir, nocc, t3_abc, None, blk)
            got = torch.zeros(want.shape, dtype=torch.float64, device="cuda")
            cq.fill_t3_from_abc(got, a0, a1, b0, b1, nvir, nocc, d_abc, blk)
            assert np.array_equal(host(got), want)


@pytest.mark.parametrize("nvir", [1, 2, 5, 11])
def test_t4_project(C, oracle, nvir):
    c4 = C[2]
    rng = np.random.default_rng(7)
    A = rng.standard_normal((3,) + (nvir,) * 4)
    for alpha, beta in [(1.0, 0.0), (-1.0, 1.0)]:
        want = oracle.t4_project(A.copy(), 3, nvir, alpha, beta)
        d = dev(A)
        c4.t4_project_1_minus_p4_p31_inplace_(d, 3, nvir, alpha, beta)
        assert np.array_equal(host(d), want)


@pytest.mark.parametrize("n", [1, 3, 6, 10])
@pytest.mark.parametrize("pattern", P4)
def test_t4_spin_sum(C, oracle, n, pattern):
    cq, c4 = C[1], C[2]
    rng = np.random.default_rng(8)
    A = rng.standard_normal((4,) + (n,) * 4)
    want = oracle.t4_spin_sum(A.copy(), 4, n, pattern, 0.5, 1.0)
    d = dev(A)
    cq.t4_spin_summation_inplace_(d, 4, n, pattern, 0.5, 1.0)
    assert np.array_equal(host(d), want)
    if pattern != "P4_444":
        d1 = dev(A[0])
        c4.t4_single_spin_summation_inplace_(d1, n, pattern, 0.5, 1.0)
        assert np.array_equal(host(d1), want[0])


@pytest.mark.parametrize("nvir", [1, 4, 11])
def test_t4_elementwise(C, oracle, nvir):
    c4 = C[2]
    rng = np.random.default_rng(9)
    A = rng.standard_normal((nvir,) * 4)
    dA = dev(A)
    D = torch.empty_like(dA)
    c4.t4_transpose_add_(dA, D, nvir)
    assert np.array_equal(host(D), oracle.t4_transpose_add(A, nvir))
    B = [torch.empty_like(dA) for _ in range(4)]
    c4.t4_spin_summation_quadruple_sym_(dA, *B, nvir)
    for m, w in enumerate(oracle.t4_quadruple_sym(A, nvir)):
        assert np.array_equal(host(B[m]), w)
    R = rng.standard_normal((nvir,) * 4)
    dT = dev(A)
    c4.t4_add_(dT, dev(R), 1, nvir)
    assert np.array_equal(host(dT), A + R)


@pytest.mark.parametrize("nblk,nvir", [(1, 3), (7, 11), (161, 11), (3, 20)])
def test_t4_forms_batched(C, oracle, nblk, nvir):
    """All blocks' transpose-add and quadruple-sym forms in one launch each: bit-identical
    to the oracle applied block by block."""
    c4 = C[2]
    rng = np.random.default_rng(nblk + nvir)
    A = rng.standard_normal((nblk,) + (nvir,) * 4)
    T3, V = c4.t4_forms_batched(dev(A).view(nblk, -1), nvir)
    T3, V = host(T3).reshape(A.shape), [host(v).reshape(A.shape) for v in V]
    for q in range(nblk):
        assert np.array_equal(T3[q], oracle.t4_transpose_add(A[q], nvir))
        for m, w in enumerate(oracle.t4_quadruple_sym(A[q], nvir)):
            assert np.array_equal(V[m][q], w)


def test_r4_divide_unpack_gather(C, oracle):
    c4 = C[2]
    rng = np.random.default_rng(10)
    nocc, nvir = 4, 5
    stored = [(i, j, k, l) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)
              for l in range(k, nocc) if not ((i == j == k) or (j == k == l))]
    nfull = nocc * (nocc + 1) * (nocc + 2) * (nocc + 3) // 24
    f2l = np.full(nfull, -1, dtype=np.int64)
    for q, t in enumerate(stored):
        f2l[oracle.ijkl_to_linear(*t, nocc)] = q
    r4 = rng.standard_normal((len(stored),) + (nvir,) * 4)
    eia = rng.uniform(-3, -0.5, (nocc, nvir))
    ijkl = np.array(stored, dtype=np.int32)
    d = dev(r4)
    c4.r4_local_tri_divide(d, dev(eia), dev(ijkl))
    assert np.array_equal(host(d), oracle.r4_divide(r4.copy(), eia, ijkl))
    d_t4 = dev(r4)
    for i, j, k, l in itertools.product(range(nocc), repeat=4):
        want, rc = oracle.unpack_t4(r4, f2l, i, j, k, l, nocc, nvir)
        assert rc == 0
        out = torch.full((nvir,) * 4, 7.0, dtype=torch.float64, device="cuda")
        c4.unpack_t4_ijkl_single_(d_t4, out, f2l, i, j, k, l, nocc, nvir)
        assert np.array_equal(host(out), want)
    req = np.array([3, 0, 17], dtype=np.int32)
    send = torch.zeros((3,) + (nvir,) * 4, dtype=torch.float64, device="cuda")
    c4.fill_local_data_ijkl_(d_t4, send, dev(req), dev(f2l), 3, nvir)
    want = np.stack([r4[f2l[r]] if f2l[r] >= 0 else np.zeros((nvir,) * 4) for r in req])
    assert np.array_equal(host(send), want)


def _q_task_reference(oracle, t4, z4, vvoo, t2, eo, ev, task, blk, nocc):
    """The reference's per-task sequence on the oracle (distr_cc/rccsdt_q.py:1131-1154)."""
    a0, a1, b0, b1, c0, c1, d0, d1 = task
    t = t4 + z4
    oracle.e_abcdijkl_division(t, eo, ev, a0, a1, b0, b1, c0, c1, d0, d1, blk, blk, blk, nocc)
    oracle.t4_spin_sum(t, blk ** 4, nocc, "P4_444", 1.0, 0.0)
    factor = np.zeros((blk,) * 4)
    for ia, ib, ic, id_ in itertools.product(range(blk), repeat=4):
        if ia < a1 - a0 and ib < b1 - b0 and ic < c1 - c0 and id_ < d1 - d0:
            factor[ia, ib, ic, id_] = oracle.q_factor(a0 + ia, b0 + ib, c0 + ic, d0 + id_)
    oracle.t4_multiply_factor(t, factor, blk, blk, blk, blk, nocc)
    paren = np.dot(t.ravel(), z4.ravel()) / 12.0
    zsq = np.zeros_like(z4)
    sl = lambda x0, x1, y0, y1: np.s_[x0:x1, y0:y1]  # noqa: E731
    ba, bb, bc, bd = a1 - a0, b1 - b0, c1 - c0, d1 - d0
    zsq[:ba, :bb, :bc, :bd] = (
        np.einsum("abij,cdkl->abcdijkl", vvoo[sl(a0, a1, b0, b1)], t2[sl(c0, c1, d0, d1)])
        + np.einsum("acik,bdjl->abcdijkl", vvoo[sl(a0, a1, c0, c1)], t2[sl(b0, b1, d0, d1)])
        + np.einsum("adil,bcjk->abcdijkl", vvoo[sl(a0, a1, d0, d1)], t2[sl(b0, b1, c0, c1)])
        + np.einsum("bcjk,adil->abcdijkl", vvoo[sl(b0, b1, c0, c1)], t2[sl(a0, a1, d0, d1)])
        + np.einsum("bdjl,acik->abcdijkl", vvoo[sl(b0, b1, d0, d1)], t2[sl(a0, a1, c0, c1)])
        + np.einsum("cdkl,abij->abcdijkl", vvoo[sl(c0, c1, d0, d1)], t2[sl(a0, a1, b0, b1)]))
    bracket = np.dot(t.ravel(), zsq.ravel()) / 12.0
    return bracket, paren + bracket


@pytest.mark.parametrize("nocc,nvir,blk", [(3, 7, 3), (4, 9, 4)])
def test_q_epilogue(C, oracle, nocc, nvir, blk):
    cq = C[1]
    rng = np.random.default_rng(11)
    eo, ev = rng.uniform(-1.5, -0.3, nocc), rng.uniform(0.1, 3.0, nvir)
    vvoo = rng.standard_normal((nvir, nvir, nocc, nocc)) * 0.1
    t2 = rng.standard_normal((nvir, nvir, nocc, nocc)) * 0.01
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    tot = np.zeros(2)
    d_args = [dev(vvoo), dev(t2), dev(eo), dev(ev)]
    tasks = []
    for d0 in range(0, nvir, blk):
        for c0 in range(0, d0 + 1, blk):
            for b0 in range(0, c0 + 1, blk):
                for a0 in range(0, b0 + 1, blk):
                    tasks.append((a0, min(a0 + blk, nvir), b0, min(b0 + blk, nvir), c0, min(c0 + blk, nvir),
                                  d0, min(d0 + blk, nvir)))
    for task in tasks[:12]:
        t4 = rng.standard_normal((blk,) * 4 + (nocc,) * 4) * 1e-3
        z4 = rng.standard_normal(t4.shape) * 1e-3
        br, pa = _q_task_reference(oracle, t4, z4, vvoo, t2, eo, ev, task, blk, nocc)
        tot += [br, pa]
        cq.q_task_epilogue(dev(t4), dev(z4), *d_args, task, blk, nocc, nvir, out)
    np.testing.assert_allclose(host(out), tot, rtol=1e-12, atol=1e-300)


def test_q_division_and_factor(C, oracle):
    cq = C[1]
    rng = np.random.default_rng(12)
    nocc, nvir, blk = 3, 8, 3
    eo, ev = rng.uniform(-1.5, -0.3, nocc), rng.uniform(0.1, 3.0, nvir)
    r4 = rng.standard_normal((blk,) * 4 + (nocc,) * 4)
    task = (0, 3, 3, 6, 6, 8, 6, 8)
    want = oracle.e_abcdijkl_division(r4.copy(), eo, ev, *task, blk, blk, blk, nocc)
    d = dev(r4)
    cq.e_abcdijkl_division_(d, dev(eo), dev(ev), *task, blk, blk, blk, blk, nocc)
    assert np.array_equal(host(d), want)
    factor = rng.choice([0.0, 6.0, 12.0, 24.0], size=(blk,) * 4)
    want2 = oracle.t4_multiply_factor(want.copy(), factor, blk, blk, blk, blk, nocc)
    cq.t4_multiply_factor_(d, dev(factor), blk, blk, blk, blk, nocc)
    assert np.array_equal(host(d), want2)


@pytest.mark.parametrize("nocc,nvir,aligned", [(1, 3, True), (3, 5, True), (4, 9, True), (3, 17, True), (2, 4, True),
                                               (3, 10, True), (4, 18, True), (1, 2, True), (5, 8, True), (2, 90, True),
                                               (3, 10, False), (2, 93, True), (3, 25, False), (1, 106, True),
                                               (2, 112, True), (1, 105, True)])
def test_unpack_all(C, oracle, nocc, nvir, aligned):
    """nvir <= 104 runs the row kernel with staged column tiles; above it even nvir with 16-byte
    aligned buffers the row-band TMA kernel, the rest the orbit-tile kernel."""
    from dcc import t3_residual
    rng = np.random.default_rng(13)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    t3 = rng.standard_normal((n3,) + (nvir,) * 3)
    loc = np.arange(n3, dtype=np.int64)
    shape = (nocc ** 3,) + (nvir,) * 3
    if aligned:
        U = torch.full(shape, 7.0, dtype=torch.float64, device="cuda")
    else:
        U = torch.full((int(np.prod(shape)) + 1,), 7.0, dtype=torch.float64, device="cuda")[1:].view(shape)
    t3_residual.unpack_all_(dev(t3), U, nocc, nvir)
    got = host(U)
    for q, (i, j, k) in enumerate(itertools.product(range(nocc), repeat=3)):
        want, rc = oracle.take_t3(t3, loc, i, j, k, nocc, nvir)
        assert rc == 0 and np.array_equal(got[q], want)
    assert C[0].symmetrize_status() == 0
