"""Split-precision tcgen05 GEMM against FP64 references.

Tolerances (relative to the largest reference magnitude): split-BF16x3 keeps
about 16 significant bits per product (error ~2^-16); TF32x3 about 21 bits;
both accumulate in FP32.  The bars below are 1e-4 and 1e-5."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 1e-4, "tf32x3": 1e-5}


@pytest.fixture(scope="module")
def C():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import contract
    return contract


def einsum_reference(W, t3):
    """numpy FP64 restatement of the three W_vvvv.t3 einsums (distr_cc/rccsdt.py:421-427)."""
    r = np.zeros_like(t3)
    for q in range(t3.shape[0]):
        r[q] += np.einsum("abde,dec->abc", W, t3[q])
        r[q] += np.einsum("acde,dbe->abc", W, t3[q])
        r[q] += np.einsum("bcde,ade->abc", W, t3[q])
    return r


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.fixture(params=[256, 128])
def tile(request, C):
    """Run the test under 128 x 256 tiles (default pipeline) and 128 x 128 tiles (two CTAs per SM)."""
    from dcc import autotune
    old = autotune.get_config()
    autotune.set_config(*((64, 4, 16, 256) if request.param == 256 else (64, 2, 16, 128)))
    yield request.param
    autotune.set_config(*old)


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 500, 200), (1000, 257, 1000), (7, 9, 5)])
def test_matmul(C, kind, M, N, K):
    g = torch.Generator(device="cuda").manual_seed(M * N + K)
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
    got, st = C.matmul_split3(A, B, kind)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = A @ B.t()
    assert _rel(got, ref) < TOL[kind]


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("nblk,nv", [(3, 5), (4, 12), (2, 31)])
def test_wvvvv_t3_matches_einsum(C, kind, nblk, nv):
    rng = np.random.default_rng(nv)
    W = rng.standard_normal((nv,) * 4) * 0.1
    t3 = rng.standard_normal((nblk,) + (nv,) * 3) * 1e-3
    r0 = rng.standard_normal(t3.shape) * 1e-3
    want = r0 + einsum_reference(W, t3)
    dW, dt3 = torch.from_numpy(W).cuda(), torch.from_numpy(t3).cuda()
    r = torch.from_numpy(r0.copy()).cuda()
    op = C.WvvvvT3(nblk, nv, kind)
    op(r, dW, dt3)
    torch.cuda.synchronize()
    assert int(op.status.item()) == 0
    assert _rel(r - torch.from_numpy(r0).cuda(), torch.from_numpy(want - r0).cuda()) < TOL[kind]
    r64 = torch.from_numpy(r0.copy()).cuda()
    C.wvvvv_t3_fp64_(r64, dW, dt3)
    np.testing.assert_allclose(r64.cpu().numpy(), want, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("cfg", [(128, 2, 16), (64, 4, 16), (64, 3, 8), (32, 8, 32), (64, 4, 1), (64, 2, 16, 128),
                                 (64, 2, 1, 128)])
@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
def test_every_pipeline_shape(C, cfg, kind):
    from dcc import autotune
    old = autotune.get_config()
    try:
        autotune.set_config(*cfg)
        # K > 4096: the configurable pipeline (shorter K runs the fixed wide-epilogue one)
        g = torch.Generator(device="cuda").manual_seed(sum(cfg))
        A = torch.randn(300, 4500, dtype=torch.float64, device="cuda", generator=g)
        B = torch.randn(260, 4500, dtype=torch.float64, device="cuda", generator=g)
        got, st = C.matmul_split3(A, B, kind)
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        # FP32 accumulation over K = 4500 bounds both kinds near 3e-5 of the largest entry
        assert _rel(got, A @ B.t()) < 1e-4
    finally:
        autotune.set_config(*old)


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("transposed", [False, True])
def test_persistent_tiles_and_epilogue_orientation(C, kind, transposed, tile):
    """More output tiles than two rounds of CTAs (both TMEM accumulators reused
    several times); beta != 0; output written row-contiguous (lanes along
    columns) or column-contiguous (lanes along rows)."""
    M, N, K = 2000, 5000, 128
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
    k = C.KIND[kind]
    a = C.Split(M, K, k).fill(A, C.lin(K), C.lin(1))
    b = C.Split(N, K, k).fill(B, C.lin(K), C.lin(1))
    C0 = torch.randn(M * N, dtype=torch.float64, device="cuda", generator=g)
    out = C0.clone()
    fr, fc = (C.lin(1), C.lin(M)) if transposed else (C.lin(N), C.lin(1))
    st = C.gemm_(a, b, out, fr, fc, 0.5, -1.0)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    ref = 0.5 * (A @ B.t())
    got = (out.view(N, M).t() if transposed else out.view(M, N)) + (C0.view(N, M).t() if transposed else C0.view(M, N))
    assert _rel(got, ref) < TOL[kind]


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("transposed", [False, True])
@pytest.mark.parametrize("beta", [0.0, -1.0, 1.0])
def test_fp32_output(C, kind, transposed, beta, tile):
    """An FP32 C (the split path's S accumulator): with beta = 0 (C never read) or beta = -1 every
    element is the FP64 C's result for the same inputs rounded once to FP32 (the epilogue sums in
    FP64); with beta = 1 the epilogue adds fp32(alpha acc) by L2 reductions, within two FP32
    roundings of it.  Both epilogue orientations; a ragged M and N and K > 4096."""
    for M, N, K in ((2000, 5000, 128), (333, 517, 4200)):
        g = torch.Generator(device="cuda").manual_seed(M + N + K)
        A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
        B = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
        k = C.KIND[kind]
        a = C.Split(M, K, k).fill(A, C.lin(K), C.lin(1))
        b = C.Split(N, K, k).fill(B, C.lin(K), C.lin(1))
        C0 = torch.randn(M * N, dtype=torch.float64, device="cuda", generator=g).float()
        if beta == 0.0:
            C0.fill_(float("nan"))  # never read
        out32, out64 = C0.clone(), C0.double()
        fr, fc = (C.lin(1), C.lin(M)) if transposed else (C.lin(N), C.lin(1))
        st = C.gemm_(a, b, out32, fr, fc, 0.5, beta)
        C.gemm_(a, b, out64, fr, fc, 0.5, beta, st)
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        if beta == 1.0:
            scale = float(out64.abs().max())
            assert float((out32.double() - out64).abs().max()) <= 2.0 ** -22 * scale
        else:
            assert torch.equal(out32, out64.float())
        ref = 0.5 * (A @ B.t())
        got = out64.view(N, M).t() if transposed else out64.view(M, N)
        if beta != 0.0:
            got = got - beta * (C0.view(N, M).t() if transposed else C0.view(M, N)).double()
        # the FP32 accumulation error grows with K: the bar of the short cases, times 10 at K = 4200
        assert _rel(got, ref) < TOL[kind] * (1 if K <= 1024 else 10)


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
def test_concatenated_pieces_and_leading_columns(C, kind):
    """[A1 | A2] [B1 | B2]^T = A1 B1^T + A2 B2^T over a K-concatenated split, and a
    GEMM over the leading piece only (ldb > Kp) with an A that covers just that piece."""
    M, N, K1, K2 = 300, 700, 90, 50
    g = torch.Generator(device="cuda").manual_seed(6)
    A1 = torch.randn(M, K1, dtype=torch.float64, device="cuda", generator=g)
    A2t = torch.randn(K2, M, dtype=torch.float64, device="cuda", generator=g)  # stored k-major
    B1 = torch.randn(N, K1, dtype=torch.float64, device="cuda", generator=g)
    B2 = torch.randn(N, K2, dtype=torch.float64, device="cuda", generator=g)
    k = C.KIND[kind]
    a = C.Split(M, kind=k, pieces=[K1, K2])
    a.fill_piece(0, A1, C.lin(K1), C.lin(1)).fill_piece(1, A2t, C.lin(1), C.lin(M))
    b = C.Split(N, kind=k, pieces=[K1, K2])
    b.fill_piece(0, B1, C.lin(K1), C.lin(1)).fill_piece(1, B2, C.lin(K2), C.lin(1))
    out = torch.zeros(M, N, dtype=torch.float64, device="cuda")
    st = C.gemm_(a, b, out, C.lin(N), C.lin(1), 1.0, 0.0)
    ref = A1 @ B1.t() + A2t.t() @ B2.t()
    a1 = C.Split(M, K1, k).fill(A1, C.lin(K1), C.lin(1))
    out1 = torch.zeros(M, N, dtype=torch.float64, device="cuda")
    st1 = C.gemm_(a1, b, out1, C.lin(N), C.lin(1), 1.0, 0.0, Kp=a1.Kp)
    torch.cuda.synchronize()
    assert int(st.item()) == 0 and int(st1.item()) == 0
    assert _rel(out, ref) < TOL[kind]
    assert _rel(out1, A1 @ B1.t()) < TOL[kind]


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
def test_split_middle_digit_rows(C, kind):
    """Rows (p, x, y) whose contiguous source index is the middle digit x (the
    split's third read orientation) give the same GEMM as a plain transpose."""
    P, X, Yd, K = 6, 40, 7, 33
    g = torch.Generator(device="cuda").manual_seed(7)
    src = torch.randn(P, K, Yd, X, dtype=torch.float64, device="cuda", generator=g)  # [p][k][y][x]
    Bm = torch.randn(50, K, dtype=torch.float64, device="cuda", generator=g)
    k = C.KIND[kind]
    # row m = (p, x, y): p stride K*Yd*X, x stride 1, y stride X; k stride Yd*X
    a = C.Split(P * X * Yd, K, k).fill(src, C.three(X, Yd, K * Yd * X, 1, X), C.lin(Yd * X))
    b = C.Split(50, K, k).fill(Bm, C.lin(K), C.lin(1))
    out = torch.zeros(P * X * Yd, 50, dtype=torch.float64, device="cuda")
    st = C.gemm_(a, b, out, C.lin(50), C.lin(1), 1.0, 0.0)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    Am = src.permute(0, 3, 2, 1).reshape(P * X * Yd, K)
    assert _rel(out, Am @ Bm.t()) < TOL[kind]


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
def test_wvvvv_with_fvv_folded(C, kind):
    """W_vvvv.t3 + F_vv.t3 through the three GEMMs with F folded into W."""
    nblk, nv = 4, 12
    rng = np.random.default_rng(21)
    W = rng.standard_normal((nv,) * 4) * 0.1
    F = rng.standard_normal((nv, nv))
    t3 = rng.standard_normal((nblk,) + (nv,) * 3) * 1e-3
    e = np.einsum
    want = einsum_reference(W, t3) + e('ad,qdbc->qabc', F, t3) + e('bd,qadc->qabc', F, t3) + e('cd,qabd->qabc', F, t3)
    r = torch.zeros(t3.shape, dtype=torch.float64, device="cuda")
    op = C.WvvvvT3(nblk, nv, kind)
    op(r, torch.from_numpy(W).cuda(), torch.from_numpy(t3).cuda(), F=torch.from_numpy(F).cuda())
    torch.cuda.synchronize()
    assert int(op.status.item()) == 0
    assert _rel(r, torch.from_numpy(want).cuda()) < TOL[kind]


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("maps", ["k_contiguous", "rows_contiguous", "middle_digit"])
def test_split_of_fp32_source(C, kind, maps):
    """An FP32 source splits into the pieces of the same values as FP64, bit for bit, in each
    read mode (k contiguous, rows contiguous, rows along a middle digit)."""
    from dcc import contract as c
    k = c.KIND[kind]
    rng = np.random.default_rng(5)
    X32 = torch.from_numpy(rng.standard_normal((5, 3, 6, 40)).astype(np.float32)).cuda()  # [k][p][q][r]
    X64 = X32.double()
    if maps == "k_contiguous":       # rows (k,p,q), K = r
        M, K, fm, fk = 90, 40, c.lin(40), c.lin(1)
    elif maps == "rows_contiguous":  # rows (q,r), K = (k,p)
        M, K, fm, fk = 240, 15, c.lin(1), c.two(3, 720, 240)
    else:                            # rows (p,r,q): the contiguous r is the middle digit; K = k
        M, K, fm, fk = 720, 5, c.three(40, 6, 240, 1, 40), c.lin(720)
    s32 = c.Split(M, K, k).fill(X32, fm, fk)
    s64 = c.Split(M, K, k).fill(X64, fm, fk)
    assert torch.equal(s32.hi, s64.hi) and torch.equal(s32.lo, s64.lo)
