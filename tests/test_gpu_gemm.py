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


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


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
    want = r0 + C.einsum_reference(W, t3)
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


@pytest.mark.parametrize("cfg", [(128, 2, 16), (64, 4, 16), (64, 3, 8), (32, 8, 32), (64, 4, 1)])
@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
def test_every_pipeline_shape(C, cfg, kind):
    from dcc import autotune
    old = autotune.get_config()
    try:
        autotune.set_config(*cfg)
        g = torch.Generator(device="cuda").manual_seed(sum(cfg))
        A = torch.randn(700, 300, dtype=torch.float64, device="cuda", generator=g)
        B = torch.randn(600, 300, dtype=torch.float64, device="cuda", generator=g)
        got, st = C.matmul_split3(A, B, kind)
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        assert _rel(got, A @ B.t()) < TOL[kind]
    finally:
        autotune.set_config(*old)
