"""Grouped split, grouped GEMM and the (Q) group epilogue on the GPU.

* grouped split: bit-exact against one dcc_split_operand_at4 call per operand
  (float64 sources) and against the float64 copy of a float32 source;
* grouped GEMM: problems sharing an output, against FP64 torch (split
  tolerance 1e-4 bf16x3 / 1e-5 tf32x3, relative to the largest magnitude);
* group epilogue: the sum of the per-task oracle sequence over the tasks of a
  group (relative 1e-12 for float64 blocks, 1e-6 for float32 blocks)."""
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from test_gpu_kernels import _q_task_reference  # noqa: E402

TOL = {"bf16x3": 1e-4, "tf32x3": 1e-5}


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import contract, _c_rccsdt_q
    return contract, _c_rccsdt_q


def _split_row(c, S, K, fm, fk, f32):
    return [S.hi.data_ptr(), S.lo.data_ptr(), S.M, K, S.pieces[0][2], S.Kp, 0] + list(c.as4(fm)) + list(c.as4(fk)) + \
        [int(f32)]


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
def test_grouped_split_bit_exact(mods, kind):
    c, _ = mods
    k = c.KIND[kind]
    g = torch.Generator(device="cuda").manual_seed(5)
    X = torch.randn(6, 7, 9, 11, dtype=torch.float64, device="cuda", generator=g)
    # (rows, K, row map, k map) cases covering the four read modes
    cases = [(6 * 7, 9 * 11, c.two(7, 7 * 99, 99), c.lin(1)),          # k contiguous
             (9 * 11, 6 * 7, c.lin(1), c.two(7, 7 * 99, 99)),          # rows contiguous
             (6 * 9 * 11, 7, c.three(9, 11, 7 * 99, 11, 1), c.lin(99)),  # rows contiguous, k strided
             (7 * 11, 6 * 9, c.two(11, 99, 1), c.two(9, 7 * 99, 11)),
             (6 * 11 * 7, 9, c.three(11, 7, 7 * 99, 1, 99), c.lin(11))]  # short contiguous middle digit
    rows, refs, srcs = [], [], []
    for M, K, fm, fk in cases:
        S = c.Split(M, K, k, "cuda")
        R = c.Split(M, K, k, "cuda")
        R.fill(X, fm, fk)
        rows.append(_split_row(c, S, K, fm, fk, False))
        refs.append((S, R))
        srcs.append(X.data_ptr())
    X32 = X.float()
    S = c.Split(6 * 7, 9 * 11, k, "cuda")
    R = c.Split(6 * 7, 9 * 11, k, "cuda")
    R.fill(X32.double(), cases[0][2], cases[0][3])
    rows.append(_split_row(c, S, 9 * 11, cases[0][2], cases[0][3], True))
    refs.append((S, R))
    srcs.append(X32.data_ptr())
    gs = c.GroupedSplit(np.array(rows, dtype=np.int64), k, "cuda")
    gs.run(srcs)
    torch.cuda.synchronize()
    for S, R in refs:
        assert torch.equal(S.hi, R.hi) and torch.equal(S.lo, R.lo)


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("out_f32", [True, False])
def test_grouped_gemm_shared_output(mods, kind, out_f32):
    c, _ = mods
    k = c.KIND[kind]
    g = torch.Generator(device="cuda").manual_seed(7)
    M, N = 300, 270
    dt = torch.float32 if out_f32 else torch.float64
    Cout = torch.zeros(M, N, dtype=dt, device="cuda")
    ref = torch.zeros(M, N, dtype=torch.float64, device="cuda")
    rows, alphas, keep = [], [], []
    for i, (K, alpha, trans) in enumerate([(64, 1.0, False), (90, -0.5, True), (10, 2.0, False), (300, 1.0, True)]):
        A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
        B = torch.randn(N, K, dtype=torch.float64, device="cuda", generator=g)
        a = c.Split(M, K, k, "cuda").fill(A, c.lin(K), c.lin(1))
        b = c.Split(N, K, k, "cuda").fill(B, c.lin(K), c.lin(1))
        keep += [a, b]
        if trans:  # rows of B index the output's rows: C^T += alpha B A^T
            rows.append([b.hi.data_ptr(), b.lo.data_ptr(), b.Kp, a.hi.data_ptr(), a.lo.data_ptr(), a.Kp, N, M, a.Kp,
                         Cout.data_ptr(), int(out_f32)] + list(c.as4(c.lin(1))) + list(c.as4(c.lin(N))))
        else:
            rows.append([a.hi.data_ptr(), a.lo.data_ptr(), a.Kp, b.hi.data_ptr(), b.lo.data_ptr(), b.Kp, M, N, a.Kp,
                         Cout.data_ptr(), int(out_f32)] + list(c.as4(c.lin(N))) + list(c.as4(c.lin(1))))
        alphas.append(alpha)
        ref += alpha * (A @ B.t())
    gg = c.GroupedGemm(np.array(rows, dtype=np.int64), np.array(alphas), k, "cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    gg.run(status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    rel = float((Cout.double() - ref).abs().max() / ref.abs().max())
    assert rel < TOL[kind] + (1e-6 if out_f32 else 0.0)


def _group_blocks(rng, no, V, dtype):
    t4 = rng.standard_normal((no,) * 4 + (V,)) * 1e-3
    z4 = rng.standard_normal(t4.shape) * 1e-3
    if dtype == np.float32:
        t4, z4 = t4.astype(np.float32).astype(np.float64), z4.astype(np.float32).astype(np.float64)
    return t4, z4


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("nocc,nvir,blk,gi", [(3, 7, 3, 2), (4, 9, 4, 4), (2, 6, 2, 7)])
def test_q_group_epilogue(mods, oracle, f32, nocc, nvir, blk, gi):
    from dcc import rccsdt_q as gq
    _, cq = mods
    rng = np.random.default_rng(13 + gi)
    eo, ev = rng.uniform(-1.5, -0.3, nocc), rng.uniform(0.1, 3.0, nvir)
    vvoo = rng.standard_normal((nvir, nvir, nocc, nocc)) * 0.1
    t2 = rng.standard_normal((nvir, nvir, nocc, nocc)) * 0.01
    a0, a1, b0, b1, c0, c1 = gq.groups(nvir, blk)[gi]
    ba, bb, bc, dn = a1 - a0, b1 - b0, c1 - c0, nvir - c0
    t4g, z4g = _group_blocks(rng, nocc, ba * bb * bc * dn, np.float32 if f32 else np.float64)
    tot = np.zeros(2)
    G4 = lambda x: x.reshape((nocc,) * 4 + (ba, bb, bc, dn)).transpose(4, 5, 6, 7, 0, 1, 2, 3)  # noqa: E731
    for d0, d1 in gq.prange(c0, nvir, blk):
        t4 = np.zeros((blk,) * 4 + (nocc,) * 4)
        z4 = np.zeros_like(t4)
        t4[:ba, :bb, :bc, :d1 - d0] = G4(t4g)[..., d0 - c0:d1 - c0, :, :, :, :]
        z4[:ba, :bb, :bc, :d1 - d0] = G4(z4g)[..., d0 - c0:d1 - c0, :, :, :, :]
        tot += _q_task_reference(oracle, t4, z4, vvoo, t2, eo, ev, (a0, a1, b0, b1, c0, c1, d0, d1), blk, nocc)
    tt = torch.float32 if f32 else torch.float64
    dev = lambda a, t=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", t)  # noqa: E731
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    cq.q_group_epilogue(dev(t4g, tt), dev(z4g, tt), dev(vvoo.transpose(0, 2, 3, 1)), dev(t2.transpose(0, 2, 3, 1)),
                        dev(eo), dev(ev), (a0, a1, b0, b1, c0, c1, c0, nvir), nocc, nvir, out)
    np.testing.assert_allclose(out.cpu().numpy(), tot, rtol=1e-11, atol=1e-300)


@pytest.mark.parametrize("kind", ["bf16x3", "tf32x3"])
@pytest.mark.parametrize("K", [6, 10, 90])
def test_grouped_compact_k(mods, kind, K):
    """Operands stored with only their K columns (pitch K rounded up to 8, below the
    padded Kp): the grouped split writes them and the GEMM reads zeros past the pitch."""
    c, _ = mods
    k = c.KIND[kind]
    g = torch.Generator(device="cuda").manual_seed(K)
    M, N = 200, 300
    k8, kp = (K + 7) // 8 * 8, c.padded_k(K, k)
    dt = torch.bfloat16 if k == 0 else torch.float32
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(K, N, dtype=torch.float64, device="cuda", generator=g)  # K-major source for B: strided rows
    bufs = [torch.full((r, k8), float("nan"), dtype=dt, device="cuda") for r in (M, M, N, N)]
    spec = [[bufs[0].data_ptr(), bufs[1].data_ptr(), M, K, k8, k8, 0] + list(c.as4(c.lin(K))) + list(c.as4(c.lin(1))) + [0],
            [bufs[2].data_ptr(), bufs[3].data_ptr(), N, K, k8, k8, 0] + list(c.as4(c.lin(1))) + list(c.as4(c.lin(N))) + [0]]
    gs = c.GroupedSplit(np.array(spec, dtype=np.int64), k, "cuda")
    gs.run([A.data_ptr(), B.data_ptr()])
    out = torch.zeros(M, N, dtype=torch.float32, device="cuda")
    row = [bufs[0].data_ptr(), bufs[1].data_ptr(), k8, bufs[2].data_ptr(), bufs[3].data_ptr(), k8, M, N, kp,
           out.data_ptr(), 1] + list(c.as4(c.lin(N))) + list(c.as4(c.lin(1)))
    gg = c.GroupedGemm(np.array([row], dtype=np.int64), np.array([1.0]), k, "cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    gg.run(status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert not torch.isnan(bufs[0]).any() and not torch.isnan(bufs[2]).any()
    ref = A @ B
    rel = float((out.double() - ref).abs().max() / ref.abs().max())
    assert rel < TOL[kind] + 1e-6
