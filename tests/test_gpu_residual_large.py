"""The T3 path at the benchmark shapes, where the index arithmetic is widest: nocc=10 /
nvir=90 (220 blocks) and the benzene cc-pVDZ shape nocc=15 / nvir=93 (680 blocks, odd
nvir, contraction offsets cut into pieces for the 31-bit split kernel).

* compute_r3_tri (T3Residual, FP64 and bf16x3) on sampled canonical blocks -- the first
  and last block and one block of every occupied case (i<j<k, i=j<k, i<j=k, i=j=k) --
  against the oracle's literal per-block restatement computed for those blocks only
  (oracle/einsum_ref.py, pinned to the reference's own compute_r3_tri by
  tests/test_ref_fixtures.py).  FP64: 1e-11 relative to the largest entry; bf16x3: 1e-4.
* the T3 -> r2 / W_vooo / W_vvvo feedback of the split path (tcgen05 GEMMs over X with the
  contraction cut into runs) against the FP64 feedback on the same device: 1e-4."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [(10, 90), (15, 93)]


def _targets(nocc):
    trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
    pick = {0, len(trip) - 1}
    for case in ((True, True), (False, True), (True, False), (False, False)):
        idx = [q for q, (i, j, k) in enumerate(trip) if ((i < j), (j < k)) == case]
        pick.add(idx[len(idx) // 2])
    return sorted(pick)


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import synthetic, t3_residual
    from oracle import einsum_ref
    return synthetic, t3_residual, einsum_ref


@pytest.mark.parametrize("nocc,nvir", SHAPES)
def test_residual_sampled_blocks(mods, nocc, nvir):
    syn, tr, er = mods
    d = syn.make_inputs(nocc, nvir, seed=nocc + nvir)
    names = ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")
    imds = er.Imds(*[getattr(d, k).cpu().numpy() for k in names])
    t3h = d.t3.cpu().numpy()
    tg = _targets(nocc)
    want = er.compute_r3_tri_ref(imds, d.t2.cpu().numpy(), t3h, nocc, targets=tg)
    del t3h
    scale = np.abs(want).max()
    for precision, bar in (("fp64", 1e-11), ("bf16x3", 1e-4)):
        res = tr.T3Residual(nocc, nvir, precision, with_oo=True)
        r3 = res.compute(d, d.t3)
        assert res.status_ok()
        got = r3[tg].cpu().numpy()
        del r3, res
        torch.cuda.empty_cache()
        err = np.abs(got - want).max() / scale
        assert err <= bar, (precision, err)


@pytest.mark.parametrize("nocc,nvir", SHAPES)
def test_split_feedback_vs_fp64(mods, nocc, nvir):
    syn, _, _ = mods
    from dcc import t3_feedback as fb
    d = syn.make_inputs(nocc, nvir, seed=3)
    g = torch.Generator(device="cuda").manual_seed(4)
    nmo = nocc + nvir
    o, v = slice(0, nocc), slice(nocc, nmo)
    sl = {"oovv": torch.randn(nocc, nocc, nvir, nvir, dtype=torch.float64, device="cuda", generator=g) * 0.1,
          "vovv": torch.randn(nvir, nocc, nvir, nvir, dtype=torch.float64, device="cuda", generator=g) * 0.1,
          "ooov": torch.randn(nocc, nocc, nocc, nvir, dtype=torch.float64, device="cuda", generator=g) * 0.1}
    X = fb.p3_201_all(d.t3, nocc)
    outs = {}
    for precision in ("fp64", "bf16x3"):
        r2 = torch.zeros(nocc, nocc, nvir, nvir, dtype=torch.float64, device="cuda")
        Wo = torch.zeros(nvir, nocc, nocc, nocc, dtype=torch.float64, device="cuda")
        Wv = torch.zeros(nvir, nvir, nvir, nocc, dtype=torch.float64, device="cuda")
        if precision == "fp64":
            zero = torch.zeros(nocc, nvir, dtype=torch.float64, device="cuda")
            fb.r2_add_t3_x_(r2, zero, sl["vovv"], sl["ooov"], X)
            fb.intermediates_t3_add_x_(Wo, Wv, sl["oovv"], X)
        else:
            s = fb.SplitFeedback(nocc, nvir, precision)
            s.run(X, sl, {"r2": r2, "W_vooo": Wo, "W_vvvo": Wv})
            torch.cuda.synchronize()
            assert int(s.status.item()) == 0
            del s
        outs[precision] = (r2, Wo, Wv)
        torch.cuda.empty_cache()
    for a, b in zip(outs["bf16x3"], outs["fp64"]):
        assert float((a - b).abs().max() / b.abs().max()) <= 1e-4
