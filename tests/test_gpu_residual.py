"""Batched T3 residual (W.t2 via full-X GEMM + S3 gather, F_vv.t3, W_vvvv.t3)
and the fused update, against the literal per-block numpy restatement of
compute_r3_tri.  FP64 path: rtol 1e-11.  Split paths: relative to the largest
|r3|, 1e-4 (bf16x3) and 1e-5 (tf32x3 -- its accumulation limits it to that)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 1e-4, "tf32x3": 1e-4}


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import synthetic, t3_residual
    from oracle import einsum_ref
    return synthetic, t3_residual, einsum_ref


def _ref_r3(er, dn, with_oo=True):
    imds = er.Imds(dn.F_vv, dn.F_oo, dn.W_vvvo, dn.W_vooo, dn.W_vvvv, dn.W_ovov, dn.W_ovvo, dn.W_oooo)
    return er.compute_r3_tri_ref(imds, dn.t2, dn.t3, dn.nocc, with_oo=with_oo)


@pytest.mark.parametrize("nocc,nvir", [(2, 5), (3, 7), (4, 10), (3, 18)])
@pytest.mark.parametrize("precision", ["fp64", "bf16x3", "tf32x3"])
@pytest.mark.parametrize("with_oo", [False, True])
def test_residual(mods, nocc, nvir, precision, with_oo):
    syn, tr, er = mods
    d = syn.make_inputs(nocc, nvir, seed=nocc * 100 + nvir)
    dn = syn.to_numpy(d)
    want = _ref_r3(er, dn, with_oo)
    res = tr.T3Residual(nocc, nvir, precision, with_oo=with_oo)
    got = res.compute(d, d.t3).cpu().numpy()
    assert res.status_ok()
    if precision == "fp64":
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-13 * np.abs(want).max())
    else:
        assert np.abs(got - want).max() / np.abs(want).max() < TOL[precision]


@pytest.mark.parametrize("nocc,nvir,nact", [(3, 7, 5), (4, 9, 9)])
def test_update(mods, nocc, nvir, nact):
    syn, tr, er = mods
    d = syn.make_inputs(nocc, nvir, seed=7)
    dn = syn.to_numpy(d)
    r3 = torch.randn_like(d.t3) * 1e-4
    want_t3, want_r3, want_n = er.r3_update_ref(dn.t3, r3.cpu().numpy(), dn.eia, nocc, nact)
    t3 = d.t3.clone()
    norms = tr.update_t3_(t3, r3, d, nvir_active=nact)
    assert np.array_equal(r3.cpu().numpy(), want_r3)
    assert np.array_equal(t3.cpu().numpy(), want_t3)
    np.testing.assert_allclose(norms.cpu().numpy(), want_n, rtol=1e-12)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_residual_without_woooo_pair_symmetry(mods, precision):
    """A W_oooo without W[l,m,i,j] = W[m,l,j,i] keeps its antisymmetric part on the
    reference's own permutation set (a second gather pass)."""
    syn, tr, er = mods
    nocc, nvir = 3, 10
    d = syn.make_inputs(nocc, nvir, seed=4)
    g = torch.Generator(device="cuda").manual_seed(9)
    d.W_oooo = d.W_oooo + 0.05 * torch.randn(d.W_oooo.shape, dtype=torch.float64, device="cuda", generator=g)
    dn = syn.to_numpy(d)
    want = _ref_r3(er, dn, True)
    res = tr.T3Residual(nocc, nvir, precision, with_oo=True)
    got = res.compute(d, d.t3).cpu().numpy()
    assert res.status_ok() and res.Ganti is not None
    if precision == "fp64":
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-11 * np.abs(want).max())
    else:
        assert np.abs(got - want).max() / np.abs(want).max() < TOL[precision]


@pytest.mark.parametrize("nvir", [10, 18, 9])
@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_tma_gather_matches_cp_async_gather(mods, nvir, beta):
    """The TMA-pipelined permutation gather equals the cp.async kernel bit for bit
    (same summation order) for the full-layout and the Y-layout sources, every
    mask used by the residual, edge tiles (nvir = 10, 18) and the fallback (nvir = 9)."""
    syn, tr, er = mods
    no = 4
    d = syn.make_inputs(no, nvir, seed=1, with_t3=False)
    n3 = d.ijk.shape[0]
    g = torch.Generator(device="cuda").manual_seed(nvir)
    full = torch.randn((no ** 3, nvir, nvir, nvir), dtype=torch.float64, device="cuda", generator=g)
    Y = torch.randn((no * no * nvir, no * nvir * nvir), dtype=torch.float64, device="cuda", generator=g)
    Ny = no * nvir * nvir
    ys = (no * nvir * Ny, nvir * Ny, nvir * nvir, Ny, nvir, 1)
    r0 = torch.randn((n3, nvir, nvir, nvir), dtype=torch.float64, device="cuda", generator=g)
    for src in ([(full, 1.0, tr.full_strides(no, nvir), tr.ALL_S3), (Y, -1.0, ys, tr.ALL_S3)],
                [(full, 0.5, tr.full_strides(no, nvir), tr.OOOO_SET)],
                [(full, 1.0, tr.full_strides(no, nvir), tr.OO_SET), (Y, 2.0, ys, tr.OOOO_SET)]):
        a, b = r0.clone(), r0.clone()
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        tr.perm_gather_(a, d.ijk, nvir, beta, src)
        tr.perm_gather_(b, d.ijk, nvir, beta, src, nocc=no, status=st)
        torch.cuda.synchronize()
        assert int(st.item()) == 0
        assert torch.equal(a, b)


@pytest.mark.parametrize("no,nvir", [(1, 3), (2, 1), (3, 5), (4, 9), (3, 13), (2, 93), (3, 10), (2, 90)])
@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_row_gather_matches_cp_async_gather(mods, no, nvir, beta):
    """The full-layout, every-permutation gather of the residual runs by rows (two whole rows and
    four staged column tiles per output row) for nvir <= 104: bit for bit the cp.async kernel."""
    syn, tr, er = mods
    d = syn.make_inputs(no, nvir, seed=2, with_t3=False)
    n3 = d.ijk.shape[0]
    g = torch.Generator(device="cuda").manual_seed(nvir + 7 * no)
    full = torch.randn((no ** 3, nvir, nvir, nvir), dtype=torch.float64, device="cuda", generator=g)
    r0 = torch.randn((n3, nvir, nvir, nvir), dtype=torch.float64, device="cuda", generator=g)
    src = [(full, -1.25, tr.full_strides(no, nvir), tr.ALL_S3)]
    a, b = r0.clone(), r0.clone()
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    tr.perm_gather_(a, d.ijk, nvir, beta, src)
    tr.perm_gather_(b, d.ijk, nvir, beta, src, nocc=no, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert torch.equal(a, b)


@pytest.mark.parametrize("no,nvir", [(1, 3), (2, 1), (3, 5), (3, 13), (2, 93), (2, 90), (2, 104)])
@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_fp32_gather_matches_fp64_gather(mods, no, nvir, beta):
    """The gather from an FP32 S (the split path's accumulator) equals the FP64 row gather over
    the same values widened to FP64, bit for bit (the same FP64 sums in the same order)."""
    syn, tr, er = mods
    d = syn.make_inputs(no, nvir, seed=3, with_t3=False)
    n3 = d.ijk.shape[0]
    g = torch.Generator(device="cuda").manual_seed(nvir + 11 * no)
    full = torch.randn((no ** 3, nvir, nvir, nvir), dtype=torch.float64, device="cuda", generator=g).float()
    r0 = torch.randn((n3, nvir, nvir, nvir), dtype=torch.float64, device="cuda", generator=g)
    a, b = r0.clone(), r0.clone()
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    tr.s3_gather_f32_(a, d.ijk, nvir, beta, full, -1.25, no)
    tr.perm_gather_(b, d.ijk, nvir, beta, [(full.double(), -1.25, tr.full_strides(no, nvir), tr.ALL_S3)], nocc=no,
                    status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    assert torch.equal(a, b)


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_autotuned_wvvvv_gemms(mods, precision):
    """T3Residual.tune times every pipeline candidate of the W_vvvv.t3 GEMMs (K = nvir^2 >
    4096 takes the configurable pipeline) and keeps the fastest; the tuned residual still
    matches the FP64 path within the split tolerance, and t3 is not modified by tuning."""
    syn, tr, _ = mods
    from dcc import autotune
    old = autotune.get_config()
    try:
        d = syn.make_inputs(2, 72, seed=7)
        t3_0 = d.t3.clone()
        res = tr.T3Residual(2, 72, precision, with_oo=True)
        cfg = res.tune(d, d.t3)
        assert cfg in autotune.candidates() and autotune.get_config() == cfg
        assert torch.equal(d.t3, t3_0)
        # every S GEMM was tuned over the tile widths and raster groups
        chosen = res.s_tuning()
        assert set(chosen) == {"y", "x", "oo", "t1", "woooo"}
        assert all(c in autotune.tile_candidates() for c, _ in chosen.values())
        autotune.set_config(*old)
        got = res.compute(d, d.t3)
        # the residual applies each tuned shape around its own launches and restores the previous one
        assert autotune.get_config() == old and autotune.chosen(res.wvvvv.key()) == cfg and res.status_ok()
        want = tr.T3Residual(2, 72, "fp64", with_oo=True).compute(d, d.t3)
        assert float((got - want).abs().max() / want.abs().max()) < TOL[precision]
    finally:
        autotune.set_config(*old)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_inputs_uploaded_during_the_unpack(mods, precision):
    """compute(..., inputs_ready=event): the intermediates arrive on a copy stream from pinned
    host memory while the unpack of t3 runs; the residual equals the one with resident inputs
    bit for bit (same kernels in the same order)."""
    syn, tr, _ = mods
    d = syn.make_inputs(4, 10, seed=21)
    res = tr.T3Residual(4, 10, precision, with_oo=True)
    want = res.compute(d, d.t3).clone()
    names = ("t2", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo", "F_vv", "F_oo")
    host = {k: getattr(d, k).cpu().pin_memory() for k in names}

    class Dev:
        pass

    dd = Dev()
    dd.ijk = d.ijk
    for k, v in host.items():
        setattr(dd, k, torch.full(v.shape, float("nan"), dtype=v.dtype, device="cuda"))
    torch.cuda.synchronize()
    side, ready = torch.cuda.Stream(), torch.cuda.Event()
    with torch.cuda.stream(side):
        for k, v in host.items():
            getattr(dd, k).copy_(v, non_blocking=True)
        ready.record(side)
    got = res.compute(dd, d.t3, inputs_ready=ready)
    torch.cuda.synchronize()
    assert torch.equal(got, want) and res.status_ok()


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_woooo_split_in_k_pieces(mods, precision):
    """The W_oooo / F_oo GEMM with its K-major U operand cut into K pieces (what nocc=15 /
    nvir=93 needs to keep the split's offsets within 31 bits), forced here at a small shape:
    same residual as one piece, within the split tolerance of the FP64 path."""
    syn, tr, _ = mods
    d = syn.make_inputs(5, 6, seed=31)
    one = tr.T3Residual(5, 6, precision, with_oo=True)
    cut = tr.T3Residual(5, 6, precision, with_oo=True, woooo_piece_limit=8 * 5 * 6 ** 3 + 1)
    assert one.woo_pieces == [25] and cut.woo_pieces == [8, 8, 8, 1]
    want = tr.T3Residual(5, 6, "fp64", with_oo=True).compute(d, d.t3)
    a, b = one.compute(d, d.t3), cut.compute(d, d.t3)
    assert one.status_ok() and cut.status_ok()
    scale = want.abs().max()
    assert float((b - want).abs().max() / scale) < TOL[precision]
    assert float((b - a).abs().max() / scale) < 1e-6
