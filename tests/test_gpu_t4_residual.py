"""T4 residual on the GPU against the oracle's per-block einsums: the dense
F_vv.t4 / W_vvvv.t4 strings (distr_cc/rccsdtq.py:1039-1055) and the whole of
compute_r4_tri with its OO batch (:700-1349, W builders included), up to
the N2 6-31G shape (nocc=7, nvir=11, 161 stored blocks).  FP64: 1e-11
relative; split paths: 1e-4 of the largest |r4|."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "bf16x3", "tf32x3"])
@pytest.mark.parametrize("nblk,nv", [(5, 6), (20, 11)])
def test_dense_t4(precision, nblk, nv):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import t4_residual
    from oracle import t4_ref
    rng = np.random.default_rng(nv)
    W = rng.standard_normal((nv,) * 4) * 0.1
    F = rng.standard_normal((nv, nv))
    t4 = rng.standard_normal((nblk,) + (nv,) * 4) * 1e-3
    r0 = rng.standard_normal(t4.shape) * 1e-3
    want = t4_ref.dense_vvvv_fvv_ref(r0, t4, W, F)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    r = dev(r0)
    t4_residual.dense_vvvv_fvv_(r, dev(t4), dev(W), dev(F), precision)
    got = r.cpu().numpy()
    tol = 1e-12 if precision == "fp64" else 1e-4
    assert np.abs(got - want).max() <= tol * np.abs(want - r0).max()


_REF = {}


def _case(oracle, no, nv):
    """Inputs and the oracle's r4 (computed once per shape)."""
    if (no, nv) not in _REF:
        from oracle import t4_ref
        from test_t4_residual_algebra import _inputs, stab_symmetric
        d = _inputs(no, nv, 5 + no)
        rng = np.random.default_rng(no)
        d["t4"] = stab_symmetric(d["t4"], t4_ref.stored_quadruples(no))
        d["F_oo"] = rng.standard_normal((no, no))
        d["W_ovvo"] = rng.standard_normal((no, nv, nv, no)) * 0.1
        want = t4_ref.compute_r4_tri_ref(d["eris"], d["F_vv"], d["W_vvvo"], d["W_vooo"], d["W_vvvv"], d["W_oooo"],
                                         d["W_ovov"], d["t2"], d["t3"], d["t4"], no, oracle, d["F_oo"],
                                         d["W_ovvo"])
        _REF[(no, nv)] = (d, want)
    return _REF[(no, nv)]


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
@pytest.mark.parametrize("no,nv", [(4, 5), (7, 11)])
def test_compute_r4_tri(oracle, precision, no, nv):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import t4_residual
    d, want = _case(oracle, no, nv)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in d.items()}
    r4 = torch.zeros_like(t["t4"])
    t4_residual.compute_r4_tri_(r4, t["eris"], t["F_vv"], t["W_vvvo"], t["W_vooo"], t["W_vvvv"], t["W_oooo"],
                                t["W_ovov"], t["t2"], t["t3"], t["t4"], no, precision, F_oo=t["F_oo"],
                                W_ovvo=t["W_ovvo"])
    got = r4.cpu().numpy()
    tol = 1e-11 if precision == "fp64" else 1e-4
    assert np.abs(got - want).max() <= tol * np.abs(want).max()
    assert int(t4_residual.fused_status(r4.device).item()) == 0


@pytest.mark.parametrize("nv", [3, 5, 11, 13])
def test_fused_strings_split_rows(nv):
    """The fused strings kernel at sizes where its row split (output rows a per CTA) and its
    warp tiles are ragged: its r4 against the batched per-string einsums of the same strings
    on the same device (rtol 1e-12)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import t4_residual as tr, _c_rccsdtq
    no = 4
    g = torch.Generator(device="cuda").manual_seed(nv)
    nq = len(tr.stored_quadruples(no))
    shp = tr._operand_shapes(no, nv, nq)
    ops = {n: torch.randn(sh, dtype=torch.float64, device="cuda", generator=g) for n, sh in shp.items()}
    desc, quads, names, _ = tr.fused_plan(no, nv, True, "cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    r4 = torch.full((nq, nv ** 4), 7.0, dtype=torch.float64, device="cuda")
    _c_rccsdtq.t4_strings([ops[n] for n in names], desc, quads, no, nv, r4, 0.0, status)
    want = torch.zeros((nq,) + (nv,) * 4, dtype=torch.float64, device="cuda")
    T = {"t3": ops["t3"], "t3_m": ops["t3"], "t3_mn": ops["t3"], "t3p_m": ops["t3p"], "t3s_m": ops["t3s"],
         "t2_m": ops["t2"], "t2": ops["t2"]}
    cache = {}
    for sub, wn, ws, tn, ts, al in tr._R4_STRINGS:
        sw, st = sub.split(",")
        gw, lw = tr._gather_slots(ops[wn], tr._slots(wn, ws, sw), no, cache, wn)
        gt, lt = tr._gather_slots(T[tn], tr._slots(tn, ts, st), no, cache, tn)
        want.add_(torch.einsum("q" + lw + ",q" + lt + "->qabcd", gw, gt), alpha=al)
    for n, s in enumerate(tr.STRINGS):
        want += torch.einsum(s, ops["Wf" if n in (0, 5) else "W_vvvv"], ops["t4"])
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    err = (r4.view_as(want) - want).abs().max() / want.abs().max()
    assert float(err) <= 1e-12
    # beta = 1 adds to r4
    r4b = r4.clone()
    _c_rccsdtq.t4_strings([ops[n] for n in names], desc, quads, no, nv, r4b, 1.0, status)
    assert float((r4b - 2 * r4).abs().max() / r4.abs().max()) <= 1e-15


def test_fused_strings_checks():
    """Descriptors, blocks and pairs the fused kernel refuses before touching memory: an
    operand index past the table, a stride whose last element lies past its operand, an
    occupied index out of range, a pair with m outside [0, nocc), a pair range past the list.
    The string is skipped (status bit 2), the block left unwritten (bit 1), the pair or pair
    range skipped (bit 4); the other strings, blocks and pairs still run."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import t4_residual as tr, _c_rccsdtq
    no, nv = 4, 5
    nq = len(tr.stored_quadruples(no))
    shp = tr._operand_shapes(no, nv, nq)
    g = torch.Generator(device="cuda").manual_seed(1)
    ops = {n: torch.randn(sh, dtype=torch.float64, device="cuda", generator=g) for n, sh in shp.items()}
    desc, quads, names, _ = tr.fused_plan(no, nv, False, "cuda")
    args = [ops[n] for n in names]
    good = torch.zeros(nq, nv ** 4, dtype=torch.float64, device="cuda")
    _c_rccsdtq.t4_strings(args, desc[1:], quads, no, nv, good, 0.0)
    for bad in ("op", "stride"):
        d = desc.clone()
        if bad == "op":
            d[0, 0] = len(names)
        else:  # W_vvvo [a, b, e, j]: stride of e grown until e's last value lies past the end
            d[0, 22] = 1 + (ops["W_vvvo"].numel() - 1) // (d[0, 21] - 1)
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        r4 = torch.zeros_like(good)
        _c_rccsdtq.t4_strings(args, d, quads, no, nv, r4, 0.0, st)
        torch.cuda.synchronize()
        assert int(st.item()) == 2, bad
        assert torch.equal(r4, good), bad
    qd = quads.clone()
    qd[3, 2] = no
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    r4 = torch.full_like(good, 5.0)
    _c_rccsdtq.t4_strings(args, desc, qd, no, nv, r4, 0.0, st)
    torch.cuda.synchronize()
    assert int(st.item()) == 1
    assert bool((r4[3] == 5.0).all()) and not bool((r4[4] == 5.0).all())
    # pair mode: a pair whose m lies outside [0, nocc), a pair range past the list
    desc, quads, names, (off, sm) = tr.fused_plan(no, nv, False, "cuda", oo=True)
    shp.update({n: tr._operand_shapes(no, nv, nq)[n] for n in tr._OO_OPS})
    ops = {n: torch.randn(shp[n], dtype=torch.float64, device="cuda", generator=g) for n in names}
    args = [ops[n] for n in names]
    good = torch.zeros(nq, nv ** 4, dtype=torch.float64, device="cuda")
    _c_rccsdtq.t4_strings(args, desc, quads, no, nv, good, 0.0, pairs=(off, sm))
    for bad in ("m", "range"):
        o2, s2 = off.clone(), sm.clone()
        if bad == "m":
            s2[0, 1] = no
        else:
            o2[2, 5] = s2.shape[0] + 1
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        r4 = torch.zeros_like(good)
        _c_rccsdtq.t4_strings(args, desc, quads, no, nv, r4, 0.0, st, pairs=(o2, s2))
        torch.cuda.synchronize()
        assert int(st.item()) == 4, bad
        assert torch.isfinite(r4).all(), bad


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
@pytest.mark.parametrize("no,nv", [(4, 5), (7, 11)])
def test_t4_feedback(oracle, precision, no, nv):
    """r2_add_t4_tri_ / r3_add_t4_tri_ (distr_cc/rccsdtq.py:471-683) on the GPU (P4_442 /
    P4_201 kernels, full-space strings) against the oracle's literal per-block loops."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import t4_residual
    from oracle import t4_ref
    rng = np.random.default_rng(7 * no + nv)
    nmo = no + nv
    t4 = rng.standard_normal((len(t4_ref.stored_quadruples(no)),) + (nv,) * 4) * 0.01
    eris = rng.standard_normal((nmo,) * 4) * 0.1
    fock = rng.standard_normal((nmo, nmo)) * 0.1
    r2 = rng.standard_normal((no, no, nv, nv)) * 1e-3
    r3 = rng.standard_normal((no,) * 3 + (nv,) * 3) * 1e-3
    want2 = t4_ref.r2_add_t4_tri_ref(r2, t4, eris, no, oracle)
    want3 = t4_ref.r3_add_t4_tri_ref(r3, t4, fock, eris, no, oracle)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got2 = t4_residual.r2_add_t4_(dev(r2), dev(t4), dev(eris), no, precision).cpu().numpy()
    got3 = t4_residual.r3_add_t4_(dev(r3), dev(t4), dev(fock), dev(eris), no, precision).cpu().numpy()
    tol = 1e-11 if precision == "fp64" else 1e-4
    assert np.abs(got2 - want2).max() <= tol * np.abs(want2 - r2).max()
    assert np.abs(got3 - want3).max() <= tol * np.abs(want3 - r3).max()
