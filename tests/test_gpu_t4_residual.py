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
