"""Dense T4-residual strings (F_vv.t4, W_vvvv.t4; distr_cc/rccsdtq.py:1039-1055)
on the GPU against the oracle's per-block einsums.  FP64: 1e-12 relative;
split paths: 1e-4 of the largest |r4| change."""
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
