"""Device DIIS against the numpy restatement of the reference's DIIS update:
same extrapolated vectors (1e-12 relative) and update norms over a sequence
longer than the slot count (circular reuse), with scaled segments."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import diis
    from oracle import diis_ref
    return diis, diis_ref


@pytest.mark.parametrize("space,nupd", [(3, 8), (6, 10)])
def test_diis_matches_reference(mods, space, nupd):
    diis, diis_ref = mods
    rng = np.random.default_rng(space)
    sizes, scales = [7, 40, 3000], [0.5, 0.5, 1.0]
    ref = diis_ref.DIISRef(space)
    dev = diis.DIIS(space)
    x = [rng.standard_normal(n) for n in sizes]
    for it in range(nupd):
        # a converging sequence with noise, as amplitudes over iterations
        x = [0.7 * v + 0.05 * rng.standard_normal(v.size) for v in x]
        segs = [torch.from_numpy(v.copy()).cuda() for v in x]
        want = ref.update(np.concatenate([v * s for v, s in zip(x, scales)]))
        dev.update(segs, scales)
        got = np.concatenate([t.cpu().numpy() * s for t, s in zip(segs, scales)])
        np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)
        if ref.last_delta_norm_sq is None:
            assert dev.last_delta_norm_sq is None
        else:
            assert abs(dev.last_delta_norm_sq - ref.last_delta_norm_sq) <= 1e-10 * max(ref.last_delta_norm_sq, 1e-30)
        x = [t.cpu().numpy() for t in segs]
