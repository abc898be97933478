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


@pytest.mark.parametrize("scratch_start", [0, 2])
def test_diis_host_slots_equal_device_slots(mods, scratch_start):
    """Slots kept in pinned host memory (the out-of-core slots) give bit for bit the
    results of slots in HBM: the same kernels read them through their unified addresses."""
    diis, _ = mods
    rng = np.random.default_rng(5)
    sizes, scales = [11, 300, 5000], [0.5, 0.5, 1.0]
    dev, host = diis.DIIS(4), diis.DIIS(4, scratch_start=scratch_start)
    x = [rng.standard_normal(n) for n in sizes]
    for it in range(7):
        x = [0.7 * v + 0.05 * rng.standard_normal(v.size) for v in x]
        a = [torch.from_numpy(v.copy()).cuda() for v in x]
        b = [t.clone() for t in a]
        dev.update(a, scales)
        host.update(b, scales)
        for p, q in zip(a, b):
            assert torch.equal(p, q)
        assert dev.last_delta_norm_sq == host.last_delta_norm_sq
        x = [t.cpu().numpy() for t in a]
    assert all(not host.xs[i].is_cuda and host.xs[i].is_pinned() for i in range(scratch_start, 4))
    assert all(host.xs[i].is_cuda for i in range(scratch_start))


def test_diis_refuses_pageable_slots(mods):
    diis, _ = mods
    d = diis.DIIS(2)
    segs = [torch.ones(64, dtype=torch.float64, device="cuda")]
    d.update(segs)
    d.xs[0] = torch.empty(64, dtype=torch.float64)  # pageable: the kernels could not read it
    d.es[0] = torch.empty(64, dtype=torch.float64)
    from dcc._lib import DccError
    with pytest.raises(DccError, match="pageable host memory"):
        d.update(segs)
