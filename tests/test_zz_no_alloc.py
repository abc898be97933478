"""The allocation-free update entry point against the workspace one.

dcc_t3_divide_update_noalloc exists for callers that cannot allocate device
memory: a host runtime that owns all device allocations in its own pool and
forbids libraries to call cudaMalloc, or a thin ctypes caller that holds only
the amplitude tensors and has no allocator to get a workspace from.  It keeps
its partial sums in a static device array instead.  This file is collected
last so that a failure here leaves every other test already run; it does not
rely on anything the other tests set up.

Both entry points do the same per-element arithmetic, so t3 and r3 must agree
bit for bit; the norms are summed over a different number of partial sums,
so they agree to rtol 1e-12.
"""
import ctypes

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import _lib as L
    f = L.bind("dcc_t3_divide_update_noalloc", [L.c_vp, L.c_vp, L.c_vp, L.c_vp, L.c_i64, L.c_i64, L.c_i64,
                                                L.c_int, L.c_vp, L.c_vp])
    return L, f


def _inputs(nocc, nvir, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    trip = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]
    ijk = torch.tensor(trip, dtype=torch.int32, device="cuda")
    t3 = torch.randn((len(trip),) + (nvir,) * 3, dtype=torch.float64, device="cuda", generator=g) * 1e-3
    r3 = torch.randn(t3.shape, dtype=torch.float64, device="cuda", generator=g) * 1e-4
    eo = -1.5 + 1.2 * torch.rand(nocc, dtype=torch.float64, device="cuda", generator=g)
    ev = 0.1 + 2.9 * torch.rand(nvir, dtype=torch.float64, device="cuda", generator=g)
    eia = (eo[:, None] - ev[None, :]).contiguous()
    return t3, r3, eia, ijk


@pytest.mark.parametrize("nocc,nvir,nact", [(6, 40, 30), (10, 90, 90)])
def test_noalloc_matches_workspace_entry_twice(lib, nocc, nvir, nact):
    L, noalloc = lib
    from dcc import _c_rccsdt
    t3, r3, eia, ijk = _inputs(nocc, nvir, seed=nocc)
    t3_ref, r3_ref = t3.clone(), r3.clone()
    n_ref = _c_rccsdt.t3_divide_update_(t3_ref, r3_ref, eia, ijk, nvir_active=nact, write_r3=True)
    torch.cuda.synchronize()
    for _ in range(2):  # two calls in a row share the static scratch
        t3_n, r3_n = t3.clone(), r3.clone()
        norms = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        L.check(noalloc(L.ptr(t3_n), L.ptr(r3_n), L.ptr(eia), L.ptr(ijk), ijk.shape[0], nvir, nact, 1, L.ptr(norms),
                        stream))
        torch.cuda.synchronize()
        assert torch.equal(r3_n, r3_ref)
        assert torch.equal(t3_n, t3_ref)
        torch.testing.assert_close(norms, n_ref, rtol=1e-12, atol=0.0)


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    """One row more than the static array covers is refused before any launch.  The buffers
    are real and sized for the call (nvir = 2, so 2^21 + 1 blocks are 134 MB each), so even a
    launch would stay in bounds."""
    L, noalloc = lib
    nblk, nvir = (1 << 21) + 1, 2  # rows = nblk * nvir^2 = 8 388 612 > 8 388 608
    t3 = torch.zeros((nblk, nvir, nvir, nvir), dtype=torch.float64, device="cuda")
    r3 = torch.zeros_like(t3)
    eia = torch.full((1, nvir), -1.0, dtype=torch.float64, device="cuda")
    ijk = torch.zeros((nblk, 3), dtype=torch.int32, device="cuda")
    norms = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = noalloc(L.ptr(t3), L.ptr(r3), L.ptr(eia), L.ptr(ijk), nblk, nvir, nvir, 1, L.ptr(norms), stream)
    assert rc == 2 and "no-allocation limit" in L.last_error()
