"""The "cuda" einsum-backend router on the CPU: wrapped reference functions
call the GPU implementations only when mycc.einsum_backend == "cuda", call
the originals otherwise, refuse communicators of more than one rank, and
install is idempotent; the one-rank communicator shim behaves as MPI at one
rank."""
import types

import numpy as np
import pytest

from dcc import backend


def _fake_module():
    calls = []
    mod = types.SimpleNamespace()
    for name in ("r1r2_add_t3_tri_", "intermediates_t3_add_t3_tri", "compute_r3_tri"):
        def f(mycc, *a, _n=name, **k):
            calls.append(("orig", _n))
            return "orig:" + _n
        setattr(mod, name, f)
    qmod = types.SimpleNamespace(kernel=lambda mycc, *a, **k: calls.append(("orig", "q")) or "orig:q")
    return mod, qmod, calls


def test_routing_and_idempotence(monkeypatch):
    mod, qmod, calls = _fake_module()
    routed = []
    monkeypatch.setitem(backend._ROUTES, "compute_r3_tri", lambda mycc, *a, **k: routed.append("r3") or "gpu:r3")
    names = backend.install(mod, qmod)
    assert set(names) == {"r1r2_add_t3_tri_", "intermediates_t3_add_t3_tri", "compute_r3_tri", "rccsdt_q.kernel"}
    assert backend.install(mod, qmod) == []  # already wrapped
    mycc = types.SimpleNamespace(einsum_backend="numpy", comm=backend.SingleRankComm())
    assert mod.compute_r3_tri(mycc, None, None, None) == "orig:compute_r3_tri"
    assert qmod.kernel(mycc) == "orig:q"
    mycc.einsum_backend = "cuda"
    assert mod.compute_r3_tri(mycc, None, None, None) == "gpu:r3"
    assert routed == ["r3"]


def test_update_and_diis_routes_and_class_attributes(monkeypatch):
    """update_amps_rccsdt_tri_ / run_diis_t3 route as module functions (called with the module,
    whose lower-order functions they use) and as the RCCSDT class attributes the reference's
    kernel calls (distr_cc/rccsdt.py:1266, 1271)."""
    calls = []

    def upd(mycc, tamps, eris):
        calls.append("orig_upd")
        return "orig"

    def diis(mycc, *a, **k):
        calls.append("orig_diis")
        return "orig"

    class RCCSDT:
        update_amps_ = upd
        run_diis_t3 = diis

    mod = types.SimpleNamespace(update_amps_rccsdt_tri_=upd, run_diis_t3=diis, RCCSDT=RCCSDT)
    got = {}
    monkeypatch.setitem(backend._MOD_ROUTES, "update_amps_rccsdt_tri_",
                        lambda mycc, tamps, eris, mod=None: got.setdefault("upd_mod", mod) and "gpu")
    monkeypatch.setitem(backend._MOD_ROUTES, "run_diis_t3",
                        lambda mycc, *a, mod=None, **k: got.setdefault("diis_mod", mod) and "gpu")
    names = backend.install(mod)
    assert {"update_amps_rccsdt_tri_", "run_diis_t3", "RCCSDT.update_amps_", "RCCSDT.run_diis_t3"} <= set(names)
    cc = RCCSDT()
    cc.einsum_backend, cc.comm = "numpy", backend.SingleRankComm()
    assert cc.update_amps_([], None) == "orig" and cc.run_diis_t3([], None, 0, 0.0, 0.0, None) == "orig"
    cc.einsum_backend = "cuda"
    assert cc.update_amps_([], None) == "gpu" and cc.run_diis_t3([], None, 0, 0.0, 0.0, None) == "gpu"
    assert got["upd_mod"] is mod and got["diis_mod"] is mod
    assert calls == ["orig_upd", "orig_diis"]
    assert backend.install(mod) == []


def test_t3_local_order_checked():
    """A t3_local whose blocks are not in canonical order (e.g. loaded from a checkpoint of
    another distribution) is refused instead of being read in the wrong order."""
    from dcc.synthetic import canonical_ijk
    nocc = 3
    trip = canonical_ijk(nocc)

    class Dist:
        def __init__(self, order):
            self.order = order

        def iter_local_ijk(self):
            for q, (i, j, k) in enumerate(self.order):
                yield i, j, k, q
    mycc = types.SimpleNamespace(nocc=nocc, nmo=nocc + 4)
    t3 = np.zeros((len(trip), 4, 4, 4))
    assert backend._t3_local(mycc, (Dist(trip), t3)) is t3
    with pytest.raises(RuntimeError, match="canonical order"):
        backend._t3_local(mycc, (Dist(trip[::-1]), t3))
    with pytest.raises(RuntimeError, match="canonical order"):
        backend._t3_local(mycc, (Dist(trip), t3[:-1]))


def test_multi_rank_refused():
    class TwoRanks(backend.SingleRankComm):
        def Get_size(self):
            return 2
    mycc = types.SimpleNamespace(einsum_backend="cuda", comm=TwoRanks(), nocc=2, nmo=5)
    with pytest.raises(RuntimeError, match="one rank"):
        backend.compute_r3_tri(mycc, None, None, (None, None))
    with pytest.raises(RuntimeError, match="one rank"):
        backend.q_kernel(mycc, comm=TwoRanks())
    with pytest.raises(RuntimeError, match="one rank"):
        backend.q_kernel(mycc)  # comm=None falls back to mycc.comm, as the reference does


def test_single_rank_comm():
    c = backend.SingleRankComm()
    assert c.Get_rank() == 0 and c.Get_size() == 1 and c.bcast(5) == 5 and c.allreduce(3.0) == 3.0
    send, recv = np.arange(4.0), np.zeros(4)
    c.Allreduce(send, recv)
    np.testing.assert_array_equal(recv, send)
    buf = np.ones(3)
    c.Allreduce(buf)  # in place
    np.testing.assert_array_equal(buf, np.ones(3))


def test_rccsdtq_route(monkeypatch):
    """compute_r4_tri of distr_cc/rccsdtq.py is wrapped once and routed by the backend string."""
    orig_calls = []
    r4mod = types.SimpleNamespace(compute_r4_tri=lambda mycc, *a, **k: orig_calls.append("orig") or "orig:r4")
    routed = []
    monkeypatch.setattr(backend, "compute_r4_tri", lambda mycc, *a, **k: routed.append("gpu") or "gpu:r4")
    mod, qmod, _ = _fake_module()
    names = backend.install(mod, qmod, r4mod)
    assert "rccsdtq.compute_r4_tri" in names
    assert "rccsdtq.compute_r4_tri" not in backend.install(mod, qmod, r4mod)
    mycc = types.SimpleNamespace(einsum_backend="numpy", comm=backend.SingleRankComm())
    assert r4mod.compute_r4_tri(mycc, None, None, None, None) == "orig:r4"
    mycc.einsum_backend = "cuda"
    assert r4mod.compute_r4_tri(mycc, None, None, None, None) == "gpu:r4"
    assert orig_calls == ["orig"] and routed == ["gpu"]


def test_t4_feedback_routes(monkeypatch):
    """r2_add_t4_tri_ / r3_add_t4_tri_ of distr_cc/rccsdtq.py are routed by the backend string."""
    r4mod = types.SimpleNamespace(r2_add_t4_tri_=lambda mycc, *a: "orig:r2", r3_add_t4_tri_=lambda mycc, *a: "orig:r3")
    monkeypatch.setitem(backend._R4_ROUTES, "r2_add_t4_tri_", lambda mycc, *a: "gpu:r2")
    monkeypatch.setitem(backend._R4_ROUTES, "r3_add_t4_tri_", lambda mycc, *a: "gpu:r3")
    mod, qmod, _ = _fake_module()
    names = backend.install(mod, qmod, r4mod)
    assert {"rccsdtq.r2_add_t4_tri_", "rccsdtq.r3_add_t4_tri_"} <= set(names)
    mycc = types.SimpleNamespace(einsum_backend="numpy", comm=backend.SingleRankComm())
    assert (r4mod.r2_add_t4_tri_(mycc, 0, 0, 0), r4mod.r3_add_t4_tri_(mycc, 0, 0, 0)) == ("orig:r2", "orig:r3")
    mycc.einsum_backend = "cuda"
    assert (r4mod.r2_add_t4_tri_(mycc, 0, 0, 0), r4mod.r3_add_t4_tri_(mycc, 0, 0, 0)) == ("gpu:r2", "gpu:r3")


def test_host_einsum_reads_cuda_as_numpy():
    """Reference code left on the host calls `_einsum(mycc.einsum_backend, ...)`; after install
    the backend string "cuda" reaches the original as "numpy", other strings unchanged."""
    seen = []

    def _einsum(backend, subs, *ops, out=None, alpha=1.0, beta=0.0):
        if backend not in ("numpy", "pytblis"):
            raise ValueError("unknown einsum backend %r" % backend)
        seen.append(backend)
        res = alpha * np.einsum(subs, *ops)
        if out is None:
            return res
        out *= beta
        out += res
        return out

    mod = types.SimpleNamespace(_einsum=_einsum, __name__="fake_rccsdt")
    pyscf_mod = types.SimpleNamespace(_einsum=_einsum, __name__="fake_pyscf")
    names = backend.install(mod, host_einsum_modules=(pyscf_mod,))
    assert "fake_rccsdt._einsum" in names and "fake_pyscf._einsum" in names
    assert "fake_rccsdt._einsum" not in backend.install(mod)  # idempotent
    a, b = np.arange(6.0).reshape(2, 3), np.arange(12.0).reshape(3, 4)
    out = np.ones((2, 4))
    mod._einsum("cuda", "ij,jk->ik", a, b, out=out, alpha=2.0, beta=1.0)
    np.testing.assert_allclose(out, 1.0 + 2.0 * a @ b)
    np.testing.assert_allclose(pyscf_mod._einsum("pytblis", "ij,jk->ik", a, b), a @ b)
    assert seen == ["numpy", "pytblis"]
