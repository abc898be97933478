"""The drop-in routes on the GPU against outputs of the reference's own Python
drivers (tests/golden/ref_drivers.npz; tests/golden/make_ref_fixtures.py ran
distr_cc/rccsdt.py, rccsdt_q.py, rccsdtq.py and diis.py unmodified to make
them).  Every call goes through dcc.backend, the functions a reference
installation routes to, with host numpy inputs as the reference passes them.

Bars: FP64 paths 1e-11 relative to the largest entry (1e-10 for the four
update + DIIS iterations, energies 1e-10 relative); split-precision paths
(bf16x3, tf32x3: every large contraction a split tcgen05 GEMM with FP32
accumulation) 1e-4 relative to the largest entry or energy, 1e-3 for the
DIIS update norm (a difference of successive iterates)."""
import os
import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import ref_standins as S  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_drivers.npz")
PRECISIONS = ["fp64", "bf16x3", "tf32x3"]


@pytest.fixture(scope="module")
def fx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def backend():
    from dcc import backend
    return backend


def case(fx, tag):
    p = tag + "/"
    return {k[len(p):]: v for k, v in fx.items() if k.startswith(p)}


def bar(precision, fp64=1e-11):
    return fp64 if precision == "fp64" else 1e-4


def close(got, want, rel):
    got = np.asarray(got)
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(got - want).max() / scale
    assert err <= rel, "relative error %.3e > %.1e" % (err, rel)


def make_cc(no, nv, precision, **kw):
    cc = types.SimpleNamespace(nocc=no, nmo=no + nv, einsum_backend="cuda", dcc_precision=precision,
                               comm=S.OneRankComm(), rank=0, size=1, level_shift=0.0, nvir_diis=None,
                               diis_start_cycle=0, diis_start_energy_diff=1e9, unique_tamps_map=None)
    for k, v in kw.items():
        setattr(cc, k, v)
    cc.unique_tamps_map = S.build_unique_tamps_map(cc)
    return cc


IMDS = ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("tag", ["r3a", "r3b", "r3c"])
def test_compute_r3_tri(fx, backend, tag, precision):
    """compute_r3_tri (distr_cc/rccsdt.py:368-732), OO batch included; r3b has a W_oooo
    without the pair symmetry."""
    c = case(fx, tag)
    no, nv = (int(x) for x in c["shape"][:2])
    cc = make_cc(no, nv, precision)
    imds = types.SimpleNamespace(**{k: c[k].copy() for k in IMDS})
    r3 = backend.compute_r3_tri(cc, imds, c["t2"], (S.CanonicalT3Dist(no), c["t3"]))
    close(r3, c["r3"], bar(precision))
    assert all(getattr(imds, k) is None for k in IMDS)  # released, as the reference does


def test_feedback(fx, backend):
    """r1r2_add_t3_tri_ and intermediates_t3_add_t3_tri (distr_cc/rccsdt.py:253-366), FP64."""
    c = case(fx, "fb")
    no, nv = (int(x) for x in c["shape"][:2])
    cc = make_cc(no, nv, "fp64")
    imds = types.SimpleNamespace(t1_fock=c["t1_fock"], t1_eris=c["t1_eris"], W_vooo=c["W_vooo_in"].copy(),
                                 W_vvvo=c["W_vvvo_in"].copy())
    t3 = (S.CanonicalT3Dist(no), c["t3"])
    r1, r2 = backend.r1r2_add_t3_tri_(cc, imds, c["r1_in"].copy(), c["r2_in"].copy(), t3)
    close(r1, c["r1"], 1e-11)
    close(r2, c["r2"], 1e-11)
    backend.intermediates_t3_add_t3_tri(cc, imds, t3)
    close(imds.W_vooo, c["W_vooo"], 1e-11)
    close(imds.W_vvvo, c["W_vvvo"], 1e-11)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("tag", ["upd", "updnd"])
def test_update_amps_and_diis_routes(fx, backend, tag, precision):
    """Four iterations of update_amps_rccsdt_tri_ + run_diis_t3 (the loop body of
    distr_cc/rccsdt.py:1103-1121) through the routed versions, T3 resident on the device from
    the first call on; the lower-order PySCF steps are replayed from the same arrays the
    reference ran with.  updnd runs DIIS over the active virtual sub-block (nvir_diis)."""
    c = case(fx, tag)
    no, nv, niter, nd, space = (int(x) for x in c["shape"])
    cc = make_cc(no, nv, precision, nvir_diis=None if nd < 0 else nd)
    mod = S.route_module(S.LowerOrderReplay(c, no))
    eris = types.SimpleNamespace(mo_energy=c["mo_energy"])
    tamps = [c["t1"].copy(), c["t2"].copy(), (S.CanonicalT3Dist(no), c["t3"].copy())]
    adiis = types.SimpleNamespace(space=space, last_delta_norm_sq=None)
    rel = 1e-10 if precision == "fp64" else 1e-4
    for it in range(niter):
        res_norm = backend.update_amps_rccsdt_tri_(cc, tamps, eris, mod=mod)
        assert isinstance(tamps[2][1], backend.DeviceT3Local)
        np.testing.assert_allclose(res_norm, c["it%d/res_norm" % it], rtol=rel)
        close(np.asarray(tamps[2][1]), c["it%d/t3_pre" % it], rel)
        normt = np.linalg.norm(c["it%d/res_norm" % it])
        tamps, un = backend.run_diis_t3(cc, tamps, tamps[2][1], it, normt, 0.0, adiis, res_norm=res_norm,
                                        return_update_norm=True, mod=mod)
        close(tamps[0], c["it%d/t1" % it], rel)
        close(tamps[1], c["it%d/t2" % it], rel)
        close(np.asarray(tamps[2][1]), c["it%d/t3" % it], rel)
        # the update norm is |x_new - x_prev|, a difference of nearly equal vectors: the split
        # path's relative error in it is about 10x its error in the amplitudes themselves
        np.testing.assert_allclose(un, c["it%d/update_norm" % it], rtol=1e-8 if precision == "fp64" else 1e-3)


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("tag", ["q", "q4"])
def test_q_kernel(fx, backend, tag, precision):
    """rccsdt_q.kernel (distr_cc/rccsdt_q.py:227): all tasks, and split into jobs."""
    c = case(fx, tag)
    no, nv, n_jobs = (int(x) for x in c["shape"][:3])
    rel = 1e-10 if precision == "fp64" else 1e-4
    for blk in (int(b) for b in c["shape"][3:]):
        for job in [None] + list(range(n_jobs)):
            cc = make_cc(no, nv, precision)
            eris = types.SimpleNamespace(pppp=c["pppp"], mo_energy=c["mo_energy"])
            tamps = [c["t1"], c["t2"], (S.CanonicalT3Dist(no), c["t3"])]
            kw = {} if job is None else dict(job_idx=job, n_jobs=n_jobs)
            got = backend.q_kernel(cc, eris=eris, tamps=tamps, blksize=blk, comm=cc.comm, **kw)
            want = c["e_blk%d" % blk] if job is None else c["e_blk%d_job%d" % (blk, job)]
            scale = np.abs(c["e_blk%d" % blk]).max()
            assert np.abs(np.asarray(got) - want).max() <= rel * scale, (got, want)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_t4_routes(fx, backend, precision):
    """compute_r4_tri (OO batch included), r2_add_t4_tri_, r3_add_t4_tri_ (distr_cc/rccsdtq.py:471-1349)."""
    c = case(fx, "t4")
    no, nv = (int(x) for x in c["shape"][:2])
    cc = make_cc(no, nv, precision)
    t4 = (S.StoredT4Dist(c["ijkl"]), c["t4"])
    imds = types.SimpleNamespace(t1_eris=c["t1_eris"], t1_fock=c["t1_fock"])
    close(backend.r2_add_t4_tri_(cc, imds, c["r2_in"].copy(), t4), c["r2"], bar(precision))
    close(backend.r3_add_t4_tri_(cc, imds, c["r3_in"].copy(), t4), c["r3"], bar(precision))
    imds = types.SimpleNamespace(**{k: c[k] for k in IMDS}, t1_eris=c["t1_eris"], t1_fock=c["t1_fock"])
    close(backend.compute_r4_tri(cc, imds, c["t2"], c["t3"], t4), c["r4"], bar(precision))


def test_diis(fx):
    """DIIS.update (distr_cc/diis.py:105-177) on device segments."""
    from dcc.diis import DIIS
    c = case(fx, "diis")
    n, space = (int(x) for x in c["shape"][:2])
    d = DIIS(space=space)
    for x, want, dn in zip(c["x"], c["xnew"], c["delta_norm_sq"]):
        a = torch.from_numpy(x[: n // 3].copy()).cuda()
        b = torch.from_numpy(x[n // 3:].copy()).cuda()
        d.update([a, b])
        close(torch.cat([a, b]).cpu().numpy(), want, 1e-12)
        if np.isnan(dn):
            assert d.last_delta_norm_sq is None
        else:
            np.testing.assert_allclose(d.last_delta_norm_sq, dn, rtol=1e-10)
