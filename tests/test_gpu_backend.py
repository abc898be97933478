"""The "cuda" backend entry points with the reference's argument structure
(mycc, imds, t2, t3 = (dt3, t3_local), eris.pppp / mo_energy) on host numpy
inputs, against the oracles: the drop-in boundary end to end."""
import itertools
import types

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import backend
    from oracle import einsum_ref, feedback_ref, q_ref
    return backend, einsum_ref, feedback_ref, q_ref


def _problem(no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    g = rng.standard_normal((nmo,) * 4) * 0.1
    perms = [(0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2), (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0),
             (3, 2, 1, 0)]
    g = sum(g.transpose(p) for p in perms) / 8
    pppp = np.ascontiguousarray(g.transpose(0, 2, 1, 3))  # <pq|rs>
    o, v = slice(0, no), slice(no, nmo)
    imds = types.SimpleNamespace(
        F_vv=np.diag(rng.uniform(0.1, 3, nv)), F_oo=np.diag(rng.uniform(-1.5, -0.3, no)),
        W_vvvo=pppp[v, v, v, o].copy(), W_vooo=pppp[v, o, o, o].copy(), W_vvvv=pppp[v, v, v, v].copy(),
        W_ovov=pppp[o, v, o, v].copy(), W_ovvo=pppp[o, v, v, o].copy(), W_oooo=pppp[o, o, o, o].copy(),
        t1_eris=pppp, t1_fock=rng.standard_normal((nmo, nmo)) * 0.1)
    t2 = rng.standard_normal((no, no, nv, nv)) * 0.05
    t2 = 0.5 * (t2 + t2.transpose(1, 0, 3, 2))
    full = rng.standard_normal((no,) * 3 + (nv,) * 3) * 0.01
    U = sum(full.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3))) / 6
    t3 = np.stack([U[i, j, k] for i in range(no) for j in range(i, no) for k in range(j, no)])
    mycc = types.SimpleNamespace(nocc=no, nmo=nmo, einsum_backend="cuda", dcc_precision="fp64", comm=None)
    mo_energy = np.concatenate([np.sort(rng.uniform(-1.5, -0.3, no)), np.sort(rng.uniform(0.1, 3, nv))])
    eris = types.SimpleNamespace(pppp=pppp, mo_energy=mo_energy)
    return mycc, imds, t2, t3, U, eris


def test_compute_r3_tri(mods):
    backend, er, _, _ = mods
    mycc, imds, t2, t3, _, _ = _problem(3, 8, 1)
    want = er.compute_r3_tri_ref(er.Imds(imds.F_vv, imds.F_oo, imds.W_vvvo, imds.W_vooo, imds.W_vvvv, imds.W_ovov,
                                         imds.W_ovvo, imds.W_oooo), t2, t3, 3, with_oo=True)
    fields = dict(vars(imds))
    got = backend.compute_r3_tri(mycc, imds, t2, (None, t3))
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * np.abs(want).max())
    assert imds.W_vvvv is None and imds.W_ovov is None  # released as the reference does
    mycc.dcc_precision = "bf16x3"
    got = backend.compute_r3_tri(mycc, types.SimpleNamespace(**fields), t2, (None, t3))
    assert np.abs(got - want).max() <= 1e-4 * np.abs(want).max()


def test_feedback(mods, oracle):
    backend, _, fb, _ = mods
    mycc, imds, t2, t3, _, _ = _problem(3, 6, 2)
    rng = np.random.default_rng(0)
    r1, r2 = rng.standard_normal((3, 6)), rng.standard_normal((3, 3, 6, 6))
    w1, w2 = fb.r1r2_add_t3_ref(imds.t1_fock, imds.t1_eris, r1.copy(), r2.copy(), t3, 3, oracle)
    backend.r1r2_add_t3_tri_(mycc, imds, r1, r2, (None, t3))
    np.testing.assert_allclose(r1, w1, rtol=0, atol=1e-11 * np.abs(w1).max())
    np.testing.assert_allclose(r2, w2, rtol=0, atol=1e-11 * np.abs(w2).max())
    wo, wv = fb.intermediates_t3_add_ref(imds.t1_eris, imds.W_vooo.copy(), imds.W_vvvo.copy(), t3, 3, oracle)
    backend.intermediates_t3_add_t3_tri(mycc, imds, (None, t3))
    np.testing.assert_allclose(imds.W_vooo, wo, rtol=0, atol=1e-11 * np.abs(wo).max())
    np.testing.assert_allclose(imds.W_vvvo, wv, rtol=0, atol=1e-11 * np.abs(wv).max())


def test_q_kernel(mods, oracle):
    backend, _, _, q_ref = mods
    mycc, imds, t2, t3, U, eris = _problem(2, 6, 3)
    no, nmo = 2, 8
    p = eris.pppp
    o, v = slice(0, no), slice(no, nmo)
    er = {"vvvo": p[v, v, v, o], "vooo": p[v, o, o, o], "vvoo": p[v, v, o, o], "ovvo": p[o, v, v, o],
          "ovov": p[o, v, o, v], "vvvv": p[v, v, v, v], "oooo": p[o, o, o, o]}
    T = U.transpose(3, 4, 5, 0, 1, 2)
    want = q_ref.q_energy_ref(er, t2.transpose(2, 3, 0, 1), T, eris.mo_energy[:no], eris.mo_energy[no:], 2, oracle)
    got = backend.q_kernel(mycc, eris=eris, tamps=[None, t2, (None, t3)], blksize=2)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-14)


def test_compute_r4_tri_route(mods, oracle):
    """The reference's compute_r4_tri(mycc, imds, t2, t3, (dt4, t4_local)) on host numpy
    inputs through the backend, against the oracle's literal loop (OO batch included)."""
    backend = mods[0]
    from oracle import t4_ref
    from test_t4_residual_algebra import _inputs, stab_symmetric
    no, nv = 4, 5
    d = _inputs(no, nv, 21)
    quads = t4_ref.stored_quadruples(no)
    d["t4"] = stab_symmetric(d["t4"], quads)
    rng = np.random.default_rng(4)
    F_oo, W_ovvo = rng.standard_normal((no, no)), rng.standard_normal((no, nv, nv, no)) * 0.1
    want = t4_ref.compute_r4_tri_ref(d["eris"], d["F_vv"], d["W_vvvo"], d["W_vooo"], d["W_vvvv"], d["W_oooo"],
                                     d["W_ovov"], d["t2"], d["t3"], d["t4"], no, oracle, F_oo, W_ovvo)
    imds = types.SimpleNamespace(t1_eris=d["eris"], F_vv=d["F_vv"], W_vvvo=d["W_vvvo"], W_vooo=d["W_vooo"],
                                 W_vvvv=d["W_vvvv"], W_oooo=d["W_oooo"], W_ovov=d["W_ovov"], F_oo=F_oo,
                                 W_ovvo=W_ovvo)
    dt4 = types.SimpleNamespace(iter_local_ijkl=lambda: [q + (n,) for n, q in enumerate(quads)])
    mycc = types.SimpleNamespace(einsum_backend="cuda", comm=backend.SingleRankComm(), nocc=no,
                                 dcc_precision="fp64")
    got = backend.compute_r4_tri(mycc, imds, d["t2"], d["t3"], (dt4, d["t4"]))
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()
    assert imds.W_vvvo is None and imds.t1_eris is None  # released as the reference does


def test_q_kernel_abc_input_and_jobs(mods, oracle):
    """rccsdt_q.kernel with T3 already in the ABC layout (what the reference's
    prepare_tamps_for_q hands over, tests/test_rccsdt_q.py test_t3ijk_abc_transformation) and
    with job splitting (test_split_jobs): both give the energies of the plain call."""
    backend = mods[0]
    from dcc import _c_rccsdt
    mycc, imds, t2, t3, U, eris = _problem(2, 6, 3)
    full = np.array(backend.q_kernel(mycc, eris=eris, tamps=[None, t2, (None, t3)], blksize=2))
    t3_abc = _c_rccsdt.redistribute_ijk_to_abc(torch.from_numpy(np.ascontiguousarray(t3)).cuda(), 2, 6).cpu().numpy()

    class ABC:
        abc_to_global_idx = {}

    got = backend.q_kernel(mycc, eris=eris, tamps=[None, t2, (ABC(), t3_abc)], blksize=2)
    np.testing.assert_allclose(got, full, rtol=1e-12, atol=1e-15)
    jobs = sum(np.array(backend.q_kernel(mycc, eris=eris, tamps=[None, t2, (None, t3)], blksize=2, job_idx=j,
                                         n_jobs=3)) for j in range(3))
    np.testing.assert_allclose(jobs, full, rtol=1e-10, atol=1e-15)
