"""The oracle's numpy restatements against outputs of the reference's own
Python drivers (tests/golden/ref_drivers.npz, written by
tests/golden/make_ref_fixtures.py, which runs distr_cc/rccsdt.py,
rccsdt_q.py, rccsdtq.py and diis.py unmodified).  CPU only, FP64: relative
1e-12 of the largest entry, energies 1e-12 relative.  The GPU side of the same
fixtures is tests/test_gpu_ref_fixtures.py."""
import os

import numpy as np
import pytest

from oracle import diis_ref, einsum_ref, feedback_ref, q_ref, t4_ref

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_drivers.npz")


@pytest.fixture(scope="module")
def fx():
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


def case(fx, tag):
    p = tag + "/"
    return {k[len(p):]: v for k, v in fx.items() if k.startswith(p)}


def close(got, want, rel=1e-12):
    scale = max(np.abs(want).max(), 1e-300)
    assert np.abs(np.asarray(got) - want).max() <= rel * scale, np.abs(np.asarray(got) - want).max() / scale


IMDS = ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")


@pytest.mark.parametrize("tag", ["r3a", "r3b", "r3c"])
def test_compute_r3_tri(fx, tag):
    c = case(fx, tag)
    no = int(c["shape"][0])
    im = einsum_ref.Imds(*[c[k] for k in IMDS])
    close(einsum_ref.compute_r3_tri_ref(im, c["t2"], c["t3"], no), c["r3"])


def test_feedback(fx, oracle):
    c = case(fx, "fb")
    no = int(c["shape"][0])
    r1, r2 = feedback_ref.r1r2_add_t3_ref(c["t1_fock"], c["t1_eris"], c["r1_in"].copy(), c["r2_in"].copy(), c["t3"],
                                          no, oracle)
    close(r1, c["r1"])
    close(r2, c["r2"])
    Wo, Wv = feedback_ref.intermediates_t3_add_ref(c["t1_eris"], c["W_vooo_in"].copy(), c["W_vvvo_in"].copy(),
                                                   c["t3"], no, oracle)
    close(Wo, c["W_vooo"])
    close(Wv, c["W_vvvo"])


def _q_inputs(c, no):
    g = c["pppp"]
    o, v = slice(0, no), slice(no, g.shape[0])
    er = {"vvvo": g[v, v, v, o], "vooo": g[v, o, o, o], "vvoo": g[v, v, o, o], "ovvo": g[o, v, v, o],
          "ovov": g[o, v, o, v], "vvvv": g[v, v, v, v], "oooo": g[o, o, o, o]}
    er = {k: np.ascontiguousarray(a) for k, a in er.items()}
    t2 = np.ascontiguousarray(c["t2"].transpose(2, 3, 0, 1))
    nv = g.shape[0] - no
    U = np.zeros((no,) * 3 + (nv,) * 3)
    q = 0
    for i in range(no):
        for j in range(i, no):
            for k in range(j, no):
                for p in set(__import__("itertools").permutations((0, 1, 2))):
                    idx = (i, j, k)
                    U[tuple(idx[x] for x in p)] = c["t3"][q].transpose(p)
                q += 1
    T = np.ascontiguousarray(U.transpose(3, 4, 5, 0, 1, 2))
    e = c["mo_energy"]
    return er, t2, T, e[:no], e[no:]


@pytest.mark.parametrize("tag", ["q", "q4"])
def test_q_energies(fx, oracle, tag):
    c = case(fx, tag)
    no, nv, n_jobs = (int(x) for x in c["shape"][:3])
    er, t2, T, eo, ev = _q_inputs(c, no)
    for blk in (int(b) for b in c["shape"][3:]):
        want = c["e_blk%d" % blk]
        got = q_ref.q_energy_ref(er, t2, T, eo, ev, blk, oracle)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
        tasks = q_ref.task_list(nv, blk)
        per = (len(tasks) + n_jobs - 1) // n_jobs
        for job in range(n_jobs):
            got = q_ref.q_energy_ref(er, t2, T, eo, ev, blk, oracle, tasks=tasks[job * per:(job + 1) * per])
            np.testing.assert_allclose(got, c["e_blk%d_job%d" % (blk, job)], rtol=1e-12, atol=1e-18)


def test_t4(fx, oracle):
    c = case(fx, "t4")
    no = int(c["shape"][0])
    assert [tuple(q) for q in c["ijkl"]] == [tuple(q) for q in t4_ref.stored_quadruples(no)]
    r4 = t4_ref.compute_r4_tri_ref(c["t1_eris"], c["F_vv"], c["W_vvvo"], c["W_vooo"], c["W_vvvv"], c["W_oooo"],
                                   c["W_ovov"], c["t2"], c["t3"], c["t4"], no, oracle, c["F_oo"], c["W_ovvo"])
    close(r4, c["r4"])
    close(t4_ref.r2_add_t4_tri_ref(c["r2_in"].copy(), c["t4"], c["t1_eris"], no, oracle), c["r2"])
    close(t4_ref.r3_add_t4_tri_ref(c["r3_in"].copy(), c["t4"], c["t1_fock"], c["t1_eris"], no, oracle), c["r3"])


def test_diis(fx):
    c = case(fx, "diis")
    d = diis_ref.DIISRef(space=int(c["shape"][1]))
    for x, want, dn in zip(c["x"], c["xnew"], c["delta_norm_sq"]):
        close(d.update(x), want)
        if np.isnan(dn):
            assert d.last_delta_norm_sq is None
        else:
            np.testing.assert_allclose(d.last_delta_norm_sq, dn, rtol=1e-12)
