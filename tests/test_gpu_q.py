"""RCCSDT(Q) energies on the GPU (grouped contractions + fused epilogue)
against the oracle's literal task loop.  FP64: relative 1e-10.  Split
paths (every contraction on the tcgen05 GEMM): relative 1e-4 of the
energy, the accuracy class of the split products."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from test_q_oracle import _inputs  # noqa: E402


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import rccsdt_q
    from oracle import q_ref
    return rccsdt_q, q_ref


def _device(er, t2, T, eo, ev, no):
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    ijk = [(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)]
    Tijk = T.transpose(3, 4, 5, 0, 1, 2)
    t3 = np.stack([Tijk[i, j, k] for i, j, k in ijk])
    return {k: dev(v) for k, v in er.items()}, dev(t2), dev(t3), dev(eo), dev(ev)


@pytest.mark.parametrize("no,nv,blk", [(2, 5, 2), (3, 7, 4), (3, 9, 3)])
def test_q_energy_fp64(mods, oracle, no, nv, blk):
    gq, q_ref = mods
    er, t2, T, eo, ev = _inputs(no, nv, 5 + nv)
    want = q_ref.q_energy_ref(er, t2, T, eo, ev, blk, oracle)
    d = _device(er, t2, T, eo, ev, no)
    got = gq.q_energy(d[0], d[1], d[2], d[3], d[4], no, nv, blk, "fp64")
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_q_energy_split(mods, oracle, precision):
    gq, q_ref = mods
    no, nv, blk = 3, 9, 3
    er, t2, T, eo, ev = _inputs(no, nv, 17)
    want = q_ref.q_energy_ref(er, t2, T, eo, ev, blk, oracle)
    d = _device(er, t2, T, eo, ev, no)
    got = gq.q_energy(d[0], d[1], d[2], d[3], d[4], no, nv, blk, precision)
    assert abs(got[0] - want[0]) <= 1e-4 * abs(want[0])
    assert abs(got[1] - want[1]) <= 1e-4 * abs(want[1])


@pytest.mark.parametrize("dchunk", [1, 2, 5])
def test_q_energy_split_d_chunks(mods, oracle, dchunk):
    """The split path in d-chunks of a group (including chunks that cut task blocks):
    the same energies as the oracle's task loop."""
    gq, q_ref = mods
    from dcc import _c_rccsdt
    no, nv, blk = 3, 9, 3
    er, t2, T, eo, ev = _inputs(no, nv, 19)
    want = q_ref.q_energy_ref(er, t2, T, eo, ev, blk, oracle)
    d = _device(er, t2, T, eo, ev, no)
    q = gq.QEnergy(no, nv, blk, "bf16x3", dchunk=dchunk)
    out = q.run(d[0], d[1], _c_rccsdt.redistribute_ijk_to_abc(d[2], no, nv), d[3], d[4])
    torch.cuda.synchronize()
    assert q.status_ok()
    got = out.cpu().numpy()
    assert abs(got[0] - want[0]) <= 1e-4 * abs(want[0])
    assert abs(got[1] - want[1]) <= 1e-4 * abs(want[1])


@pytest.mark.parametrize("precision", ["bf16x3", "tf32x3"])
def test_q_energy_split_microhartree(mods, precision):
    """The 1 uEh bar against the plain FP64 GPU path, at nocc=6 / nvir=40 on every task.  The
    seeded synthetic amplitudes give an (Q) energy of O(1) Eh, far above a molecule's; t2 and t3
    are scaled by one factor s so that the FP64 (Q) energy is -1e-3 Eh (the size of a molecular
    (Q) correction), and both energies of the split path must then lie within 1e-6 Eh of FP64."""
    gq, _ = mods
    from dcc import _c_rccsdt, synthetic
    no, nv, blk = 6, 40, 4
    d = synthetic.make_inputs(no, nv, seed=41)
    er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
          "vvvv": d.W_vvvv, "oooo": d.W_oooo}
    t2 = d.t2.permute(2, 3, 0, 1).contiguous()
    t3 = _c_rccsdt.redistribute_ijk_to_abc(d.t3, no, nv)

    def energies(prec, s):
        q = gq.QEnergy(no, nv, blk, prec)
        out = q.run(er, t2 * s, t3 * s, d.e_occ, d.e_vir).cpu().numpy()
        assert q.status_ok()
        return out

    e1 = energies("fp64", 1.0)
    s = (1e-3 / abs(e1[1])) ** 0.5
    want = energies("fp64", s)
    got = energies(precision, s)
    assert 1e-4 < abs(want[1]) < 1e-2
    assert abs(got[0] - want[0]) < 1e-6, (got, want)
    assert abs(got[1] - want[1]) < 1e-6, (got, want)


@pytest.mark.parametrize("precision,n_jobs", [("fp64", 3), ("fp64", 7), ("bf16x3", 4)])
def test_q_energy_split_jobs(mods, oracle, precision, n_jobs):
    """Job splitting as the reference's test_split_jobs (tests/test_rccsdt_q.py): the energies
    of jobs 0..n_jobs-1 add up to the oracle's full energies (FP64 1e-10; split 1e-4)."""
    gq, q_ref = mods
    no, nv, blk = 3, 9, 2
    er, t2, T, eo, ev = _inputs(no, nv, 23)
    want = q_ref.q_energy_ref(er, t2, T, eo, ev, blk, oracle)
    d = _device(er, t2, T, eo, ev, no)
    got = np.zeros(2)
    for j in range(n_jobs):
        got += gq.q_energy(d[0], d[1], d[2], d[3], d[4], no, nv, blk, precision, job_idx=j, n_jobs=n_jobs)
    tol = 1e-10 if precision == "fp64" else 1e-4
    assert abs(got[0] - want[0]) <= tol * abs(want[0])
    assert abs(got[1] - want[1]) <= tol * abs(want[1])
