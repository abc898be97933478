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
