"""(Q) at the benzene cc-pVDZ shape (nocc=15, nvir=93, blksize 4: 17,550 tasks, a ragged
last virtual block of one) on sampled tasks, against the oracle's literal task loop
(oracle/q_ref.py, pinned to the reference's own kernel by tests/test_ref_fixtures.py)
evaluated for those tasks only, with T3 of every ordering read lazily from the canonical
blocks (tests/lazy_t3.py).  The device runs exactly the sampled tasks (one d-block of
three groups: the first, one in the middle, the last with its one-wide blocks).
FP64: relative 1e-10; bf16x3 (d-chunked, every contraction a tcgen05 GEMM): 1e-4."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import synthetic, _c_rccsdt
    from oracle import q_ref
    from lazy_t3 import LazyT
    no, nv, blk = 15, 93, 4
    d = synthetic.make_inputs(no, nv, seed=2)
    er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
          "vvvv": d.W_vvvv, "oooo": d.W_oooo}
    t2 = d.t2.permute(2, 3, 0, 1).contiguous()
    tasks = q_ref.task_list(nv, blk)
    sample = [tasks[0], tasks[len(tasks) // 2], tasks[-1]]
    host = {k: v.cpu().numpy() for k, v in er.items()}
    want = q_ref.q_energy_ref(host, t2.cpu().numpy(), LazyT(d.t3.cpu().numpy(), no), d.e_occ.cpu().numpy(),
                              d.e_vir.cpu().numpy(), blk, tasks=sample)
    t3_abc = _c_rccsdt.redistribute_ijk_to_abc(d.t3, no, nv)
    del d.t3
    torch.cuda.empty_cache()
    groups = [(t[0], t[1], t[3], t[4], t[6], t[7]) for t in sample]
    assert len(set(groups)) == len(groups)
    d_ranges = {g: (t[9], t[10]) for g, t in zip(groups, sample)}
    return (no, nv, blk, er, t2, t3_abc, d.e_occ, d.e_vir, groups, d_ranges), want


@pytest.mark.parametrize("precision,bar", [("fp64", 1e-10), ("bf16x3", 1e-4)])
def test_q_benzene_shape_sampled_tasks(case, precision, bar):
    from dcc import rccsdt_q
    (no, nv, blk, er, t2, t3_abc, eo, ev, groups, d_ranges), want = case
    q = rccsdt_q.QEnergy(no, nv, blk, precision)
    out = q.run(er, t2, t3_abc, eo, ev, groups, d_ranges)
    torch.cuda.synchronize()
    assert q.status_ok()
    got = [float(x) for x in out]
    for g, w in zip(got, want):
        assert abs(g - w) <= bar * abs(w), (precision, got, want)
