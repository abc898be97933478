"""Property tests of host-side logic over random sizes (hypothesis, CPU only): the (Q) job
slices partition the reference's task order for any (nvir, blksize, n_jobs), and checkpoints
round-trip for any rank count, assignment and staging chunk."""
import numpy as np
import pytest
import torch

hyp = pytest.importorskip("hypothesis")
from hypothesis import given, settings, strategies as st  # noqa: E402

from dcc import checkpoint as C  # noqa: E402
from dcc import rccsdt_q  # noqa: E402


@settings(max_examples=40, deadline=None)
@given(nvir=st.integers(1, 40), blk=st.integers(1, 9), n_jobs=st.integers(1, 30))
def test_job_slices_partition_the_tasks(nvir, blk, n_jobs):
    tasks = rccsdt_q.task_list(nvir, blk)
    seen = []
    for j in range(n_jobs):
        for (a0, a1, b0, b1, c0, c1), (d0, d1) in rccsdt_q.job_d_ranges(nvir, blk, j, n_jobs).items():
            assert c0 <= d0 < d1 <= nvir
            seen += [(a0, b0, c0, dd0) for dd0, _ in rccsdt_q.prange(d0, d1, blk)]
    assert sorted(seen) == sorted((t[0], t[3], t[6], t[9]) for t in tasks)


@settings(max_examples=25, deadline=None)
@given(nocc=st.integers(1, 5), nvir=st.integers(1, 4), nranks=st.integers(1, 12),
       dist=st.sampled_from(["round_robin", "block", "balanced"]), chunk=st.integers(1, 5000),
       kind=st.sampled_from(["t3", "t4"]), seed=st.integers(0, 2 ** 16))
def test_checkpoint_round_trip(tmp_path_factory, nocc, nvir, nranks, dist, chunk, kind, seed):
    tuples = C.canonical_triples(nocc) if kind == "t3" else C.stored_quadruples(nocc)
    if not tuples:
        return
    rank = 3 if kind == "t3" else 4
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((len(tuples),) + (nvir,) * rank, generator=g, dtype=torch.float64)
    prefix = str(tmp_path_factory.mktemp("ck") / "p_")
    save, load = (C.save_t3, C.load_t3) if kind == "t3" else (C.save_t4, C.load_t4)
    ck = save(x, prefix, nocc, nvir, distribution=dist, nranks=nranks, chunk_bytes=chunk)
    assert sum(len(r) for r in ck.rank_tuples) == len(tuples)
    ck2, y = load(prefix, device="cpu", chunk_bytes=chunk)
    assert torch.equal(y, x) and ck2.size == nranks and ck2.rank_tuples == ck.rank_tuples
    stem = "t3_local" if kind == "t3" else "t4_local"
    pos = {t: i for i, t in enumerate(tuples)}
    for r, lst in enumerate(ck.rank_tuples):
        arr = np.load("%s%s_%d.npy" % (prefix, stem, r))
        assert np.array_equal(arr, x.numpy()[[pos[t] for t in lst]].reshape(arr.shape))
