"""Checkpoints written from and read into HBM (dcc/checkpoint.py): the pinned double-buffered
path must give the files np.save writes for the same blocks, and load them back bit for bit,
for one-rank and multi-rank layouts and for pieces that split blocks."""
import filecmp
import os

import numpy as np
import pytest
import torch

from dcc import checkpoint as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,nocc,nvir", [("t3", 6, 40), ("t4", 7, 11)])
@pytest.mark.parametrize("distribution,nranks", [("balanced", 1), ("round_robin", 3), ("block", 2)])
def test_device_checkpoint_round_trip(kind, nocc, nvir, distribution, nranks, tmp_path):
    save, load = (C.save_t3, C.load_t3) if kind == "t3" else (C.save_t4, C.load_t4)
    tuples = C.canonical_triples(nocc) if kind == "t3" else C.stored_quadruples(nocc)
    rank = 3 if kind == "t3" else 4
    g = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn((len(tuples),) + (nvir,) * rank, generator=g, dtype=torch.float64, device="cuda")
    chunk = 3 << 20 if kind == "t3" else 250_000  # pieces that end inside a block
    ck = save(x, str(tmp_path / "d_"), nocc, nvir, distribution=distribution, nranks=nranks, chunk_bytes=chunk)
    host = x.cpu().numpy()
    pos = {t: i for i, t in enumerate(tuples)}
    stem = "t3_local" if kind == "t3" else "t4_local"
    for r, lst in enumerate(ck.rank_tuples):
        np.save(tmp_path / "ref.npy", host[[pos[t] for t in lst]])
        assert filecmp.cmp(tmp_path / "ref.npy", tmp_path / ("d_%s_%d.npy" % (stem, r)), shallow=False)
    ck2, y = load(str(tmp_path / "d_"), device="cuda", chunk_bytes=chunk)
    assert y.is_cuda and torch.equal(y, x) and ck2.rank_tuples == ck.rank_tuples
    out = torch.full_like(x, float("nan"))
    _, z = load(str(tmp_path / "d_"), device="cuda", out=out)
    assert z is out and torch.equal(out, x)
    os.remove(tmp_path / "ref.npy")


def test_restart_from_checkpoint_continues_the_iteration(tmp_path):
    """The device counterpart of the reference's restart test (tests/test_rccsdt.py,
    _test_restart): two T3 iterations in a row equal one iteration, a checkpoint written and
    read back (here as a 3-rank round_robin checkpoint), and the second iteration."""
    from dcc import synthetic, t3_residual
    nocc, nvir = 4, 12
    d = synthetic.make_inputs(nocc, nvir, seed=5)
    res = t3_residual.T3Residual(nocc, nvir, "fp64", with_oo=True)
    t3a = d.t3.clone()
    for _ in range(2):
        r3 = res.compute(d, t3a)
        t3_residual.update_t3_(t3a, r3, d)
    t3b = d.t3.clone()
    r3 = res.compute(d, t3b)
    t3_residual.update_t3_(t3b, r3, d)
    C.save_t3(t3b, str(tmp_path / "run_"), nocc, nvir, distribution="round_robin", nranks=3)
    del t3b
    _, t3c = C.load_t3(str(tmp_path / "run_"), device="cuda")
    r3 = res.compute(d, t3c)
    t3_residual.update_t3_(t3c, r3, d)
    torch.cuda.synchronize()
    assert torch.equal(t3c, t3a)
