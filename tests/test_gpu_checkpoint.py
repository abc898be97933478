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
