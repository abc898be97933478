"""Checkpoint interop with the reference's on-disk T3 / T4 format (dcc/checkpoint.py).

The fixtures under tests/golden/checkpoints/ were written by the reference's own
save_to_disk for every rank of 1-, 2- and 3-rank runs (tests/golden/make_checkpoints.py),
so loading them checks the reader against real reference output, and writing the same
blocks again must reproduce every file byte for byte.
"""
import filecmp
import json
import os

import numpy as np
import pytest
import torch

from dcc import checkpoint as C

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "checkpoints")
CASES = sorted(os.listdir(GOLDEN))


def _fns(kind):
    return (C.save_t3, C.load_t3, "rank_triples") if kind == "t3" else (C.save_t4, C.load_t4, "rank_quadruples")


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("chunk", [C.CHUNK_BYTES, 1000, 8])
def test_load_reference_checkpoint(case, chunk):
    _, load, _ = _fns(case[:2])
    blocks = np.load(os.path.join(GOLDEN, case, "blocks.npy"))
    ck, x = load(os.path.join(GOLDEN, case, "ckpt_"), device="cpu", chunk_bytes=chunk)
    assert np.array_equal(x.numpy(), blocks)
    with open(os.path.join(GOLDEN, case, "ckpt_metadata.json")) as f:
        meta = json.load(f)
    assert (ck.nocc, ck.nvir, ck.size, ck.distribution) == (meta["nocc"], meta["nvir"], meta["size"],
                                                            meta["distribution"])


@pytest.mark.parametrize("case", CASES)
def test_save_matches_reference_files(case, tmp_path):
    kind = case[:2]
    save, load, key = _fns(kind)
    ck, _ = load(os.path.join(GOLDEN, case, "ckpt_"), device="cpu")
    blocks = torch.from_numpy(np.load(os.path.join(GOLDEN, case, "blocks.npy")))
    kw = {key: ck.rank_tuples} if ck.batch_size is not None else {"nranks": ck.size}
    save(blocks, str(tmp_path / "ckpt_"), ck.nocc, ck.nvir, distribution=ck.distribution,
         batch_size=ck.batch_size, chunk_bytes=700, **kw)
    names = sorted(n for n in os.listdir(os.path.join(GOLDEN, case)) if n.startswith("ckpt_"))
    assert names == sorted(os.listdir(tmp_path))
    for n in names:
        assert filecmp.cmp(os.path.join(GOLDEN, case, n), str(tmp_path / n), shallow=False), n


@pytest.mark.parametrize("kind", ["t3", "t4"])
@pytest.mark.parametrize("distribution,nranks", [("round_robin", 5), ("block", 4), ("balanced", 1), ("block", 40)])
def test_round_trip_any_rank_count(kind, distribution, nranks, tmp_path):
    save, load, _ = _fns(kind)
    nocc, nvir = (4, 5) if kind == "t3" else (5, 3)
    n = len(C.canonical_triples(nocc) if kind == "t3" else C.stored_quadruples(nocc))
    g = torch.Generator().manual_seed(7)
    x = torch.randn((n,) + (nvir,) * (3 if kind == "t3" else 4), generator=g, dtype=torch.float64)
    save(x, str(tmp_path / "c_"), nocc, nvir, distribution=distribution, nranks=nranks, chunk_bytes=333)
    out = torch.zeros_like(x)
    ck, y = load(str(tmp_path / "c_"), device="cpu", out=out, chunk_bytes=256)
    assert y is out and torch.equal(y, x) and ck.size == nranks
    # A rank's file is what np.save writes for the rank's slice of the blocks.
    stem = "t3_local" if kind == "t3" else "t4_local"
    tuples = C.canonical_triples(nocc) if kind == "t3" else C.stored_quadruples(nocc)
    pos = {t: i for i, t in enumerate(tuples)}
    ref = tmp_path / "np.npy"
    for r, lst in enumerate(ck.rank_tuples):
        np.save(ref, x.numpy()[[pos[t] for t in lst]].reshape((len(lst),) + (nvir,) * (3 if kind == "t3" else 4)))
        assert filecmp.cmp(ref, tmp_path / ("c_%s_%d.npy" % (stem, r)), shallow=False)


def test_assign_ranks_matches_reference_strategies():
    t = C.canonical_triples(4)
    rr = C.assign_ranks(t, 3, "round_robin")
    assert [len(a) for a in rr] == [7, 7, 6] and rr[1][:2] == [(0, 0, 1), (0, 1, 1)]
    bl = C.assign_ranks(t, 3, "block")
    assert [len(a) for a in bl] == [7, 7, 6] and sum(bl, []) == t
    assert C.assign_ranks(t, 3, "balanced") == rr
    with pytest.raises(NotImplementedError):
        C.assign_ranks(t, 2, "balanced", batch_size=4)
    with pytest.raises(ValueError, match="Unknown distribution"):
        C.assign_ranks(t, 2, "cyclic")


def test_errors(tmp_path):
    x = torch.randn(10, 4, 4, 4, dtype=torch.float64)
    with pytest.raises(ValueError, match="shape"):
        C.save_t3(x[:9], str(tmp_path / "a_"), 3, 4)
    with pytest.raises(TypeError, match="float64"):
        C.save_t3(x.float(), str(tmp_path / "a_"), 3, 4)
    with pytest.raises(ValueError, match="more than one rank"):
        C.save_t3(x, str(tmp_path / "a_"), 3, 4, rank_triples=[[(0, 0, 0)], C.canonical_triples(3)])
    with pytest.raises(ValueError, match="no rank holds"):
        C.save_t3(x, str(tmp_path / "a_"), 3, 4, rank_triples=[C.canonical_triples(3)[1:]])
    with pytest.raises(ValueError, match="not a stored canonical"):
        C.save_t3(x, str(tmp_path / "a_"), 3, 4, rank_triples=[C.canonical_triples(3) + [(1, 0, 2)]])
    C.save_t3(x, str(tmp_path / "b_"), 3, 4, distribution="round_robin", nranks=2)
    # A truncated rank file and a float32 rank file are refused.
    path = tmp_path / "b_t3_local_1.npy"
    data = path.read_bytes()
    path.write_bytes(data[:-8])
    with pytest.raises(ValueError, match="ends 8 bytes early"):
        C.load_t3(str(tmp_path / "b_"), device="cpu")
    np.save(path, np.zeros((5, 4, 4, 4), dtype=np.float32))
    with pytest.raises(ValueError, match="dtype"):
        C.load_t3(str(tmp_path / "b_"), device="cpu")
    os.remove(path)
    with pytest.raises(FileNotFoundError):
        C.load_t3(str(tmp_path / "b_"), device="cpu")
    with pytest.raises(ValueError, match="not T4"):
        with open(tmp_path / "c_metadata.json", "w") as f:
            json.dump({"kind": "DistributedT3IJK", "nocc": 3, "nvir": 4, "dtype": "<f8", "size": 1}, f)
        C.load_t4(str(tmp_path / "c_"), device="cpu")
