"""The (Q) group contractions on the CPU against the oracle's per-task blocks:
the einsum table of dcc.rccsdt_q run by the FP64 torch path, and the grouped
split-GEMM plan (every problem's split maps, contraction maps, output maps,
origin-linear source offsets and per-value batching) emulated with numpy in
FP64.  Both must reproduce z4 / t4 of every task of the group (relative 1e-12)."""
import numpy as np
import pytest
import torch

from oracle import q_ref
from dcc import rccsdt_q as gq
from test_maps_emulated import fmap
from test_q_oracle import _inputs


def _group_cases():
    return [(2, 5, 2, 0), (3, 7, 3, 2), (3, 9, 4, 5)]


def _oracle_group(er, t2, T, blk, g):
    """z, x of the group g = (a0, a1, b0, b1, c0, c1) as [i][j][k][l][a][b][c][d] (d over [c0, nv))."""
    a0, a1, b0, b1, c0, c1 = g
    nv, no = T.shape[0], T.shape[3]
    z = np.zeros((no,) * 4 + (a1 - a0, b1 - b0, c1 - c0, nv - c0))
    x = np.zeros_like(z)
    for d0, d1 in gq.prange(c0, nv, blk):
        task = (a0, a1, a1 - a0, b0, b1, b1 - b0, c0, c1, c1 - c0, d0, d1, d1 - d0)
        z4, t4 = q_ref.task_blocks(er, t2, T, task, blk)
        sl = (slice(0, a1 - a0), slice(0, b1 - b0), slice(0, c1 - c0), slice(0, d1 - d0))
        z[..., d0 - c0:d1 - c0] = z4[sl].transpose(4, 5, 6, 7, 0, 1, 2, 3)
        x[..., d0 - c0:d1 - c0] = t4[sl].transpose(4, 5, 6, 7, 0, 1, 2, 3)
    return z, x


def _slabs(T, r):
    a0, a1, b0, b1, c0, c1, d0, d1 = r
    rng = {"a": (a0, a1), "b": (b0, b1), "c": (c0, c1), "d": (d0, d1)}
    return {s: np.ascontiguousarray(T[rng[s[1]][0]:rng[s[1]][1], rng[s[2]][0]:rng[s[2]][1]]) for s in gq._SLABS}


@pytest.mark.parametrize("no,nv,blk,gi", _group_cases())
def test_fp64_group_blocks(no, nv, blk, gi):
    er, t2, T, eo, ev = _inputs(no, nv, 11 + gi)
    g = gq.groups(nv, blk)[gi]
    r = g + (g[4], nv)
    q = gq.QEnergy(no, nv, blk, "fp64", device="cpu")
    tt = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    z, x = q._run_fp64({k: tt(v) for k, v in er.items()}, tt(t2), {k: tt(v) for k, v in _slabs(T, r).items()}, r)
    zr, xr = _oracle_group(er, t2, T, blk, g)
    np.testing.assert_allclose(z.numpy(), zr, rtol=1e-12, atol=1e-14 * np.abs(zr).max())
    np.testing.assert_allclose(x.numpy(), xr, rtol=1e-12, atol=1e-14 * np.abs(xr).max())


@pytest.mark.parametrize("no,nv,blk,gi", _group_cases())
def test_grouped_plan_emulated(no, nv, blk, gi):
    er, t2, T, eo, ev = _inputs(no, nv, 11 + gi)
    g = gq.groups(nv, blk)[gi]
    a0, a1, b0, b1, c0, c1 = g
    r = g + (c0, nv)
    sig = (a1 - a0, b1 - b0, c1 - c0, nv - c0)
    probs, outs = gq.plan_problems(no, nv, sig)
    src = {k: np.ascontiguousarray(v).ravel() for k, v in er.items()}
    src["t2"] = np.ascontiguousarray(t2).ravel()
    src.update({k: v.ravel() for k, v in _slabs(T, r).items()})
    for name, n in outs:
        src[name] = np.zeros(n)
    org = np.array([a0, b0, c0, c0])
    for phase in (0, 1):
        for pr in probs:
            if pr["phase"] != phase:
                continue

            def operand(op, rows):
                base = int(op["coef"] @ org) + op["off"]
                idx = base + fmap(op["fm"], np.arange(rows))[:, None] + fmap(op["fk"], np.arange(pr["k"]))[None, :]
                flat = src[op["src"]]
                assert idx.min() >= 0 and idx.max() < flat.size
                return flat[idx]

            A, B = operand(pr["A"], pr["m"]), operand(pr["B"], pr["n"])
            oidx = pr["ooff"] + fmap(pr["orow"], np.arange(pr["m"]))[:, None] + fmap(pr["ocol"], np.arange(pr["n"]))[None, :]
            assert len(np.unique(oidx)) == oidx.size
            np.add.at(src[pr["out"]], oidx, pr["alpha"] * (A @ B.T))
    zr, xr = _oracle_group(er, t2, T, blk, g)
    np.testing.assert_allclose(src["z"].reshape(zr.shape), zr, rtol=1e-12, atol=1e-14 * np.abs(zr).max())
    np.testing.assert_allclose(src["x"].reshape(xr.shape), xr, rtol=1e-12, atol=1e-14 * np.abs(xr).max())


def test_plan_fits_the_grouped_launch():
    """Every group shape of the nocc=10 / nvir=90 / blk=4 workload plans into at most
    256 problems per phase with 32-bit map radices."""
    import collections
    sigs = {(g[1] - g[0], g[3] - g[2], g[5] - g[4], 90 - g[4]) for g in gq.groups(90, 4)}
    for sig in sorted(sigs)[:6] + sorted(sigs)[-6:]:
        probs, outs = gq.plan_problems(10, 90, sig)
        cnt = collections.Counter(p["phase"] for p in probs)
        assert cnt[0] * 2 <= 256 and cnt[1] * 2 <= 256
        for p in probs:
            assert p["m"] < 2 ** 31 and p["n"] < 2 ** 31


@pytest.mark.parametrize("nvir,blk,n_jobs", [(9, 2, 3), (11, 4, 5), (90, 4, 7), (13, 3, 13), (7, 6, 9)])
def test_job_d_ranges_cover_each_task_once(nvir, blk, n_jobs):
    """job_d_ranges over all jobs hands every task of the reference's order to exactly one
    job, as the contiguous slices of distr_cc/rccsdt_q.py:359-366 do."""
    from dcc import rccsdt_q
    tasks = rccsdt_q.task_list(nvir, blk)
    per = (len(tasks) + n_jobs - 1) // n_jobs
    seen = []
    for j in range(n_jobs):
        want = {(t[0], t[1], t[3], t[4], t[6], t[7], t[9]) for t in tasks[j * per:(j + 1) * per]}
        got = set()
        for (a0, a1, b0, b1, c0, c1), (d0, d1) in rccsdt_q.job_d_ranges(nvir, blk, j, n_jobs).items():
            assert c0 <= d0 < d1 <= nvir
            for dd0, _ in rccsdt_q.prange(d0, d1, blk):
                got.add((a0, a1, b0, b1, c0, c1, dd0))
        assert got == want
        seen += sorted(got)
    assert len(seen) == len(set(seen)) == len(tasks)
    with pytest.raises(ValueError):
        rccsdt_q.job_d_ranges(nvir, blk, n_jobs, n_jobs)


def test_default_dchunk():
    """Chunks of whole task blocks whose two FP32 group blocks stay within 256 MiB (one pass
    over the d range when they fit)."""
    from dcc import rccsdt_q
    assert rccsdt_q.default_dchunk(10, 90, 4) == 52
    assert rccsdt_q.default_dchunk(6, 40, 4) == 40
    c = rccsdt_q.default_dchunk(15, 93, 4)
    assert c == 8 and c % 4 == 0 and 2 * 4 * 64 * 15 ** 4 * c <= 1 << 28
    assert rccsdt_q.default_dchunk(40, 200, 8) == 8  # never below one block
