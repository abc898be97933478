"""Checkpoints of the stored T3 / T4 amplitudes in the reference's on-disk format, written
from and read into device memory.

Format (DistributedT3IJK.save_to_disk, distr_cc/distribute_t3.py:959-996;
DistributedT4IJKL.save_to_disk, distr_cc/distribute_t4.py:903-925): for each rank r of the
run that wrote it, `{prefix}t3_local_{r}.npy` holds the rank's blocks, float64
[n, nv, nv, nv], in the order of `{prefix}ijk_triples_{r}.npy` (int32 [n, 3]); rank 0 adds
`{prefix}metadata.json` with nocc, nvir, distribution, batch_size, dtype and size.  T4 uses
`t4_local` / `ijkl_quadruples` (int32 [n, 4]) and adds "kind" and "zero_rule".

One GPU holds every stored block here, in canonical order (the one-rank layout), so
  * save_t3 / save_t4 write a one-rank checkpoint, or one for `nranks` ranks under the
    reference's round_robin / block assignment (distr_cc/distribute_t3.py:210-230) or an
    explicit per-rank list, which a multi-rank reference run then loads unchanged;
  * load_t3 / load_t4 take a checkpoint written by any number of ranks and put each rank's
    blocks at their canonical positions.  The reference's loader insists on the writer's
    rank count (distr_cc/distribute_t3.py:1018-1020); one device needs no such limit.

Bytes move between the file and HBM through two pinned host buffers: while one buffer is
written to (read from) the file, an asynchronous copy on the current stream fills (drains)
the other.  Blocks that are consecutive both in the file and in canonical order move as one
run.  The .npy headers are numpy's own version-1.0 headers, the ones np.save writes, so the
files equal np.save's output byte for byte.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from .t4_residual import stored_quadruples

CHUNK_BYTES = 64 << 20
T4_ZERO_RULE = "skip_i_eq_j_eq_k_or_j_eq_k_eq_l"


def canonical_triples(nocc):
    """i <= j <= k in lexicographic order (distr_cc/distribute_t3.py:180-188)."""
    return [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]


def assign_ranks(tuples, nranks, distribution="balanced", batch_size=None):
    """Per-rank lists of the canonical tuples under the reference's simple strategies:
    round_robin (tuple n to rank n % nranks), block (contiguous ranges, the first
    len % nranks ranks one longer) and balanced without batch_size, which is round_robin
    (distr_cc/distribute_t3.py:196-230; distr_cc/distribute_t4.py:225-260 for T4).  The
    cost-balanced assignment of balanced + batch_size is the reference's own heuristic;
    pass its result as `rank_tuples` instead."""
    nranks = int(nranks)
    if nranks <= 0:
        raise ValueError("nranks must be positive")
    if distribution == "balanced" and batch_size is not None and nranks > 1:
        raise NotImplementedError("the cost-balanced assignment (balanced with batch_size) is not "
                                  "restated here; pass the per-rank lists as rank_tuples")
    if distribution in ("round_robin", "balanced"):
        return [list(tuples[r::nranks]) for r in range(nranks)]
    if distribution == "block":
        base, rem = divmod(len(tuples), nranks)
        out, start = [], 0
        for r in range(nranks):
            n = base + (1 if r < rem else 0)
            out.append(list(tuples[start:start + n]))
            start += n
        return out
    raise ValueError("Unknown distribution strategy: %s" % distribution)


def _check_cover(rank_tuples, tuples, what):
    """Every canonical tuple on exactly one rank; returns the canonical positions per rank."""
    pos = {t: n for n, t in enumerate(tuples)}
    seen = np.zeros(len(tuples), dtype=bool)
    out = []
    for r, lst in enumerate(rank_tuples):
        idx = []
        for t in lst:
            t = tuple(int(x) for x in t)
            n = pos.get(t)
            if n is None:
                raise ValueError("rank %d lists %s %s, which is not a stored canonical block" % (r, what, t))
            if seen[n]:
                raise ValueError("%s %s is listed on more than one rank" % (what, t))
            seen[n] = True
            idx.append(n)
        out.append(idx)
    if not seen.all():
        missing = tuples[int(np.argmin(seen))]
        raise ValueError("no rank holds %s %s (%d of %d blocks missing)" % (what, missing, int((~seen).sum()),
                                                                          len(tuples)))
    return out


def _runs(idx):
    """(file block, canonical block, count) for maximal runs consecutive in both orders."""
    runs = []
    for n, g in enumerate(idx):
        if runs and runs[-1][1] + runs[-1][2] == g:
            runs[-1][2] += 1
        else:
            runs.append([n, g, 1])
    return [tuple(r) for r in runs]


def _pieces(runs, block_bytes, chunk_bytes):
    """(canonical byte offset, nbytes) pieces of at most chunk_bytes, in file order."""
    for _, g, cnt in runs:
        off, end = g * block_bytes, (g + cnt) * block_bytes
        while off < end:
            n = min(chunk_bytes, end - off)
            yield off, n
            off += n


class _Staging:
    """Two host buffers of `nbytes` (pinned when the amplitudes live on a GPU) with an event
    each: the event marks the end of the last asynchronous copy that used the buffer."""

    def __init__(self, nbytes, device):
        self.cuda = torch.device(device).type == "cuda"
        self.bufs = [torch.empty(nbytes, dtype=torch.uint8, pin_memory=self.cuda) for _ in range(2)]
        self.views = [b.numpy() for b in self.bufs]
        self.events = [torch.cuda.Event() if self.cuda else None for _ in range(2)]
        self.busy = [False, False]

    def record(self, k):
        if self.cuda:
            self.events[k].record()
            self.busy[k] = True

    def wait(self, k):
        if self.busy[k]:
            self.events[k].synchronize()
            self.busy[k] = False

    def drain(self):
        for k in range(2):
            self.wait(k)


def _npy_header(f, shape, descr="<f8"):
    np.lib.format.write_array_header_1_0(f, {"descr": descr, "fortran_order": False, "shape": tuple(shape)})


def _read_npy_header(f, path):
    major, _ = np.lib.format.read_magic(f)
    if major == 1:
        shape, fortran, dtype = np.lib.format.read_array_header_1_0(f)
    elif major == 2:
        shape, fortran, dtype = np.lib.format.read_array_header_2_0(f)
    else:
        raise ValueError("%s: unsupported .npy format version %d" % (path, major))
    if fortran:
        raise ValueError("%s: Fortran-ordered arrays are not amplitude blocks" % path)
    return tuple(shape), dtype


def _flat_bytes(x):
    return x.view(torch.uint8).reshape(-1)


def _write_blocks(path, x, idx, chunk_bytes):
    """x[idx] (canonical blocks of the device tensor x) as one .npy file, streamed."""
    block_bytes = x[0].numel() * x.element_size() if x.shape[0] else 0
    flat = _flat_bytes(x)
    with open(path, "wb") as f:
        _npy_header(f, (len(idx),) + tuple(x.shape[1:]))
        if not idx or block_bytes == 0:
            return
        st = _Staging(min(chunk_bytes, len(idx) * block_bytes), x.device)
        prev = None
        for i, (off, n) in enumerate(_pieces(_runs(idx), block_bytes, chunk_bytes)):
            k = i % 2
            st.bufs[k][:n].copy_(flat[off:off + n], non_blocking=st.cuda)
            st.record(k)
            if prev is not None:
                st.wait(prev[0])
                f.write(memoryview(st.views[prev[0]][:prev[1]]))
            prev = (k, n)
        st.wait(prev[0])
        f.write(memoryview(st.views[prev[0]][:prev[1]]))


def _read_blocks(path, x, idx, block_shape, chunk_bytes):
    """Fill the canonical blocks idx of x from one rank's .npy file, streamed."""
    with open(path, "rb") as f:
        shape, dtype = _read_npy_header(f, path)
        if dtype != np.dtype("<f8"):
            raise ValueError("%s: dtype %s; the stored amplitudes are float64 ('<f8')" % (path, dtype.str))
        if shape != (len(idx),) + tuple(block_shape):
            raise ValueError("%s: shape %s, expected %s" % (path, shape, (len(idx),) + tuple(block_shape)))
        block_bytes = int(np.prod(block_shape)) * 8
        if not idx or block_bytes == 0:
            return
        flat = _flat_bytes(x)
        st = _Staging(min(chunk_bytes, len(idx) * block_bytes), x.device)
        for i, (off, n) in enumerate(_pieces(_runs(idx), block_bytes, chunk_bytes)):
            k = i % 2
            st.wait(k)
            view = memoryview(st.views[k][:n])
            got = 0
            while got < n:
                m = f.readinto(view[got:])
                if not m:
                    raise ValueError("%s: file ends %d bytes early" % (path, n - got))
                got += m
            flat[off:off + n].copy_(st.bufs[k][:n], non_blocking=st.cuda)
            st.record(k)
        st.drain()


class Checkpoint:
    """What a checkpoint's metadata and per-rank lists say: nocc, nvir, distribution,
    batch_size, dtype, size (the writer's rank count) and rank_tuples (each rank's canonical
    occupied tuples in its file's block order)."""

    def __init__(self, kind, nocc, nvir, distribution, batch_size, dtype, size, rank_tuples):
        self.kind, self.nocc, self.nvir = kind, int(nocc), int(nvir)
        self.distribution, self.batch_size = distribution, batch_size
        self.dtype, self.size, self.rank_tuples = dtype, int(size), rank_tuples

    def __repr__(self):
        return "Checkpoint(%s, nocc=%d, nvir=%d, distribution=%r, batch_size=%r, size=%d)" % (
            self.kind, self.nocc, self.nvir, self.distribution, self.batch_size, self.size)


# kind -> (blocks file stem, tuples file stem, tuple width, canonical tuples, block rank)
_KINDS = {
    "t3": ("t3_local", "ijk_triples", 3, canonical_triples, 3),
    "t4": ("t4_local", "ijkl_quadruples", 4, stored_quadruples, 4),
}


def _as_blocks(x, kind, nocc, nvir):
    if not isinstance(x, torch.Tensor):
        raise TypeError("%s must be a torch tensor" % kind)
    if x.dtype != torch.float64:
        raise TypeError("%s must be float64, got %s" % (kind, x.dtype))
    if not x.is_contiguous():
        raise ValueError("%s must be C-contiguous" % kind)
    tuples = _KINDS[kind][3](nocc)
    rank = _KINDS[kind][4]
    want = (len(tuples),) + (int(nvir),) * rank
    if tuple(x.shape) != want and not (x.dim() == 2 and tuple(x.shape) == (want[0], nvir ** rank)):
        raise ValueError("%s has shape %s; the stored %s blocks are %s" % (kind, tuple(x.shape), kind, want))
    return x.reshape(want), tuples


def _save(kind, x, prefix, nocc, nvir, distribution, batch_size, nranks, rank_tuples, chunk_bytes):
    stem, tstem, width, _, _ = _KINDS[kind]
    x, tuples = _as_blocks(x, kind, nocc, nvir)
    if rank_tuples is None:
        rank_tuples = assign_ranks(tuples, nranks, distribution, batch_size)
    idx = _check_cover(rank_tuples, tuples, "triple" if kind == "t3" else "quadruple")
    for r, ids in enumerate(idx):
        _write_blocks("%s%s_%d.npy" % (prefix, stem, r), x, ids, int(chunk_bytes))
        lst = np.array([tuple(int(v) for v in t) for t in rank_tuples[r]], dtype=np.int32)
        if kind == "t4":
            lst = lst.reshape(-1, width)
        np.save("%s%s_%d.npy" % (prefix, tstem, r), lst)
    meta = {}
    if kind == "t4":
        meta["kind"] = "DistributedT4IJKL"
    meta.update({"nocc": int(nocc), "nvir": int(nvir), "distribution": str(distribution),
                 "batch_size": None if batch_size is None else int(batch_size), "dtype": "<f8",
                 "size": len(rank_tuples)})
    if kind == "t4":
        meta["zero_rule"] = T4_ZERO_RULE
    with open("%smetadata.json" % prefix, "w") as f:
        json.dump(meta, f)
    return Checkpoint(kind, nocc, nvir, distribution, batch_size, "<f8", len(rank_tuples), rank_tuples)


def _read_meta(kind, prefix):
    stem, tstem, width, canon, rank = _KINDS[kind]
    with open("%smetadata.json" % prefix) as f:
        meta = json.load(f)
    if kind == "t4" and meta.get("kind", "DistributedT4IJKL") != "DistributedT4IJKL":
        raise ValueError("%smetadata.json describes %s, not T4" % (prefix, meta.get("kind")))
    if kind == "t4" and meta.get("zero_rule", T4_ZERO_RULE) != T4_ZERO_RULE:
        raise ValueError("T4 zero rule %r is not %r" % (meta.get("zero_rule"), T4_ZERO_RULE))
    if np.dtype(meta["dtype"]) != np.dtype("<f8"):
        raise ValueError("checkpoint dtype %s; the stored amplitudes are float64" % meta["dtype"])
    rank_tuples = []
    for r in range(int(meta["size"])):
        arr = np.load("%s%s_%d.npy" % (prefix, tstem, r))
        rank_tuples.append([tuple(int(v) for v in t) for t in arr.reshape(-1, width)])
    return Checkpoint(kind, meta["nocc"], meta["nvir"], meta["distribution"], meta.get("batch_size"),
                      meta["dtype"], meta["size"], rank_tuples)


def _load(kind, prefix, device, out, chunk_bytes):
    stem, _, _, canon, rank = _KINDS[kind]
    ck = _read_meta(kind, prefix)
    tuples = canon(ck.nocc)
    idx = _check_cover(ck.rank_tuples, tuples, "triple" if kind == "t3" else "quadruple")
    block_shape = (ck.nvir,) * rank
    if out is None:
        out = torch.empty((len(tuples),) + block_shape, dtype=torch.float64, device=device)
    x, _ = _as_blocks(out, kind, ck.nocc, ck.nvir)
    for r, ids in enumerate(idx):
        _read_blocks("%s%s_%d.npy" % (prefix, stem, r), x, ids, block_shape, int(chunk_bytes))
    return ck, out


def save_t3(t3, prefix, nocc, nvir, distribution="balanced", batch_size=None, nranks=1, rank_triples=None,
            chunk_bytes=CHUNK_BYTES):
    """Write the canonical-order t3 [n3, nv, nv, nv] (any device) as the checkpoint of a run of
    `nranks` ranks (distr_cc/distribute_t3.py:959-996).  Returns the Checkpoint."""
    return _save("t3", t3, prefix, nocc, nvir, distribution, batch_size, nranks, rank_triples, chunk_bytes)


def load_t3(prefix, device="cuda", out=None, chunk_bytes=CHUNK_BYTES):
    """(Checkpoint, t3) with t3 [n3, nv, nv, nv] in canonical order on `device` (or in `out`),
    from a checkpoint of any rank count (distr_cc/distribute_t3.py:998-1059)."""
    return _load("t3", prefix, device, out, chunk_bytes)


def save_t4(t4, prefix, nocc, nvir, distribution="balanced", batch_size=None, nranks=1, rank_quadruples=None,
            chunk_bytes=CHUNK_BYTES):
    """Write the stored-order t4 [n4, nv, nv, nv, nv] (the reference's stored blocks without
    the zero-rule ones) as the checkpoint of a run of `nranks` ranks
    (distr_cc/distribute_t4.py:903-925).  Returns the Checkpoint."""
    return _save("t4", t4, prefix, nocc, nvir, distribution, batch_size, nranks, rank_quadruples, chunk_bytes)


def load_t4(prefix, device="cuda", out=None, chunk_bytes=CHUNK_BYTES):
    """(Checkpoint, t4) in stored order on `device` (or in `out`), from a checkpoint of any rank
    count (distr_cc/distribute_t4.py:927-976)."""
    return _load("t4", prefix, device, out, chunk_bytes)
