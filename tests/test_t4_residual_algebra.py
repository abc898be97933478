"""compute_r4_tri without its OO batch: dcc.t4_residual's formulation (every per-block
string as one contraction batched over the stored blocks, its operands cut at each
block's occupied slots; the W builders over every ordering of (i,j,k,l), W_oovvvv kept
for every ordered pair) against the oracle's literal per-block loop (oracle/t4_ref.py),
in FP64 on the CPU, relative 1e-12.  The P3_201 / P4_201 spin summations are the
oracle's C restatement here (the GPU path uses this library's kernels, checked bit for
bit elsewhere)."""
import numpy as np
import pytest
import torch

from oracle import t4_ref
from dcc import t4_residual as tr


def _inputs(no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    r = lambda *s, sc=0.1: rng.standard_normal(s) * sc  # noqa: E731
    return dict(eris=r(nmo, nmo, nmo, nmo), F_vv=r(nv, nv), W_vvvo=r(nv, nv, nv, no), W_vooo=r(nv, no, no, no),
                W_vvvv=r(nv, nv, nv, nv), W_oooo=r(no, no, no, no), W_ovov=r(no, nv, no, nv),
                t2=r(no, no, nv, nv, sc=0.05), t3=r(no, no, no, nv, nv, nv, sc=0.01),
                t4=r(len(t4_ref.stored_quadruples(no)), nv, nv, nv, nv, sc=0.01))


@pytest.mark.parametrize("no,nv", [(4, 3), (5, 4)])
def test_full_space_r4_matches_literal_blocks(oracle, no, nv):
    d = _inputs(no, nv, 3 + no)
    want = t4_ref.compute_r4_tri_ref(d["eris"], d["F_vv"], d["W_vvvo"], d["W_vooo"], d["W_vvvv"], d["W_oooo"],
                                     d["W_ovov"], d["t2"], d["t3"], d["t4"], no, oracle)

    def spin(pattern, n):
        def f(A):
            a = A.numpy()
            if n == 3:
                oracle.t3_spin_sum(a, nv, pattern, 1.0, 0.0)
            else:
                oracle.t4_spin_sum(a, a.size // nv ** 4, nv, pattern, 1.0, 0.0)
            return A
        return f

    t = {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in d.items()}
    r4 = torch.zeros_like(t["t4"])
    tr.compute_r4_tri_(r4, t["eris"], t["F_vv"], t["W_vvvo"], t["W_vooo"], t["W_vvvv"], t["W_oooo"], t["W_ovov"],
                       t["t2"], t["t3"], t["t4"], no, "fp64", spin3=spin("P3_201", 3), spin4=spin("P4_201", 4))
    np.testing.assert_allclose(r4.numpy(), want, rtol=1e-12, atol=1e-14 * np.abs(want).max())


def test_unpack_all_orderings_matches_oracle(oracle):
    no, nv = 4, 3
    quads = tr.stored_quadruples(no)
    assert quads == t4_ref.stored_quadruples(no)
    rng = np.random.default_rng(1)
    t4 = rng.standard_normal((len(quads),) + (nv,) * 4)
    nfull = no * (no + 1) * (no + 2) * (no + 3) // 24
    f2l = np.full(nfull, -1, dtype=np.int64)
    for n, q in enumerate(quads):
        f2l[oracle.ijkl_to_linear(*q, no)] = n
    full = tr.unpack_all_orderings(torch.from_numpy(t4), no).numpy()
    import itertools
    for o in itertools.product(range(no), repeat=4):
        want, rc = oracle.unpack_t4(t4, f2l, *o, no, nv)
        assert np.array_equal(full[o], want), o


def stab_symmetric(t4, quads):
    """Each stored block averaged over the virtual-axis permutations that fix its occupied
    tuple (i = j, k = l, ...): the symmetry every T4 block has, which the reference's
    prefactor slots rely on when they read a block in another ordering."""
    import itertools
    out = np.empty_like(t4)
    for q, quad in enumerate(quads):
        ps = [p for p in itertools.permutations(range(4)) if tuple(quad[x] for x in p) == quad]
        out[q] = sum(t4[q].transpose(p) for p in ps) / len(ps)
    return out


@pytest.mark.parametrize("no,nv", [(4, 3), (5, 3)])
def test_oo_batch_matches_literal_blocks(oracle, no, nv):
    rng = np.random.default_rng(no)
    n4 = len(t4_ref.stored_quadruples(no))
    t4 = stab_symmetric(rng.standard_normal((n4,) + (nv,) * 4) * 0.01, t4_ref.stored_quadruples(no))
    F_oo = rng.standard_normal((no, no))
    W_oooo = rng.standard_normal((no,) * 4) * 0.1
    W_ovvo = rng.standard_normal((no, nv, nv, no)) * 0.1
    W_ovov = rng.standard_normal((no, nv, no, nv)) * 0.1
    r0 = rng.standard_normal(t4.shape) * 0.01
    want = t4_ref.oo_batch_ref(r0.copy(), t4, F_oo, W_oooo, W_ovvo, W_ovov, no, oracle)

    def forms(t):
        a = t.numpy()
        T3 = np.stack([oracle.t4_transpose_add(np.ascontiguousarray(b), nv) for b in a])
        Vs = [oracle.t4_quadruple_sym(np.ascontiguousarray(b), nv) for b in a]
        return torch.from_numpy(T3), [torch.from_numpy(np.stack([v[x] for v in Vs])) for x in range(4)]

    tt = lambda a: torch.from_numpy(np.ascontiguousarray(a))  # noqa: E731
    r4 = tt(r0.copy())
    tr.oo_batch_(r4, tt(t4), tt(F_oo), tt(W_oooo), tt(W_ovvo), tt(W_ovov), no, forms=forms)
    np.testing.assert_allclose(r4.numpy(), want, rtol=1e-12, atol=1e-13 * np.abs(want - r0).max())


def _emulate_fused(desc, quads, ops, nv, pairs=None):
    """The fused strings kernel (dcc_t4_strings) in numpy: every descriptor read through
    strided views of the operands, with the kernel's bounds checks, one stored block at a
    time; pair-mode descriptors once per (source block, m) pair of the block's list."""
    nq = len(quads)
    r4 = np.zeros((nq,) + (nv,) * 4)
    flat = [np.ascontiguousarray(o).reshape(-1) for o in ops]
    for q, occ in enumerate(quads):
        for d in desc:
            wop, top, mask, mode = d[0], d[1], d[20], d[31]
            K0, K1 = d[21], d[24]
            alpha = np.frombuffer(np.int64(d[27]).tobytes(), dtype=np.float64)[0]
            ext = (nv, nv, nv, nv, K0, K1)
            for x in range(4):  # each output letter in exactly one operand
                assert (d[12 + x] == 0) if not (mask >> x) & 1 else (d[16 + x] == 0)
            # the row / column orders list W's and T's output letters once each
            rows = [(d[28] >> (4 * p) & 15) - 1 for p in range(4)]
            cols = [(d[29] >> (4 * p) & 15) - 1 for p in range(4)]
            assert sorted(x for x in rows if x >= 0) == [x for x in range(4) if mask >> x & 1]
            assert sorted(x for x in cols if x >= 0) == [x for x in range(4) if not mask >> x & 1]
            if mode:
                off, sm = pairs
                plist = [tuple(sm[p]) for p in range(off[q][mode - 1], off[q][mode])]
            else:
                plist = [(q, 0)]
            for src, m in plist:
                views = []
                for op, sl, qs, vs, k, extra in ((wop, d[2:6], d[10], d[12:16], (d[22], d[25]), d[30] * m),
                                                 (top, d[6:10], d[11], d[16:20], (d[23], d[26]), 0)):
                    base = sum(int(s) * int(o) for s, o in zip(sl, occ)) + int(qs) * (src if op == top else q)
                    base += int(extra)
                    st = [int(x) for x in vs] + [int(x) for x in k]
                    assert all(x >= 0 for x in st)
                    assert base + sum(s * (e - 1) for s, e in zip(st, ext)) < flat[op].size
                    views.append(np.lib.stride_tricks.as_strided(flat[op][base:], ext, [8 * x for x in st]))
                W, T = views
                # a letter absent from an operand has stride 0 there: multiply and sum over k0, k1
                r4[q] += alpha * np.einsum("abcdxy,abcdxy->abcd", W, T)
    return r4


def _fused_ops(t, no, nv, oracle, spin, oo):
    t3p = t["t3"].clone()
    spin("P3_201", 3)(t3p)
    W = tr.build_intermediates(t["eris"], t["W_oooo"], t["W_ovov"], t["W_vvvv"], t["t2"], t["t3"], t3p, t["t4"], no,
                               spin("P4_201", 4))
    W["W_vvvo"], W["W_vooo"] = t["W_vvvo"], t["W_vooo"]
    ops = dict(W, t3=t["t3"], t3p=t3p, t3s=t["t3"] + t["t3"].permute(0, 1, 2, 4, 5, 3), t2=t["t2"],
               Wf=tr.w_with_f(t["W_vvvv"], t["F_vv"]), W_vvvv=t["W_vvvv"], t4=t["t4"])
    if oo:
        a = t["t4"].numpy()
        Vs = [oracle.t4_quadruple_sym(np.ascontiguousarray(b), nv) for b in a]
        ops.update(F_oo=t["F_oo"], W_oooo=t["W_oooo"], T4full=tr.unpack_all_orderings(t["t4"], no),
                   W_ovov=t["W_ovov"], W_voov=t["W_ovvo"].permute(1, 0, 3, 2),
                   T3=torch.from_numpy(np.stack([oracle.t4_transpose_add(np.ascontiguousarray(b), nv) for b in a])),
                   **{"V%d" % x: torch.from_numpy(np.stack([v[x] for v in Vs])) for x in range(4)})
    return {k: v.contiguous() for k, v in ops.items()}


def _spin(oracle, nv):
    def spin(pattern, n):
        def f(A):
            a = A.numpy()
            if n == 3:
                oracle.t3_spin_sum(a, nv, pattern, 1.0, 0.0)
            else:
                oracle.t4_spin_sum(a, a.size // nv ** 4, nv, pattern, 1.0, 0.0)
            return A
        return f
    return spin


@pytest.mark.parametrize("no,nv,oo", [(4, 3, False), (5, 4, False), (4, 3, True), (5, 3, True)])
def test_fused_descriptors_emulated(oracle, no, nv, oo):
    """The descriptor table and pair lists of the fused strings kernel (every string of the
    per-block loop, the F_vv / W_vvvv strings, and with oo the whole OO batch: its F_oo /
    W_oooo slots over the unpacked T4, its W_ovov / W_voov strings in pair mode),
    interpreted in numpy, against the oracle's literal per-block compute_r4_tri:
    relative 1e-12."""
    d = _inputs(no, nv, 5 + no)
    quads = t4_ref.stored_quadruples(no)
    extra = ()
    if oo:
        rng = np.random.default_rng(no)
        d["t4"] = stab_symmetric(d["t4"], quads)
        d["F_oo"] = rng.standard_normal((no, no))
        d["W_ovvo"] = rng.standard_normal((no, nv, nv, no)) * 0.1
        extra = (d["F_oo"], d["W_ovvo"])
    want = t4_ref.compute_r4_tri_ref(d["eris"], d["F_vv"], d["W_vvvo"], d["W_vooo"], d["W_vvvv"], d["W_oooo"],
                                     d["W_ovov"], d["t2"], d["t3"], d["t4"], no, oracle, *extra)
    t = {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in d.items()}
    ops = _fused_ops(t, no, nv, oracle, _spin(oracle, nv), oo)
    desc, q, names, pairs = tr.fused_plan(no, nv, True, "cpu", oo=oo)
    n_oo = len(tr._OO_PLAIN) + sum(len(tr._OO_TABLE[g][c]) for g, c in tr.oo_pairs(no)) if oo else 0
    assert len(desc) == len(tr._R4_STRINGS) + len(tr.STRINGS) + n_oo
    if oo:
        off, sm = pairs[0].numpy(), pairs[1].numpy()
        assert off[-1, -1] == sum(len(v[0]) for v in tr.oo_pairs(no).values()) == len(sm)
        pairs = (off, sm)
    got = _emulate_fused(desc.numpy(), q.numpy(), [ops[n].numpy() for n in names], nv, pairs)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-14 * np.abs(want).max())
