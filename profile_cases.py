"""Small, self-contained launches of single kernels for profiler captures.

    python profile_cases.py gemm   [--kind bf16x3] [--reps 3] [--nocc 10 --nvir 90]
    python profile_cases.py p3     [--reps 3] [--nvir 90] [--op p3|p3_422|roundtrip|triple|transpose] [--time]
    python profile_cases.py update [--reps 3]
    python profile_cases.py q      [--reps 3]
    python profile_cases.py gather [--reps 3]
    python profile_cases.py xgemm  [--reps 3]
    python profile_cases.py oogemm [--reps 3]
    python profile_cases.py unpack [--reps 3]
    python profile_cases.py qgroup [--reps 3]
    python profile_cases.py t3half [--reps 3] [--nocc 15 --nvir 93] [--kind bf16x3|fp64] [--breakdown]
    python profile_cases.py t4     [--reps 3] [--kind bf16x3|fp64] [--breakdown]
    python profile_cases.py oddnv  [--reps 3] [--nocc 5 --nvir 93] [--time] [--passes 0,1,...]

Each case builds its inputs once and launches the kernel `reps` times, so a
profiler can skip the warm-up launches and capture the last one.  Sizes are
the nocc=10 / nvir=90 workload (inputs larger than L2, a few GB on the device).
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "distributed-cc_b200"))

import torch  # noqa: E402


def case_gemm(kind, reps, nocc=10, nvir=90):
    """One W_vvvv.t3 string (M = n3 nvir rows, N = K = nvir^2) as a split GEMM, `reps` launches."""
    from dcc import contract
    n3, nv = nocc * (nocc + 1) * (nocc + 2) // 6, nvir
    g = torch.Generator(device="cuda").manual_seed(0)
    t3 = torch.randn(n3, nv, nv, nv, dtype=torch.float64, device="cuda", generator=g) * 1e-3
    W = torch.randn(nv, nv, nv, nv, dtype=torch.float64, device="cuda", generator=g) * 0.1
    r3 = torch.zeros_like(t3)
    op = contract.WvvvvT3(n3, nv, kind)
    op.W.fill(W.reshape(nv * nv, nv * nv), contract.lin(nv * nv), contract.lin(1))
    am, ak, er, ec = op.maps[2]
    op.A.fill(t3, am, ak)
    for _ in range(reps):
        contract.gemm_(op.A, op.W, r3, er, ec, 1.0, 1.0, op.status)
    torch.cuda.synchronize()
    assert int(op.status.item()) == 0


def case_p3(reps, nvir=90, op="p3", time=False):
    """A T3 symmetrizer on 1.28 GB of blocks (220 blocks at nvir=90; as many nvir^3 blocks as fit in
    the same bytes otherwise).  op: p3 (P3_full, in place), p3_422, roundtrip (the P3 kernel's tile
    traffic with no arithmetic), triple (triple-sym, three outputs), transpose (transpose-add).
    With time=True every launch is timed with CUDA events after a 256 MB L2 flush and the mean
    of all but the first two is printed with the algorithmic bandwidth."""
    from dcc import _c_rccsdt
    nb = 220 * 90 ** 3 // nvir ** 3
    t3 = torch.randn(nb, nvir, nvir, nvir, dtype=torch.float64, device="cuda")
    outs = [torch.zeros_like(t3) for _ in range(3 if op == "triple" else 1 if op == "transpose" else 0)]
    run, nbytes = {
        "p3": (lambda: _c_rccsdt.t3_spin_summation_inplace_(t3, nb, nvir, "P3_full", -1.0 / 6.0, 1.0), 16),
        "p3_422": (lambda: _c_rccsdt.t3_spin_summation_inplace_(t3, nb, nvir, "P3_422", 1.0, 0.0), 16),
        "roundtrip": (lambda: _c_rccsdt.t3_orbit_roundtrip_(t3, nb, nvir), 16),
        "triple": (lambda: _c_rccsdt.t3_spin_summation_triple_sym_(t3, *outs, nvir), 32),
        "transpose": (lambda: _c_rccsdt.t3_transpose_add_(t3, outs[0] if outs else None, nvir), 16),
    }[op]
    flush = torch.empty(256 << 20, dtype=torch.int8, device="cuda") if time else None
    times = []
    for r in range(reps):
        if time:
            flush.fill_(r & 127)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        run()
        if time:
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    assert _c_rccsdt.symmetrize_status() == 0
    if time and len(times) > 2:
        ms = sum(times[2:]) / len(times[2:])
        print(f"{op} nvir={nvir} blocks={nb}: {ms:.4f} ms, {nbytes * nb * nvir ** 3 / ms * 1e-6:.0f} GB/s "
              f"({nbytes} B per element)")


def case_update(reps):
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(10, 90, seed=0)
    r3 = torch.randn_like(d.t3) * 1e-4
    for _ in range(reps):
        t3_residual.update_t3_(d.t3, r3, d, write_r3=False)
    torch.cuda.synchronize()


def case_q(reps):
    from dcc import _c_rccsdt_q
    no, nv, blk = 10, 90, 4
    g = torch.Generator(device="cuda").manual_seed(0)
    t4 = torch.randn((blk,) * 4 + (no,) * 4, dtype=torch.float64, device="cuda", generator=g) * 1e-3
    z4 = torch.randn_like(t4)
    vvoo = torch.randn(nv, nv, no, no, dtype=torch.float64, device="cuda", generator=g) * 0.1
    t2 = torch.randn(nv, nv, no, no, dtype=torch.float64, device="cuda", generator=g) * 0.01
    eo = torch.linspace(-1.5, -0.3, no, dtype=torch.float64, device="cuda")
    ev = torch.linspace(0.1, 3.0, nv, dtype=torch.float64, device="cuda")
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    for _ in range(reps):
        _c_rccsdt_q.q_task_epilogue(t4, z4, vvoo, t2, eo, ev, (0, 4, 4, 8, 8, 12, 12, 16), blk, no, nv, out)
    torch.cuda.synchronize()


def case_gather(reps, nocc=10):
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(nocc, 90, seed=0)
    tr = t3_residual.T3Residual(nocc, 90, "bf16x3", with_oo=False)
    r3 = torch.empty_like(d.t3)
    S = tr.s_(d, d.t3)  # the split path's S holds -W_vooo.t2 as well: one source
    src = [(S, 1.0, t3_residual.full_strides(nocc, 90), t3_residual.ALL_S3)]
    for _ in range(reps):
        t3_residual.perm_gather_(r3, d.ijk, 90, 0.0, src, nocc=nocc)
    torch.cuda.synchronize()


def case_xgemm(reps, nocc=10):
    """The W_vvvo.t2 GEMM (K = nvir, written into the full-layout S): epilogue-bound."""
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(nocc, 90, seed=0)
    tr = t3_residual.T3Residual(nocc, 90, "bf16x3", with_oo=False)
    for _ in range(reps):
        tr.s_(d, d.t3)
    torch.cuda.synchronize()
    assert tr.status_ok()


def case_oogemm(reps, nocc=6):
    """The K-concatenated OO GEMM and the T1 GEMM at nocc=6 (a few GB on the device)."""
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(nocc, 90, seed=0)
    tr = t3_residual.T3Residual(nocc, 90, "bf16x3", with_oo=True)
    for _ in range(reps):
        tr.s_(d, d.t3)
    torch.cuda.synchronize()
    assert tr.status_ok()


def case_unpack(reps, nocc=10):
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(nocc, 90, seed=0)
    U = torch.empty((nocc ** 3, 90, 90, 90), dtype=torch.float64, device="cuda")
    for _ in range(reps):
        t3_residual.unpack_all_(d.t3, U, nocc, 90)
    torch.cuda.synchronize()


def case_oddnv(reps, nocc=5, nvir=93, time=False, only=None):
    """The memory-bound T3 passes of one half-iteration at an odd nvir (no TMA: 8-byte row
    pitch), each on its own buffers: unpack t3 -> U (every ordering), X = P3_201(U) out of
    place, P3_422(t3) out of place, P3_full(r3) in place, the S3 gather S -> r3, (5) the
    unpack and X in one pass (dcc_t3_unpack_p3), and the X pass through and (6) the X pass
    through the orbit-tile kernel (the strip kernel is the default).  With time=True
    each pass is timed with CUDA events (after a 256 MB L2 flush; mean of reps) and printed with
    its algorithmic bytes and bandwidth.  only: the passes to run (indices into the list
    above, e.g. [1] for the X pass alone; buffers of the others are not allocated)."""
    from dcc import synthetic, t3_residual, _c_rccsdt
    d = synthetic.make_inputs(nocc, nvir, seed=0)
    n3, nu = d.t3.shape[0], nocc ** 3
    only = set(range(7)) if only is None else set(only)
    U = torch.empty((nu, nvir, nvir, nvir), dtype=torch.float64, device="cuda") if only & {0, 1, 4, 5, 6} else None
    X = torch.empty_like(U) if only & {1, 4, 5, 6} else None
    V = torch.empty_like(d.t3) if 2 in only else None
    r3 = torch.randn_like(d.t3) if only & {3, 4} else None
    e3, eu = n3 * nvir ** 3, nu * nvir ** 3
    passes = [
        ("unpack t3->U", lambda: t3_residual.unpack_all_(d.t3, U, nocc, nvir), 8 * (e3 + eu)),
        ("X=P3_201(U)", lambda: _c_rccsdt.t3_spin_summation(U, X, nu, nvir, "P3_201"), 16 * eu),
        ("V=P3_422(t3)", lambda: _c_rccsdt.t3_spin_summation(d.t3, V, n3, nvir, "P3_422"), 16 * e3),
        ("P3_full(r3) in place", lambda: _c_rccsdt.t3_spin_summation_inplace_(r3, n3, nvir, "P3_full", -1.0 / 6.0,
                                                                                1.0), 16 * e3),
        ("gather S->r3", lambda: t3_residual.perm_gather_(
            r3, d.ijk, nvir, 0.0, [(X, 1.0, t3_residual.full_strides(nocc, nvir), t3_residual.ALL_S3)], nocc=nocc),
         8 * (6 * e3 + e3)),
        ("unpack+X one pass", lambda: _c_rccsdt.t3_unpack_p3(d.t3, U, X, nocc, nvir, "P3_201"), 8 * (e3 + 2 * eu)),
        ("X by orbit tiles", lambda: _c_rccsdt.t3_spin_summation(U, X, nu, nvir, "P3_201", kernel=2), 16 * eu),
    ]
    flush = torch.empty(256 << 20, dtype=torch.int8, device="cuda") if time else None
    for n, (name, run, nbytes) in enumerate(passes):
        if n not in only:
            continue
        ts = []
        for r in range(reps):
            if time:
                flush.fill_(r & 127)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
            run()
            if time:
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if time:
            ms = sum(ts) / len(ts)
            print(f"{name:22s} nocc={nocc} nvir={nvir}: {ms:8.3f} ms  {nbytes / 1e9:7.3f} GB  "
                  f"{nbytes / ms * 1e-6:7.0f} GB/s")
    assert _c_rccsdt.symmetrize_status() == 0


def case_splits(reps, nocc=8, nvir=93, time=False):
    """The operand splits of a bf16x3 half-iteration that read the full-layout T3 buffers: the
    two U pieces of the OO GEMMs' B operand and the U operand of the W_oooo GEMM (residual),
    and the per-x pieces of X for the feedback's two column layouts.  With time=True each is
    timed with CUDA events (256 MB L2 flush before each; mean of reps) and printed with its
    algorithmic bytes (8 read + 4 written per element, the pieces' padding included)."""
    from dcc import contract, t3_feedback, t3_residual
    R = t3_residual.T3Residual(nocc, nvir, "bf16x3", device="cuda", with_oo=True)
    R.U.normal_()
    c = contract
    runs = []
    for i, (name, fm, fk) in enumerate(R.plan["oo"]["b"]):
        k = R.oob.pieces[i][1]
        runs.append((f"OO B piece {i}", lambda i=i, fm=fm, fk=fk: R.oob.fill_piece(i, R.U, fm, fk),
                     R.oob.M * (8 * k + 4 * R.oob.pieces[i][2])))
    n = nocc * nvir ** 3
    Uf = R.U.view(nocc * nocc, n)

    def woo():
        k0 = 0
        for i, kk in enumerate(R.woo_pieces):
            R.woob.fill_piece(i, Uf[k0:k0 + kk], c.lin(1), c.lin(n))
            k0 += kk
    runs.append(("W_oooo B", woo, n * (8 * nocc * nocc + 4 * R.woob.Kp)))
    F = t3_feedback.SplitFeedback(nocc, nvir, "bf16x3")
    Xf = R.U.reshape(-1)
    for name in ("vovv", "ooov"):
        tm = F.terms[name]
        pieces, ks, Kp = F.plans[name]
        R1, R2, S1, S2 = tm["kin"]
        B = F._operand(tm["N"], ks, Kp, F._xhi, F._xlo)

        def xs(B=B, tm=tm, pieces=pieces, R1=R1, R2=R2, S1=S1, S2=S2):
            for i, (x0, xc) in enumerate(pieces):
                B.fill_piece(i, Xf[x0 * F.Sx:], tm["fn"], c.three(R1, R2, F.Sx, S1, S2))
        runs.append((f"feedback X ({name})", xs, tm["N"] * (8 * nocc * R1 * R2 + 4 * Kp)))
    flush = torch.empty(256 << 20, dtype=torch.int8, device="cuda") if time else None
    for name, run, nbytes in runs:
        if time:
            run()  # first launch (module load) untimed
        ts = []
        for r in range(reps):
            if time:
                flush.fill_(r & 127)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
            run()
            if time:
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if time:
            ms = sum(ts) / len(ts)
            print(f"{name:22s} nocc={nocc} nvir={nvir}: {ms:8.3f} ms  {nbytes / 1e9:7.3f} GB  "
                  f"{nbytes / ms * 1e-6:7.0f} GB/s")


def case_qgroup(reps, nocc=10):
    """One (Q) task group (a, b, c blocks 0..3, d over all 90 virtuals) on the split path:
    two grouped splits, two grouped GEMMs and the group epilogue per repetition."""
    from dcc import synthetic, rccsdt_q, _c_rccsdt
    nv = 90
    d = synthetic.make_inputs(nocc, nv, seed=0)
    er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
          "vvvv": d.W_vvvv, "oooo": d.W_oooo}
    t2 = d.t2.permute(2, 3, 0, 1).contiguous()
    t3_abc = _c_rccsdt.redistribute_ijk_to_abc(d.t3, nocc, nv)
    del d.t3
    q = rccsdt_q.QEnergy(nocc, nv, 4, "bf16x3")
    g = rccsdt_q.groups(nv, 4)[:1]
    q.prepare(g)
    for _ in range(reps):
        q.run(er, t2, t3_abc, d.e_occ, d.e_vir, g)
    torch.cuda.synchronize()
    assert q.status_ok()


def case_t3iter(reps, nocc, nvir, kind="bf16x3"):
    """T3 iterations (compute_r3_tri with the OO terms, P3_full, divide, update, norms) at a
    given shape, timed with CUDA events after two warm-up iterations; the split precisions
    autotune their W_vvvv GEMMs first.  Prints ms per iteration."""
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(nocc, nvir, seed=0)
    res = t3_residual.T3Residual(nocc, nvir, kind, with_oo=True)
    r3 = torch.empty_like(d.t3)
    norms = torch.empty(2, dtype=torch.float64, device="cuda")
    if kind != "fp64":
        res.tune(d, d.t3)

    def step():
        res.compute(d, d.t3, r3)
        t3_residual.update_t3_(d.t3, r3, d, norms=norms, write_r3=False)

    for _ in range(2):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        step()
    e1.record()
    torch.cuda.synchronize()
    assert res.status_ok()
    print(f"t3iter {kind} nocc={nocc} nvir={nvir} blocks={d.t3.shape[0]}: {e0.elapsed_time(e1) / reps:.2f} ms "
          f"per iteration, peak memory {torch.cuda.max_memory_allocated() / 2**30:.1f} GiB")


def case_t3half(reps, nocc, nvir, kind="bf16x3", breakdown=False, min_ms=1.0):
    """The bench step (the T3 half-iteration: feedback, compute_r3_tri, P3_full, divide, update,
    norms, unified DIIS; bench.Workload) at a given shape: three warm-up steps, then `reps`
    steps timed with CUDA events.  With breakdown, one more step under torch.profiler prints
    the device time of every kernel name (this library's and cuBLAS's / torch's)."""
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import bench
    from dcc.t3_iteration import T3Iteration
    w = bench.Workload(torch, nocc, nvir)
    it = T3Iteration(nocc, nvir, kind)
    if kind != "fp64":
        it.res.tune(w.dd, w.t3_0)
    w.start(it)
    for _ in range(3):
        w.step(it)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        w.step(it)
    e1.record()
    torch.cuda.synchronize()
    assert it.status_ok()
    print(f"t3half {kind} nocc={nocc} nvir={nvir}: {e0.elapsed_time(e1) / max(reps, 1):.2f} ms per step, "
          f"peak memory {torch.cuda.max_memory_allocated() / 2**30:.1f} GiB")
    if breakdown:
        _breakdown(lambda: w.step(it), min_ms=min_ms)


def _breakdown(step, top=40, min_ms=1.0):
    """One more `step` under torch.profiler: the device time and launch count of every kernel
    name (this library's and cuBLAS's / torch's), largest first."""
    from torch.profiler import profile, ProfilerActivity
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step()
        torch.cuda.synchronize()
    tot = {}
    for ev in prof.events():
        if ev.device_type == torch.autograd.DeviceType.CUDA:
            n, t = tot.get(ev.name, (0, 0.0))
            tot[ev.name] = (n + 1, t + ev.device_time_total / 1e3)
    total = sum(t for _, t in tot.values())
    print(f"breakdown: {total:.2f} ms of kernels in one step, {sum(n for n, _ in tot.values())} launches")
    for name, (n, t) in sorted(tot.items(), key=lambda kv: -kv[1][1])[:top]:
        print(f"  {t:9.3f} ms {100 * t / total:5.1f} % x{n:<4d} {name[:150]}")
    # the launches of min_ms or more, in launch order
    seq = [ev for ev in prof.events() if ev.device_type == torch.autograd.DeviceType.CUDA]
    seq.sort(key=lambda ev: ev.time_range.start)
    print(f"launches of {min_ms} ms or more, in order:")
    for i, ev in enumerate(seq):
        if ev.device_time_total >= 1000 * min_ms:
            print(f"  #{i:<4d} {ev.device_time_total / 1e3:8.3f} ms  {ev.name[:70]}")


def case_qsample(nocc, nvir, kind="bf16x3", ngroups=12, blksize=4, dchunk=None):
    """[Q] / (Q) on `ngroups` task groups spread over all groups (as the bench samples them),
    split path and FP64 path on the same inputs: ms and energies of each, printed."""
    from dcc import synthetic, rccsdt_q, _c_rccsdt
    d = synthetic.make_inputs(nocc, nvir, seed=0)
    er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
          "vvvv": d.W_vvvv, "oooo": d.W_oooo}
    t2 = d.t2.permute(2, 3, 0, 1).contiguous()
    t3_abc = _c_rccsdt.redistribute_ijk_to_abc(d.t3, nocc, nvir)
    del d.t3
    G = rccsdt_q.groups(nvir, blksize)
    sample = G[::max(1, len(G) // ngroups)][:ngroups]
    for prec in (kind, "fp64"):
        q = rccsdt_q.QEnergy(nocc, nvir, blksize, prec, dchunk=dchunk)
        q.prepare(sample)
        q.run(er, t2, t3_abc, d.e_occ, d.e_vir, sample[:1])
        q.out.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        q.run(er, t2, t3_abc, d.e_occ, d.e_vir, sample)
        e1.record()
        torch.cuda.synchronize()
        assert q.status_ok()
        print(f"qsample {prec} nocc={nocc} nvir={nvir} groups={len(sample)} dchunk={dchunk}: "
              f"{e0.elapsed_time(e1):.2f} ms, "
              f"E[Q]={float(q.out[0]):.10e} E(Q)={float(q.out[1]):.10e}, "
              f"peak memory {torch.cuda.max_memory_allocated() / 2**30:.1f} GiB")
        del q


def case_t4(reps, kind="bf16x3", breakdown=False):
    """T4 updates at the N2 6-31G shape (nocc=7, nvir=11, 161 stored blocks): compute_r4_tri
    with its OO batch, projector, divide, norms, t4 += r4 (dcc.graph.T4Iteration), eager:
    three warm-up steps, then `reps` steps timed with CUDA events."""
    from dcc import graph, synthetic
    it = graph.T4Iteration(synthetic.make_t4_inputs(7, 11, seed=3), kind)
    for _ in range(3):
        it.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        it.step()
    e1.record()
    torch.cuda.synchronize()
    print(f"t4 {kind} nocc=7 nvir=11: {e0.elapsed_time(e1) / max(reps, 1):.2f} ms per step (eager)")
    if breakdown:
        _breakdown(it.step)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["gemm", "p3", "update", "q", "gather", "xgemm", "oogemm", "unpack", "qgroup",
                                         "t4", "t3iter", "qsample", "t3half", "oddnv", "splits"])
    ap.add_argument("--kind", default="bf16x3")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--nocc", type=int, default=None, help="occupied orbitals (xgemm, oogemm, gather, unpack)")
    ap.add_argument("--nvir", type=int, default=None,
                    help="virtual orbitals (default 90; 93 for oddnv, splits and t3half)")
    ap.add_argument("--op", default="p3", choices=["p3", "p3_422", "roundtrip", "triple", "transpose"],
                    help="p3 case: which symmetrizer")
    ap.add_argument("--time", action="store_true", help="p3 case: print CUDA-event timings")
    ap.add_argument("--dchunk", type=int, default=None, help="qsample case: d-chunk of the split path")
    ap.add_argument("--breakdown", action="store_true", help="t3half / t4 case: per-kernel device times")
    ap.add_argument("--min-ms", type=float, default=1.0, help="t3half breakdown: list the launches this long or longer")
    ap.add_argument("--passes", default=None, help="oddnv case: comma-separated pass indices (default all)")
    a = ap.parse_args()
    if a.case == "gemm":
        case_gemm(a.kind, a.reps, a.nocc or 10, a.nvir or 90)
    elif a.case == "p3":
        case_p3(a.reps, a.nvir or 90, a.op, a.time)
    elif a.case == "update":
        case_update(a.reps)
    elif a.case == "t4":
        case_t4(a.reps, a.kind, a.breakdown)
    elif a.case == "t3iter":
        case_t3iter(a.reps, a.nocc or 10, a.nvir or 90, a.kind)
    elif a.case == "oddnv":
        case_oddnv(a.reps, a.nocc or 5, a.nvir or 93, a.time,
                   [int(x) for x in a.passes.split(",")] if a.passes else None)
    elif a.case == "splits":
        case_splits(a.reps, a.nocc or 8, a.nvir or 93, a.time)
    elif a.case == "t3half":
        case_t3half(a.reps, a.nocc or 15, a.nvir or 93, a.kind, a.breakdown, a.min_ms)
    elif a.case == "qsample":
        case_qsample(a.nocc or 10, a.nvir or 90, a.kind, dchunk=a.dchunk)
    elif a.case in ("gather", "xgemm", "oogemm", "unpack", "qgroup"):
        fn = {"gather": case_gather, "xgemm": case_xgemm, "oogemm": case_oogemm, "unpack": case_unpack,
              "qgroup": case_qgroup}[a.case]
        fn(a.reps, **({} if a.nocc is None else {"nocc": a.nocc}))
    else:
        case_q(a.reps)
    print("ok")


if __name__ == "__main__":
    main()
