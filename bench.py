"""Benchmark: one RCCSDT T3 iteration on the kernel-level synthetic workload
(nocc=10, nvir=90, 220 canonical i<=j<=k blocks of 90^3, FP64 storage).

A step is one pass of the triples hot path over the 220 blocks:
  r3 = compute_r3_tri: W_vvvo.t2 - W_vooo.t2 + F_vv.t3 + OO batch terms
       (W_ovov / W_ovvo / F_oo / W_oooo . t3) + W_vvvv.t3, batched over all
       blocks as one all-S3 source built by split GEMMs + a permutation gather
  r3 <- P3_full(r3, -1/6, 1); r3 /= D; t3 += r3; |r3|^2 (update)
with the large contractions as split-BF16x3 tcgen05 GEMMs (FP32 accumulate,
FP64 storage, denominators, update and norms).  The same step on the plain
FP64 GPU path (cuBLAS DGEMM) is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun): every rank runs an independent replica of the workload
(value = all ranks' iterations / max time).  Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "distributed-cc_b200"))

NOCC, NVIR = 10, 90
Q_BLK, Q_GROUPS = 4, 24  # (Q) task block and the number of sampled task groups
METRIC = "RCCSDT T3 iteration time (mixed split-BF16x3 batched path), nocc=10 nvir=90 synthetic"
UNIT = "s/iter"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def profile_traffic(name):
    """Per-launch DRAM bytes of a kernel from a committed ncu summary (profiles/<name>.md)."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while the timed region runs."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------------- CPU side

def cpu_sample(nblk_sample=2, seed=0):
    """The reference's CPU path of one step on a bounded sample of blocks: the
    reference C helpers (oracle/_ref, OpenMP) for P3 symmetrize and division,
    numpy (BLAS) for the einsums.  Returns seconds for the sample and the
    scale factor to the full 220-block step."""
    import numpy as np
    import ctypes
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    from oracle.oracle import Reference, reference_available, Oracle
    rng = np.random.default_rng(seed)
    no, nv = NOCC, NVIR
    trip = [(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)]
    sample = trip[::len(trip) // nblk_sample][:nblk_sample]
    W_vvvv = rng.standard_normal((nv,) * 4) * 0.1
    W_ovov = rng.standard_normal((no, nv, no, nv)) * 0.1
    W_ovvo = rng.standard_normal((no, nv, nv, no)) * 0.1
    t3_src = rng.standard_normal((3, nv, nv, nv)) * 1e-3  # stand-ins for the batch blocks each l reads
    t3_batch = rng.standard_normal((len(trip) // 10, nv * nv * nv)) * 1e-3
    W_vvvo = rng.standard_normal((nv, nv, nv, no)) * 0.1
    W_vooo = rng.standard_normal((nv, no, no, no)) * 0.1
    F_vv = np.diag(rng.uniform(0.1, 3.0, nv))
    t2 = rng.standard_normal((no, no, nv, nv)) * 1e-2
    t3 = rng.standard_normal((len(sample), nv, nv, nv)) * 1e-3
    eia = rng.uniform(-4.5, -0.4, (no, nv))
    use_ref = reference_available()
    lib = Reference() if use_ref else Oracle()
    e = lambda s, a, b: np.einsum(s, a, b, optimize=True)  # noqa: E731
    t0 = time.perf_counter()
    r3 = np.empty_like(t3)
    for q, (i, j, k) in enumerate(sample):
        r = e('abd,dc->abc', W_vvvo[..., j], t2[i, k])
        r += e('acd,db->abc', W_vvvo[..., k], t2[i, j])
        r += e('bad,dc->abc', W_vvvo[..., i], t2[j, k])
        r += e('bcd,da->abc', W_vvvo[..., k], t2[j, i])
        r += e('cad,db->abc', W_vvvo[..., i], t2[k, j])
        r += e('cbd,da->abc', W_vvvo[..., j], t2[k, i])
        r -= e('al,lbc->abc', W_vooo[:, :, i, j], t2[:, k])
        r -= e('al,lcb->abc', W_vooo[:, :, i, k], t2[:, j])
        r -= e('bl,lac->abc', W_vooo[:, :, j, i], t2[:, k])
        r -= e('bl,lca->abc', W_vooo[:, :, j, k], t2[:, i])
        r -= e('cl,lab->abc', W_vooo[:, :, k, i], t2[:, j])
        r -= e('cl,lba->abc', W_vooo[:, :, k, j], t2[:, i])
        r += e('ad,dbc->abc', F_vv, t3[q])
        r += e('bd,adc->abc', F_vv, t3[q])
        r += e('cd,abd->abc', F_vv, t3[q])
        # OO batch terms: per target block, for every l the four W_ovov/W_ovvo einsums of
        # each of the three parts (distr_cc/rccsdt.py:538-596), plus the transpose-add /
        # triple-sym of the batch blocks (reference C helpers) and the prefactor GEMMs
        for l in range(no):
            T, T2_, V0 = t3_src[0], t3_src[1], t3_src[2]
            for occ in (i, j, k):
                r -= e('bd,dca->abc', W_ovov[l, :, occ, :], T)
                r -= 0.5 * e('ad,dcb->abc', W_ovov[l, :, occ, :], T2_)
                r -= e('cd,bda->abc', W_ovov[l, :, occ, :], T)
                r += 0.5 * e('ad,bcd->abc', W_ovvo[l, :, :, occ], V0)
        pf = rng.standard_normal((6, t3_batch.shape[0]))
        for m in range(6):  # 'pq,pabc->qabc' column of one target block, on a tenth of the batch
            r += (10.0 * (pf[m] @ t3_batch)).reshape(nv, nv, nv)
        r += e('abde,dec->abc', W_vvvv, t3[q])
        r += e('acde,dbe->abc', W_vvvv, t3[q])
        r += e('bcde,ade->abc', W_vvvv, t3[q])
        r3[q] = r
    # per-step helper work on the batch blocks, scaled to this sample's share of blocks
    for q in range(len(sample)):
        blk = np.ascontiguousarray(t3[q])
        if use_ref:
            b0, b1, b2, b3 = (np.empty_like(blk) for _ in range(4))
            lib.t3_transpose_add_(blk.ctypes.data_as(ctypes.c_void_p), b0.ctypes.data_as(ctypes.c_void_p), nv)
            lib.t3_spin_summation_triple_sym_(blk.ctypes.data_as(ctypes.c_void_p), b1.ctypes.data_as(ctypes.c_void_p),
                                              b2.ctypes.data_as(ctypes.c_void_p), b3.ctypes.data_as(ctypes.c_void_p),
                                              nv)
    for q in range(len(sample)):
        blk = np.ascontiguousarray(r3[q])
        if use_ref:
            lib.t3_single_spin_summation_inplace_(blk.ctypes.data_as(ctypes.c_void_p), nv, b"P3_full",
                                                  -1.0 / 6.0, 1.0)
        else:
            lib.t3_spin_sum(blk, nv, "P3_full", -1.0 / 6.0, 1.0)
        i, j, k = sample[q]
        blk /= eia[i][:, None, None] + eia[j][None, :, None] + eia[k][None, None, :]
        t3[q] += blk
    float(np.sum(r3 ** 2))
    dt = time.perf_counter() - t0
    kind = "reference" if use_ref else "port"
    return dt, len(trip) / len(sample), kind, len(sample)


def iteration_energy_proxy(d, r_ref, r_mix):
    """How the split path's error in one T3 iteration reaches the correlation energy.

    Both residuals go through the same update (P3_full, divide, t3 += r3); the difference of the
    two new T3 is fed to the T2 residual by the T3 -> r2 strings (distr_cc/rccsdt.py:300-316, FP64)
    and, divided by the T2 denominators, to E = sum (2<ij|ab> - <ij|ba>) t2.  The same chain on the
    FP64 T3 itself gives the triples' share of E.  r3 is linear in (t2, t3), so the ratio of the
    two is independent of the amplitudes' scale: abs_dE_at_10mEh is the error of a molecule whose
    triples contribute 10 mEh (the synthetic amplitudes are far larger than a molecule's)."""
    import torch
    from dcc import t3_feedback, t3_residual
    no, nv = d.nocc, d.nvir
    ws = torch.empty(1 << 16, dtype=torch.float64, device="cuda")
    t3f, t3m = d.t3.clone(), d.t3.clone()
    t3_residual.update_t3_(t3f, r_ref.clone(), d, workspace=ws)
    t3_residual.update_t3_(t3m, r_mix.clone(), d, workspace=ws)
    E_vovv = d.W_vvvo.permute(2, 3, 0, 1)  # <cx|ad> = <ad|cx>
    E_ooov = d.W_vooo.permute(3, 2, 1, 0)  # <zx|la> = <al|xz>
    D2 = (d.e_occ[:, None, None, None] + d.e_occ[None, :, None, None]
          - d.e_vir[None, None, :, None] - d.e_vir[None, None, None, :])
    L = 2.0 * d.eris_vvoo.permute(2, 3, 0, 1) - d.eris_vvoo.permute(2, 3, 1, 0)  # [i,j,a,b]

    def energy(t3):
        X = t3_feedback.p3_201_all(t3, no)
        r2 = torch.einsum('cxad,xyzdba->yzbc', E_vovv, X) - torch.einsum('zxla,xyzabc->ylbc', E_ooov, X)
        del X
        return float((L * (r2 + r2.permute(1, 0, 3, 2)) / 2 / D2).sum())

    e_t3 = energy(t3f)
    de = energy(t3m - t3f)
    del t3f, t3m
    return {"e_t3_share_fp64": e_t3, "abs_dE": abs(de), "relative": abs(de / e_t3),
            "abs_dE_at_10mEh": abs(de / e_t3) * 1e-2}


def reference_arm(args, rank, world):
    """`--impl reference`: the reference's CPU path on this host's cores."""
    if rank != 0:
        return 0
    times = []
    nblk = 2
    for s in range(args.warmup + args.steps):
        dt, scale, kind, n = cpu_sample(nblk, seed=s)
        if s >= args.warmup:
            times.append(dt * scale)
    v = statistics.mean(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded numpy; e_occ U[-1.5,-0.3], e_vir U[0.1,3.0], t2 N(0,1e-2), ERIs N(0,0.1) 8-fold symmetric)",
            "config": {"workload": "rccsdt_t3_iteration", "nocc": NOCC, "nvir": NVIR, "n_blocks": 220},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
                             "sample": "%d of 220 blocks per step, scaled by 220/%d; reference C helpers (OpenMP) for "
                                       "P3/divide, numpy+BLAS einsums" % (n, n)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- GPU side

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dcc", choices=["dcc", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "tf32x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-path comparison (profiling runs)")
    ap.add_argument("--no-q", action="store_true", help="skip the (Q) energy sample")
    ap.add_argument("--no-t4", action="store_true", help="skip the T4 update at the N2 6-31G shape")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference's CPU path needs no GPU and no process group: rank 0 alone runs it
        return reference_arm(args, rank, world)
    import torch
    from dcc import ranks
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    torch.cuda.set_device(local)
    from dcc import synthetic, t3_residual, contract

    d = synthetic.make_inputs(NOCC, NVIR, seed=0)
    n3 = d.t3.shape[0]
    mixed = t3_residual.T3Residual(NOCC, NVIR, args.precision, with_oo=True)
    fp64 = None if args.no_fp64 else t3_residual.T3Residual(NOCC, NVIR, "fp64", with_oo=True)
    r3 = torch.empty_like(d.t3)
    t3w = d.t3.clone()
    norms = torch.empty(2, dtype=torch.float64, device="cuda")
    ws = torch.empty(1 << 16, dtype=torch.float64, device="cuda")

    # accuracy of the split path against the FP64 path on identical inputs
    rel_err = None
    energy_proxy = None
    if fp64 is not None:
        r_ref = fp64.compute(d, d.t3)
        r_mix = mixed.compute(d, d.t3)
        torch.cuda.synchronize()
        rel_err = float((r_mix - r_ref).abs().max() / r_ref.abs().max())
        energy_proxy = iteration_energy_proxy(d, r_ref, r_mix)
        del r_ref, r_mix

    def barrier():
        ranks.barrier("cuda")

    def step(res):
        res.compute(d, t3w, r3)
        t3_residual.update_t3_(t3w, r3, d, norms=norms, workspace=ws, write_r3=False)

    # live timing of the dominant kernel (the W_vvvv.t3 split GEMM launches)
    gemm_ev = []
    orig_gemm = contract.gemm_

    def timed_gemm(A, B, C, frow, fcol, alpha=1.0, beta=1.0, status=None, Kp=None):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st = orig_gemm(A, B, C, frow, fcol, alpha, beta, status, Kp)
        e1.record()
        if A.M == mixed.wvvvv.A.M and B.M == mixed.wvvvv.W.M:
            gemm_ev.append((e0, e1))
        return st

    def timed_run(res, steps, warmup, track=False):
        for _ in range(warmup):
            step(res)
        barrier()
        if track:
            contract.gemm_ = timed_gemm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            step(res)
        e1.record()
        barrier()
        contract.gemm_ = orig_gemm
        return ranks.max_over_ranks(e0.elapsed_time(e1), "cuda")

    # pipeline shape of the W_vvvv.t3 GEMMs chosen by the autotuner (untimed, like planning)
    from dcc import autotune
    tuned = mixed.tune(d, t3w)

    # this library's kernels per mixed step, counted on one untimed step
    from torch.profiler import profile, ProfilerActivity
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step(mixed)
        torch.cuda.synchronize()
    launches_per_step = sum(1 for ev in prof.events()
                            if ev.device_type == torch.autograd.DeviceType.CUDA and "dcc::" in ev.name)
    del prof

    with ClockSampler(local) as clk:
        ms_mixed = timed_run(mixed, args.steps, args.warmup, track=True)
    ok = mixed.status_ok()
    fp64_steps = max(2, args.steps // 3)
    ms_fp64 = timed_run(fp64, fp64_steps, 3) if fp64 is not None else None

    # the same step captured as one CUDA graph (the synthetic W_oooo has the RHF pair symmetry)
    from dcc import graph as dgraph
    mixed.woooo_pair_symmetric = True
    t3g = d.t3.clone()
    gstep = dgraph.T3IterationGraph(mixed, d, t3g, r3=r3, norms=norms, workspace=ws)
    for _ in range(2):
        gstep.replay()
    barrier()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    for _ in range(args.steps):
        gstep.replay()
    g1.record()
    barrier()
    graph_ms = ranks.max_over_ranks(g0.elapsed_time(g1), "cuda") / args.steps
    graph_ok = gstep.status_ok()
    del gstep, t3g
    mixed.woooo_pair_symmetric = False

    gemm_ms = [a.elapsed_time(b) for a, b in gemm_ev]
    gemm_avg = statistics.mean(gemm_ms) if gemm_ms else None
    flops_launch = 2.0 * n3 * NVIR ** 5  # one of the three W_vvvv.t3 strings
    hbm, bf16, bf16_sus, src = peaks()
    peak_useful = bf16_sus / 3.0  # three bf16 products per FP64-equivalent flop
    achieved = flops_launch / (gemm_avg * 1e-3) / 1e12 if gemm_avg else None

    # e2e through the public API: every step's inputs (t2 and the intermediates, which the
    # lower-order equations rebuild on the host each iteration) come from pinned host memory and
    # the step's result (the residual norms) is read back; t3 stays resident on the device, as
    # it stays in each rank's memory in the reference.  The uploads run on a copy stream
    # (e2e_step) and overlap the parts of the step that do not need them.
    host = {k: getattr(d, k).cpu().pin_memory() for k in
            ("t2", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo", "F_vv", "F_oo", "eia")}
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    norms_host = torch.empty(2, dtype=torch.float64).pin_memory()
    d2h = norms_host.numel() * 8

    class Dev:
        pass

    dd = Dev()
    dd.ijk = d.ijk
    for k, v in host.items():
        setattr(dd, k, torch.empty(v.shape, dtype=v.dtype, device="cuda"))
    t3e = d.t3.clone()
    side = torch.cuda.Stream()
    in_ready, w_ready, in_free = torch.cuda.Event(), torch.cuda.Event(), torch.cuda.Event()
    in_free.record()

    def e2e_step():
        # one copy stream, the small inputs first: they arrive while the unpack of t3 (which
        # needs none of them) runs, and W_vvvv (0.52 GB) streams on while the W.t2 / OO terms run
        side.wait_event(in_free)  # the previous step is done with the input buffers
        with torch.cuda.stream(side):
            for k, v in host.items():
                if k != "W_vvvv":
                    getattr(dd, k).copy_(v, non_blocking=True)
            in_ready.record(side)
            dd.W_vvvv.copy_(host["W_vvvv"], non_blocking=True)
            w_ready.record(side)
        mixed.compute(dd, t3e, r3, wvvvv_ready=w_ready, inputs_ready=in_ready)
        t3_residual.update_t3_(t3e, r3, dd, norms=norms, workspace=ws, write_r3=False)
        in_free.record()
        norms_host.copy_(norms, non_blocking=True)

    for _ in range(2):
        e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(2, args.steps // 2)
    e0.record()
    in_free.record()  # the first timed step's uploads start after e0
    for _ in range(e2e_steps):
        e2e_step()
    e1.record()
    barrier()
    e2e_ms_max = ranks.max_over_ranks(e0.elapsed_time(e1), "cuda")
    e2e_ms = e2e_ms_max / e2e_steps

    # (Q): [Q]/(Q) energies on a sample of task groups (every group = the tasks sharing
    # (a, b, c) blocks), split path and FP64 path, scaled to all tasks by task count
    q_line = None
    if not args.no_q:
        from dcc import rccsdt_q, _c_rccsdt
        er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
              "vvvv": d.W_vvvv, "oooo": d.W_oooo}
        t2q = d.t2.permute(2, 3, 0, 1).contiguous()
        t3_abc = _c_rccsdt.redistribute_ijk_to_abc(d.t3, NOCC, NVIR)
        G = rccsdt_q.groups(NVIR, Q_BLK)
        sample = G[::max(1, len(G) // Q_GROUPS)][:Q_GROUPS]
        ntask = len(rccsdt_q.task_list(NVIR, Q_BLK))
        nsample = sum(len(rccsdt_q.prange(g[4], NVIR, Q_BLK)) for g in sample)
        q_line = {"blksize": Q_BLK, "tasks": ntask, "sample_groups": len(sample), "sample_tasks": nsample}
        for prec in (args.precision, "fp64"):
            q = rccsdt_q.QEnergy(NOCC, NVIR, Q_BLK, prec)
            q.prepare(sample)  # grouped tables of every sampled group shape, outside the timed region
            q.run(er, t2q, t3_abc, d.e_occ, d.e_vir, sample[:1])  # warm-up
            q.out.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            q.run(er, t2q, t3_abc, d.e_occ, d.e_vir, sample)
            e1.record()
            barrier()
            ms = e0.elapsed_time(e1)
            q_line[prec] = {"s_sample": ms / 1e3, "s_all_tasks_est": ms / 1e3 * ntask / nsample,
                            "e_bracket_sample": float(q.out[0]), "e_paren_sample": float(q.out[1]),
                            "status_ok": q.status_ok()}
        q_line["speedup_vs_fp64"] = q_line["fp64"]["s_sample"] / q_line[args.precision]["s_sample"]
        q_line["abs_dE_paren_sample"] = abs(q_line["fp64"]["e_paren_sample"] - q_line[args.precision]["e_paren_sample"])
        # the synthetic amplitudes give energies of O(10) Eh: the same sample with t2 and t3 scaled by
        # one factor s so that the FP64 (Q) energy is -1e-3 Eh (a molecular (Q) correction), untimed
        s = (1e-3 / max(abs(q_line["fp64"]["e_paren_sample"]), 1e-300)) ** 0.5
        ms_line = {"amplitude_scale": s}
        for prec in (args.precision, "fp64"):
            q = rccsdt_q.QEnergy(NOCC, NVIR, Q_BLK, prec)
            q.prepare(sample)
            q.run(er, t2q * s, t3_abc * s, d.e_occ, d.e_vir, sample)
            ms_line[prec] = {"e_bracket_sample": float(q.out[0]), "e_paren_sample": float(q.out[1]),
                             "status_ok": q.status_ok()}
        ms_line["abs_dE_bracket"] = abs(ms_line["fp64"]["e_bracket_sample"] - ms_line[args.precision]["e_bracket_sample"])
        ms_line["abs_dE_paren"] = abs(ms_line["fp64"]["e_paren_sample"] - ms_line[args.precision]["e_paren_sample"])
        q_line["molecule_scale"] = ms_line
        del t3_abc

    # One T4 update (compute_r4_tri with its OO batch, projector, divide, norms, t4 += r4) at the
    # N2 6-31G shape (nocc=7, nvir=11, 161 stored blocks): eager and replayed as one CUDA graph.
    t4_line = None
    if not args.no_t4:
        from dcc import graph as dgraph, synthetic as dsyn
        t4_line = {"nocc": 7, "nvir": 11, "stored_blocks": 161}

        def t4_ms(fn, n=5):
            for _ in range(3):
                fn()
            barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(n):
                fn()
            b.record()
            barrier()
            return ranks.max_over_ranks(a.elapsed_time(b), "cuda") / n

        for prec in (args.precision, "fp64"):
            it = dgraph.T4Iteration(dsyn.make_t4_inputs(7, 11, seed=3), prec)
            t4_line[prec] = {"eager_ms": t4_ms(it.step)}
            del it
            gt4 = dgraph.T4IterationGraph(dgraph.T4Iteration(dsyn.make_t4_inputs(7, 11, seed=3), prec))
            t4_line[prec]["graph_ms"] = t4_ms(gt4.replay)
            del gt4
        d4 = dsyn.make_t4_inputs(7, 11, seed=3)
        r4s = {}
        from dcc import t4_residual as dt4
        for prec in (args.precision, "fp64"):
            r4s[prec] = torch.zeros_like(d4.t4)
            dt4.compute_r4_tri_(r4s[prec], d4.eris, d4.F_vv, d4.W_vvvo, d4.W_vooo, d4.W_vvvv, d4.W_oooo,
                                d4.W_ovov, d4.t2, d4.t3, d4.t4, 7, prec, F_oo=d4.F_oo, W_ovvo=d4.W_ovvo)
        t4_line["r4_max_rel_err_vs_fp64"] = float((r4s[args.precision] - r4s["fp64"]).abs().max()
                                                  / r4s["fp64"].abs().max())
        del d4, r4s

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        dt, scale, kind, n = cpu_sample(2)
        cpu = {"value": dt * scale, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
               "sample": "%d of 220 blocks of one step, scaled by 220/%d; reference C helpers (OpenMP) for "
                         "P3/divide/transpose-add/triple-sym + numpy/BLAS einsums" % (n, n)}

    value = ranks.job_seconds_per_iteration(ms_mixed, args.steps, world)  # whole job, replicas
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_mixed / args.steps, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 storage; " + args.precision + " products, f32 accumulate",
        "data": "synthetic (seeded torch generator; e_occ U[-1.5,-0.3], e_vir U[0.1,3.0], t2 N(0,1e-2), ERIs N(0,0.1) 8-fold symmetric)",
        "config": {"workload": "rccsdt_t3_iteration", "nocc": NOCC, "nvir": NVIR, "n_blocks": n3,
                   "terms": "compute_r3_tri (W_vvvo.t2, W_vooo.t2, F_vv.t3, OO W_ovov/W_ovvo/F_oo/W_oooo.t3, "
                            "W_vvvv.t3), P3_full, divide, update, norms",
                   "precision": args.precision, "l2": "inputs larger than L2 (t3 1.28 GB, W_vvvv 0.52 GB)",
                   "parallelism": "replicas" if world > 1 else "single"},
        "fp64_path_s_per_iter": ms_fp64 / fp64_steps / 1e3 if ms_fp64 else None,
        "speedup_vs_fp64": (ms_fp64 / fp64_steps) / (ms_mixed / args.steps) if ms_fp64 else None,
        "r3_max_rel_err_vs_fp64": rel_err, "iteration_energy_error": energy_proxy, "device_status_ok": ok,
        "cuda_graph_ms_per_step": graph_ms, "cuda_graph_status_ok": graph_ok,
        "wvvvv_gemm_pipeline": None if tuned is None else {
            "kb_bytes": tuned[0], "stages": tuned[1], "group_m": tuned[2], "chosen_by": "dcc.autotune",
            "candidates_ms": {"%d/%d/%d" % c: round(ms, 4) for c, ms in
                              (autotune.timings(mixed.wvvvv.key()) or {}).items()}},
        "roofline": {"kernel": "dcc::k_gemm_split3<0> (W_vvvv.t3 string)", "bound": "tensor",
                     "achieved": achieved, "peak": peak_useful, "unit": "TFLOP/s",
                     "frac": (achieved / peak_useful) if achieved else None,
                     "peak_note": "bf16 dense %s sustained %.1f TF/s / 3 products (of %s)" % (src, bf16_sus, src),
                     "flops_per_launch": flops_launch, "launch_ms": gemm_avg,
                     "traffic": profile_traffic("gemm_split3_wvvvv_nocc10_nvir90")},
        "cpu_baseline": cpu,
        "e2e": {"value": ranks.job_seconds_per_iteration(e2e_ms_max, e2e_steps, world), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step * args.steps,
        "q_energy": q_line,
        "t4_iteration": t4_line,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
