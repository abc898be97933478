"""Benchmark: the T3 half of one RCCSDT iteration at the benzene cc-pVDZ shape
(nocc=15, nvir=93: 680 canonical i<=j<=k blocks of 93^3, 4.4 GB of T3 in FP64).

A step is every T3 step of one iteration of the reference's RCCSDT loop
(distr_cc/rccsdt.py:916-971 and :1026-1067), on T3 resident in HBM:
  feedback   T3 -> r1, r2 (r1r2_add_t3_tri_) and T3 -> W_vooo, W_vvvo
             (intermediates_t3_add_t3_tri)
  residual   r3 = compute_r3_tri: W_vvvo.t2 - W_vooo.t2 + F_vv.t3 + the OO
             batch (W_ovov / W_ovvo / F_oo / W_oooo . t3) + W_vvvv.t3
  update     r3 <- P3_full(r3, -1/6, 1); r3 /= D; norms; t3 += r3
  DIIS       one unified T1/T2/T3 DIIS update (6 slots) of the vector
with the large contractions as split-BF16x3 tcgen05 GEMMs (FP32 accumulate;
FP64 storage, denominators, update, norms and DIIS).  The same step on the
plain FP64 GPU path (cuBLAS DGEMM) is timed beside it.  `e2e` is the same
step through the drop-in routes (dcc.backend.update_amps_rccsdt_tri_ +
run_diis_t3) with every host-side input a numpy array, as the reference
passes them.  Secondary lines: the same step at nocc=10 / nvir=90, the (Q)
energies on sampled task groups, one T4 update at the N2 6-31G shape.

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
import types

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "distributed-cc_b200"))

HEADLINE = (15, 93)   # benzene cc-pVDZ, 6 C1s frozen
SECONDARY = (10, 90)  # the kernel-level synthetic configuration
Q_BLK = 4
DIIS_SPACE = 6
METRIC = ("RCCSDT T3 half-iteration time (feedback, compute_r3_tri, P3_full, divide, update, norms, unified DIIS), "
          "mixed split-BF16x3 batched path, nocc=15 nvir=93 synthetic")
UNIT = "s/iter"
DATA = ("synthetic (seeded torch generator; e_occ U[-1.5,-0.3], e_vir U[0.1,3.0], t2 N(0,1e-2) with "
        "t2[ijab]=t2[jiba], ERIs N(0,0.1) 8-fold symmetric, t3 N(0,1e-3) symmetric)")


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

def cpu_step_seconds(nocc, nvir, steps, warmup):
    """The reference's CPU path of one T3 half-iteration, sampled and extrapolated
    (oracle/cpu_t3_step.py); returns per-step estimates, the helper kind and threads."""
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    from oracle import cpu_t3_step
    w = cpu_t3_step.T3StepCPU(nocc, nvir, seed=0)
    out = []
    for s in range(warmup + steps):
        v = w.step()
        if s >= warmup:
            out.append(v)
    return out, ("reference" if w.h.ref else "port"), len(w.sample)


def reference_arm(args, rank, world):
    """`--impl reference`: the reference's CPU path on this host's cores, rank 0 only."""
    if rank != 0:
        return 0
    no, nv = HEADLINE
    t0 = time.perf_counter()
    vals, kind, nsamp = cpu_step_seconds(no, nv, args.steps, args.warmup)
    wall = time.perf_counter() - t0
    v = statistics.mean(vals)
    n3 = no * (no + 1) * (no + 2) // 6
    from oracle import cpu_t3_step
    sample = cpu_t3_step.describe(no, nv)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": DATA.replace("torch generator", "numpy generator"),
            "config": {"workload": "rccsdt_t3_half_iteration", "nocc": no, "nvir": nv, "n_blocks": n3},
            "label": "reference C helpers + numpy restatement, sampled",
            "extrapolated_from_blocks": nsamp,
            "sampled_wall_s": wall,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                             "helpers": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------- GPU side

def measure_fp64_tf32_peaks(torch):
    """Dense FP64 and TF32 GEMM throughput of this GPU (torch matmul 8192^3, best of 5)."""
    out = {}
    n = 8192
    for name, dt, tf32 in (("fp64_tflops", torch.float64, False), ("tf32_tflops", torch.float32, True)):
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(n, n, dtype=dt, device="cuda")
        b = torch.randn(n, n, dtype=dt, device="cuda")
        c = torch.empty(n, n, dtype=dt, device="cuda")
        best = None
        for _ in range(6):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        torch.backends.cuda.matmul.allow_tf32 = prev
        out[name] = 2.0 * n ** 3 / (best * 1e-3) / 1e12
        del a, b, c
    torch.cuda.empty_cache()
    out["how"] = "torch.matmul 8192^3, best of 6, CUDA events"
    return out


def feedback_inputs(d, torch, seed=7):
    """The dressed-Fock / ERI slices the T3 feedback reads, from the synthetic physicist ERIs
    (<pq|rs> = <rs|pq> for real orbitals): oovv <ij|ab>, vovv <cx|ad> = <ad|cx>, ooov
    <zx|la> = <al|xz>; fock_ov N(0, 1e-2)."""
    g = torch.Generator(device="cuda").manual_seed(seed)
    return {"oovv": d.eris_vvoo.permute(2, 3, 0, 1).contiguous(),
            "vovv": d.W_vvvo.permute(2, 3, 0, 1).contiguous(),
            "ooov": d.W_vooo.permute(3, 2, 1, 0).contiguous(),
            "fock_ov": torch.randn(d.nocc, d.nvir, dtype=torch.float64, device="cuda", generator=g) * 1e-2}


class Workload:
    """Device-resident inputs of the T3 half-iteration at one shape, and the step."""

    def __init__(self, torch, nocc, nvir, seed=0):
        from dcc import synthetic
        self.torch = torch
        self.no, self.nv = nocc, nvir
        self.d = synthetic.make_inputs(nocc, nvir, seed=seed)
        self.sl = feedback_inputs(self.d, torch)
        self.t3_0 = self.d.t3  # pristine start
        npair = nocc * (nocc + 1) // 2
        g = torch.Generator(device="cuda").manual_seed(seed + 11)
        self.lower0 = torch.randn(nocc * nvir + npair * nvir * nvir, dtype=torch.float64, device="cuda",
                                  generator=g) * 1e-2
        d = self.d
        self.dd = types.SimpleNamespace(**{k: getattr(d, k) for k in
                                           ("F_vv", "F_oo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo", "t2", "ijk",
                                            "eia")})
        self.dd.W_vooo, self.dd.W_vvvo = d.W_vooo.clone(), d.W_vvvo.clone()

    def start(self, it):
        """Fresh state for a run: t3, the lower-order DIIS vector and a new DIIS history."""
        self.T = self.t3_0.clone()
        self.lower = self.lower0.clone()
        self.key = object()
        it.diis = None

    def step(self, it):
        """One T3 half-iteration on the device (intermediates rebuilt from the pristine
        ones, as the host rebuilds them every iteration)."""
        dd, sl = self.dd, self.sl
        dd.W_vooo.copy_(self.d.W_vooo)
        dd.W_vvvo.copy_(self.d.W_vvvo)
        it.feedback_r1r2(self.T, sl["fock_ov"], sl["oovv"], sl["vovv"], sl["ooov"])
        it.feedback_w(dd.W_vooo, dd.W_vvvo, sl["oovv"])
        it.residual(dd, self.T)
        it.update(self.T, dd.eia)
        it.diis_update(self.lower, self.T, DIIS_SPACE, key=self.key)


def timed(torch, ranks, fn, steps, warmup):
    for _ in range(warmup):
        fn()
    ranks.barrier("cuda")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    ranks.barrier("cuda")
    return ranks.max_over_ranks(e0.elapsed_time(e1), "cuda")


def t3_line(torch, ranks, contract, nocc, nvir, precision, steps, warmup, track_gemm=False, tune=True,
            count_launches=False, e2e=None):
    """Time the T3 half-iteration at one shape and precision; returns (info, it, workload)."""
    from dcc.t3_iteration import T3Iteration
    w = Workload(torch, nocc, nvir)
    it = T3Iteration(nocc, nvir, precision)
    info = {"precision": precision}
    if tune and precision != "fp64":
        tuned = it.res.tune(w.dd, w.t3_0)
        from dcc import autotune
        info["wvvvv_gemm_pipeline"] = {
            "kb_bytes": tuned[0], "stages": tuned[1], "group_m": tuned[2], "chosen_by": "dcc.autotune",
            "tile_n": tuned[3], "candidates_ms": {"%d/%d/%d/%d" % c: round(ms, 4) for c, ms in
                                                  (autotune.timings(it.res.wvvvv.key()) or {}).items()}}
        # the S GEMMs' tile width (128 x 256 or 128 x 128) and raster group, each tuned alone
        info["s_gemm_tiles"] = {
            name: {"chosen": "%d/%d/%d/%d" % cfg,
                   "candidates_ms": {"%d/%d/%d/%d" % c: round(ms, 4) for c, ms in times.items()}}
            for name, (cfg, times) in it.res.s_tuning().items()}
    w.start(it)
    if count_launches:
        from torch.profiler import profile, ProfilerActivity
        w.step(it)
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            w.step(it)
            torch.cuda.synchronize()
        names = [ev.name for ev in prof.events() if ev.device_type == torch.autograd.DeviceType.CUDA]
        info["launches_per_step"] = sum(1 for n in names if "dcc::" in n)
        info["library_launches_per_step"] = len(names) - info["launches_per_step"]
        del prof
        w.start(it)
    gemm_ev = []
    orig_gemm = contract.gemm_
    if track_gemm:
        wa, ww = it.res.wvvvv.A.M, it.res.wvvvv.W.M

        def timed_gemm(A, B, C, frow, fcol, alpha=1.0, beta=1.0, status=None, Kp=None):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            st = orig_gemm(A, B, C, frow, fcol, alpha, beta, status, Kp)
            e1.record()
            if A.M == wa and B.M == ww:
                gemm_ev.append((e0, e1))
            return st

    for _ in range(warmup):
        w.step(it)
    if track_gemm:
        contract.gemm_ = timed_gemm
    try:
        ms = timed(torch, ranks, lambda: w.step(it), steps, 0)
    finally:
        contract.gemm_ = orig_gemm
    info["ms_total"] = ms
    info["ms_per_step"] = ms / steps
    info["status_ok"] = it.status_ok()
    info["t3_finite"] = bool(torch.isfinite(w.T).all())
    if gemm_ev:
        info["gemm_ms"] = [a.elapsed_time(b) for a, b in gemm_ev]
    return info, it, w


def e2e_run(torch, ranks, it, w, precision, steps, warmup):
    """The same step through the drop-in routes, host numpy inputs: per iteration the host
    lower-order code (here a replay of stored arrays, where a real run calls PySCF) hands
    numpy intermediates to backend.update_amps_rccsdt_tri_, and backend.run_diis_t3 takes the
    host t1/t2; T3 stays resident (it was uploaded once, before the timed region)."""
    import numpy as np
    from dcc import backend
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import ref_standins as S
    no, nv, d = w.no, w.nv, w.d
    nmo = no + nv
    host = {k: getattr(d, k).cpu().numpy() for k in
            ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")}
    t1_eris = np.zeros((nmo,) * 4)
    o, v = slice(0, no), slice(no, nmo)
    t1_eris[o, o, v, v] = w.sl["oovv"].cpu().numpy()
    t1_eris[v, o, v, v] = w.sl["vovv"].cpu().numpy()
    t1_eris[o, o, o, v] = w.sl["ooov"].cpu().numpy()
    t1_fock = np.zeros((nmo, nmo))
    t1_fock[o, v] = w.sl["fock_ov"].cpu().numpy()
    rng = np.random.default_rng(5)
    r1_lower, r2_lower = rng.standard_normal((no, nv)) * 1e-4, rng.standard_normal((no, no, nv, nv)) * 1e-4

    class Replay:
        """Hands out the stored host arrays the way the lower-order code returns fresh ones."""

        def update_t1_fock_eris(self, mycc, imds, t1, eris):
            imds.t1_fock, imds.t1_eris = t1_fock, t1_eris

        def intermediates_t1t2(self, mycc, imds, t2):
            return imds

        def compute_r1r2(self, mycc, imds, t2):
            return r1_lower.copy(), r2_lower.copy()

        def r1r2_divide_e_(self, mycc, r1, r2, mo_energy):
            eia = mo_energy[:no, None] - mo_energy[None, no:]
            r1 /= eia
            r2 /= eia[:, None, :, None] + eia[None, :, None, :]

        def intermediates_t3(self, mycc, imds, t2):
            for k, a in host.items():
                setattr(imds, k, a)

    mod = types.SimpleNamespace(_IMDS=S.IMDS, resolve_nvir_diis=S.resolve_nvir_diis,
                                pack_unique_replicated_tamps=S.pack_unique_replicated_tamps,
                                unpack_unique_replicated_tamps=S.unpack_unique_replicated_tamps,
                                _max_t_diis_update_norm=S._max_t_diis_update_norm)
    for name in S.LowerOrderReplay.NAMES:
        setattr(mod, name, getattr(Replay(), name))
    mycc = types.SimpleNamespace(nocc=no, nmo=nmo, einsum_backend="cuda", dcc_precision=precision,
                                 comm=backend.SingleRankComm(), size=1, level_shift=0.0, nvir_diis=None,
                                 diis_start_cycle=0, diis_start_energy_diff=1e9)
    mycc.unique_tamps_map = S.build_unique_tamps_map(mycc)
    mycc._dcc_state = {("t3it", no, nv, precision): it}
    eris = types.SimpleNamespace(mo_energy=np.concatenate([d.e_occ.cpu().numpy(), d.e_vir.cpu().numpy()]))
    t1 = rng.standard_normal((no, nv)) * 1e-2
    t2 = d.t2.cpu().numpy()
    tamps = [t1, t2, (S.CanonicalT3Dist(no), w.t3_0.cpu().numpy())]
    adiis = types.SimpleNamespace(space=DIIS_SPACE, last_delta_norm_sq=None)
    state = {"istep": 0}

    def step():
        res_norm = backend.update_amps_rccsdt_tri_(mycc, tamps, eris, mod=mod)
        normt = float(np.linalg.norm(res_norm))
        backend.run_diis_t3(mycc, tamps, tamps[2][1], state["istep"], normt, 0.0, adiis, res_norm=res_norm,
                            return_update_norm=True, mod=mod)  # updates tamps in place
        state["istep"] += 1

    step()  # the first call uploads t3_local once and puts the device array into tamps
    for _ in range(max(0, warmup - 1)):
        step()
    backend.TRANSFER.reset()
    ms = timed(torch, ranks, step, steps, 0)
    h2d, d2h = backend.TRANSFER.h2d // steps, backend.TRANSFER.d2h // steps
    return ms, h2d, d2h


def q_line(torch, ranks, nocc, nvir, precision, ngroups, seed=0):
    """[Q]/(Q) energies on sampled task groups (tasks sharing (a, b, c) blocks), split and FP64,
    extrapolated to all tasks by task count; plus the same sample at a molecular energy scale."""
    from dcc import _c_rccsdt, rccsdt_q, synthetic
    d = synthetic.make_inputs(nocc, nvir, seed=seed)
    er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
          "vvvv": d.W_vvvv, "oooo": d.W_oooo}
    t2q = d.t2.permute(2, 3, 0, 1).contiguous()
    t3_abc = _c_rccsdt.redistribute_ijk_to_abc(d.t3, nocc, nvir)
    del d.t3
    torch.cuda.empty_cache()
    G = rccsdt_q.groups(nvir, Q_BLK)
    sample = G[::max(1, len(G) // ngroups)][:ngroups]
    ntask = len(rccsdt_q.task_list(nvir, Q_BLK))
    nsample = sum(len(rccsdt_q.prange(g[4], nvir, Q_BLK)) for g in sample)
    out = {"nocc": nocc, "nvir": nvir, "blksize": Q_BLK, "tasks": ntask, "sample_groups": len(sample),
           "sample_tasks": nsample}
    for prec in (precision, "fp64"):
        q = rccsdt_q.QEnergy(nocc, nvir, Q_BLK, prec)
        q.prepare(sample)  # grouped tables of every sampled group shape, outside the timed region
        q.run(er, t2q, t3_abc, d.e_occ, d.e_vir, sample[:1])  # warm-up
        q.out.zero_()
        ranks.barrier("cuda")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        q.run(er, t2q, t3_abc, d.e_occ, d.e_vir, sample)
        e1.record()
        ranks.barrier("cuda")
        ms = ranks.max_over_ranks(e0.elapsed_time(e1), "cuda")
        out[prec] = {"s_sample": ms / 1e3, "s_all_tasks_est": ms / 1e3 * ntask / nsample,
                     "e_bracket_sample": float(q.out[0]), "e_paren_sample": float(q.out[1]),
                     "status_ok": q.status_ok()}
        del q
        torch.cuda.empty_cache()
    out["speedup_vs_fp64"] = out["fp64"]["s_sample"] / out[precision]["s_sample"]
    out["abs_dE_paren_sample"] = abs(out["fp64"]["e_paren_sample"] - out[precision]["e_paren_sample"])
    # the synthetic amplitudes give energies of O(10-100) Eh: the same sample with t2 and t3 scaled
    # by one factor s so that the FP64 (Q) energy is -1e-3 Eh (a molecular (Q) correction), untimed
    s = (1e-3 / max(abs(out["fp64"]["e_paren_sample"]), 1e-300)) ** 0.5
    ms_line = {"amplitude_scale": s}
    for prec in (precision, "fp64"):
        q = rccsdt_q.QEnergy(nocc, nvir, Q_BLK, prec)
        q.prepare(sample)
        q.run(er, t2q * s, t3_abc * s, d.e_occ, d.e_vir, sample)
        ms_line[prec] = {"e_bracket_sample": float(q.out[0]), "e_paren_sample": float(q.out[1]),
                         "status_ok": q.status_ok()}
        del q
        torch.cuda.empty_cache()
    ms_line["abs_dE_bracket"] = abs(ms_line["fp64"]["e_bracket_sample"] - ms_line[precision]["e_bracket_sample"])
    ms_line["abs_dE_paren"] = abs(ms_line["fp64"]["e_paren_sample"] - ms_line[precision]["e_paren_sample"])
    out["molecule_scale"] = ms_line
    del t3_abc, er, d
    torch.cuda.empty_cache()
    return out


def t4_line(torch, ranks, precision):
    """One T4 update (compute_r4_tri with its OO batch, projector, divide, norms, t4 += r4) at the
    N2 6-31G shape (nocc=7, nvir=11, 161 stored blocks): eager and replayed as one CUDA graph."""
    from dcc import graph as dgraph, synthetic as dsyn, t4_residual as dt4
    out = {"nocc": 7, "nvir": 11, "stored_blocks": 161}
    for prec in (precision, "fp64"):
        it = dgraph.T4Iteration(dsyn.make_t4_inputs(7, 11, seed=3), prec)
        out[prec] = {"eager_ms": timed(torch, ranks, it.step, 5, 3) / 5}
        del it
        gt4 = dgraph.T4IterationGraph(dgraph.T4Iteration(dsyn.make_t4_inputs(7, 11, seed=3), prec))
        out[prec]["graph_ms"] = timed(torch, ranks, gt4.replay, 5, 3) / 5
        del gt4
    d4 = dsyn.make_t4_inputs(7, 11, seed=3)
    r4s = {}
    for prec in (precision, "fp64"):
        r4s[prec] = torch.zeros_like(d4.t4)
        dt4.compute_r4_tri_(r4s[prec], d4.eris, d4.F_vv, d4.W_vvvo, d4.W_vooo, d4.W_vvvv, d4.W_oooo,
                            d4.W_ovov, d4.t2, d4.t3, d4.t4, 7, prec, F_oo=d4.F_oo, W_ovvo=d4.W_ovvo)
    out["r4_max_rel_err_vs_fp64"] = float((r4s[precision] - r4s["fp64"]).abs().max() / r4s["fp64"].abs().max())
    out["speedup_graph_vs_fp64"] = out["fp64"]["graph_ms"] / out[precision]["graph_ms"]
    return out


class TriplesEnergy:
    """E(t3): the T3 -> r2 strings (distr_cc/rccsdt.py:300-316, FP64), r2 symmetrized and
    divided by the T2 denominators, contracted with (2<ij|ab> - <ij|ba>) -- how T3 reaches
    the correlation energy through t2.  Linear in t3."""

    def __init__(self, torch, d):
        self.torch, self.d = torch, d
        self.E_vovv = d.W_vvvo.permute(2, 3, 0, 1)  # <cx|ad> = <ad|cx>
        self.E_ooov = d.W_vooo.permute(3, 2, 1, 0)  # <zx|la> = <al|xz>
        self.D2 = (d.e_occ[:, None, None, None] + d.e_occ[None, :, None, None]
                   - d.e_vir[None, None, :, None] - d.e_vir[None, None, None, :])
        self.L = 2.0 * d.eris_vvoo.permute(2, 3, 0, 1) - d.eris_vvoo.permute(2, 3, 1, 0)
        self.fock0 = torch.zeros(d.nocc, d.nvir, dtype=torch.float64, device="cuda")

    def __call__(self, t3):
        from dcc import t3_feedback
        torch, d = self.torch, self.d
        X = t3_feedback.p3_201_all(t3, d.nocc)
        r2 = torch.zeros(d.nocc, d.nocc, d.nvir, d.nvir, dtype=torch.float64, device="cuda")
        t3_feedback.r2_add_t3_x_(r2, self.fock0, self.E_vovv, self.E_ooov, X)
        del X
        return float((self.L * (r2 + r2.permute(1, 0, 3, 2)) / 2 / self.D2).sum())


def iteration_energy_error(torch, nocc, nvir, precision):
    """How the split path's error in one T3 iteration reaches the correlation energy.

    The FP64 and split residuals of the same inputs go through the same update (P3_full,
    divide, t3 += r3); the difference of the two new T3 goes through TriplesEnergy, and so
    does the FP64 T3 itself (the triples' share of E).  r3 is linear in (t2, t3), so the ratio
    is independent of the amplitudes' scale: abs_dE_at_10mEh is the error of a molecule whose
    triples contribute 10 mEh (the synthetic amplitudes are far larger than a molecule's)."""
    from dcc import synthetic, t3_residual
    d = synthetic.make_inputs(nocc, nvir, seed=0)
    rs = {}
    for prec in ("fp64", precision):
        res = t3_residual.T3Residual(nocc, nvir, prec, with_oo=True)
        rs[prec] = res.compute(d, d.t3)
        del res
        torch.cuda.empty_cache()
    ws = torch.empty(1 << 16, dtype=torch.float64, device="cuda")
    t3f, t3m = d.t3.clone(), d.t3.clone()
    t3_residual.update_t3_(t3f, rs["fp64"].clone(), d, workspace=ws)
    t3_residual.update_t3_(t3m, rs[precision].clone(), d, workspace=ws)
    rel_r3 = float((rs[precision] - rs["fp64"]).abs().max() / rs["fp64"].abs().max())
    del rs
    energy = TriplesEnergy(torch, d)
    e_t3 = energy(t3f)
    de = energy(t3m - t3f)
    del t3f, t3m, d, energy
    torch.cuda.empty_cache()
    return {"nocc": nocc, "nvir": nvir, "r3_max_rel_err_vs_fp64": rel_r3, "e_t3_share_fp64": e_t3,
            "abs_dE": abs(de), "relative": abs(de / e_t3), "abs_dE_at_10mEh": abs(de / e_t3) * 1e-2}


def converged_energy_error(torch, nocc, nvir, precision, sigma=0.2, tol=1e-9, max_iter=80, space=8,
                           conv_tol_rel=1e-6, conv_tol_normt=1e-5):
    """The T3 equations alone (t2 and the intermediates fixed) iterated to convergence with
    DIIS in FP64 and in split precision from t3 = 0: t3 += P3_full(r3)/D with r3 =
    compute_r3_tri (the update of distr_cc/rccsdt.py:941-971), DIIS over t3 (distr_cc/diis.py).
    The intermediates that couple t3 to itself (W_vvvv, W_ovov, W_ovvo, W_oooo) are scaled by
    `sigma` so that this fixed-point iteration contracts for the synthetic integrals (molecular
    ones do without help).

    FP64 runs to a relative update below `tol` (the tight solution).  The split path runs the
    reference's convergence test (distr_cc/rccsdt.py:1140: |dE| < conv_tol and the residual
    norm < conv_tol_normt) with E = TriplesEnergy(t3): conv_tol is the 1e-8 Eh of the
    molecular runs taken at a 10 mEh triples share (relative 1e-6), the norm test relative to
    |t3|; it then keeps iterating to max_iter and reports the update it levels off at (the
    split precision's floor).  The converged T3 of the two precisions go through
    TriplesEnergy; their difference, relative to the FP64 triples share, is scaled to a
    molecule whose triples contribute 10 mEh."""
    import math
    from dcc import synthetic, t3_residual
    from dcc.diis import DIIS
    d = synthetic.make_inputs(nocc, nvir, seed=0)
    for k in ("W_vvvv", "W_ovov", "W_ovvo", "W_oooo"):
        setattr(d, k, getattr(d, k) * sigma)
    energy = TriplesEnergy(torch, d)
    out = {"nocc": nocc, "nvir": nvir, "coupling_scale": sigma, "fp64_tol": tol,
           "split_test": {"conv_tol_rel": conv_tol_rel, "conv_tol_normt_rel": conv_tol_normt}}
    t3s = {}
    for prec in ("fp64", precision):
        res = t3_residual.T3Residual(nocc, nvir, prec, with_oo=True)
        t3 = torch.zeros_like(d.t3)
        r3 = torch.empty_like(t3)
        diis = DIIS(space)
        rel, e_old, passed = None, 0.0, None
        for it in range(1, max_iter + 1):
            res.compute(d, t3, r3)
            n = t3_residual.update_t3_(t3, r3, d, write_r3=True)
            diis.update([t3])
            rel = math.sqrt(float(n[0])) / max(float(t3.norm()), 1e-300)
            if prec == "fp64":
                if rel < tol:
                    break
            else:
                e = energy(t3)
                if passed is None and abs(e - e_old) < conv_tol_rel * abs(e) and rel < conv_tol_normt:
                    passed = it
                e_old = e
        out[prec] = {"iterations": it, "final_rel_update": rel, "status_ok": res.status_ok(),
                     "e_t3_share": energy(t3)}
        if prec == "fp64":
            out[prec]["converged"] = rel < tol
        else:
            out[prec]["reference_test_passed_at_iteration"] = passed
        t3s[prec] = t3
        del res, r3, diis
        torch.cuda.empty_cache()
    de = energy(t3s[precision] - t3s["fp64"])
    e = out["fp64"]["e_t3_share"]
    out["abs_dE"] = abs(de)
    out["relative"] = abs(de / e)
    out["abs_dE_at_10mEh"] = abs(de / e) * 1e-2
    out["t3_max_rel_diff"] = float((t3s[precision] - t3s["fp64"]).abs().max() / t3s["fp64"].abs().max())
    del t3s, d, energy
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dcc", choices=["dcc", "reference"])
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "tf32x3"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-path comparison (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="headline only: no secondary shape, (Q), T4, energy-error or peak lines")
    ap.add_argument("--shape", default=None, help="nocc,nvir of the headline step (default 15,93)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # the reference's CPU path needs no GPU and no process group: rank 0 alone runs it
        return reference_arm(args, rank, world)
    import torch
    from dcc import contract, ranks
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    no, nv = HEADLINE if args.shape is None else tuple(int(x) for x in args.shape.split(","))
    n3 = no * (no + 1) * (no + 2) // 6

    # ---- headline: the mixed T3 half-iteration, device-resident inputs
    with ClockSampler(local) as clk:
        mix, it, w = t3_line(torch, ranks, contract, no, nv, args.precision, args.steps, args.warmup,
                             track_gemm=True, count_launches=True)
    # ---- e2e: the same step through the drop-in routes, host numpy inputs
    e2e_steps = max(2, args.steps // 2)
    e2e_ms, h2d, d2h = e2e_run(torch, ranks, it, w, args.precision, e2e_steps, 2)
    del it, w
    torch.cuda.empty_cache()
    # ---- the plain FP64 GPU path, same step
    f64 = None
    if not args.no_fp64:
        fsteps = max(2, args.steps // 4)
        f64, it, w = t3_line(torch, ranks, contract, no, nv, "fp64", fsteps, 3)
        f64["steps"] = fsteps
        del it, w
        torch.cuda.empty_cache()

    extras = {}
    if not args.no_extras:
        extras["fp64_tf32_gemm_peaks"] = measure_fp64_tf32_peaks(torch)
        s_no, s_nv = SECONDARY
        sec, it, w = t3_line(torch, ranks, contract, s_no, s_nv, args.precision, args.steps, args.warmup)
        del it, w
        torch.cuda.empty_cache()
        sf, it, w = t3_line(torch, ranks, contract, s_no, s_nv, "fp64", max(2, args.steps // 3), 3)
        del it, w
        torch.cuda.empty_cache()
        extras["secondary_nocc10_nvir90"] = {"mixed_s_per_iter": sec["ms_per_step"] / 1e3,
                                             "fp64_s_per_iter": sf["ms_per_step"] / 1e3,
                                             "speedup_vs_fp64": sf["ms_per_step"] / sec["ms_per_step"],
                                             "status_ok": sec["status_ok"] and sf["status_ok"]}
        extras["q_energy"] = q_line(torch, ranks, no, nv, args.precision, 12)
        extras["q_energy_nocc10_nvir90"] = q_line(torch, ranks, s_no, s_nv, args.precision, 24)
        extras["t4_iteration"] = t4_line(torch, ranks, args.precision)
        extras["iteration_energy_error"] = iteration_energy_error(torch, s_no, s_nv, args.precision)
        extras["converged_energy_error"] = [converged_energy_error(torch, 6, 40, args.precision),
                                            converged_energy_error(torch, s_no, s_nv, args.precision)]

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import cpu_t3_step
        vals, kind, nsamp = cpu_step_seconds(no, nv, 1, 0)
        cpu = {"value": vals[0], "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "helpers": kind,
               "label": "reference C helpers + numpy restatement, sampled", "extrapolated_from_blocks": nsamp,
               "sample": cpu_t3_step.describe(no, nv)}

    gemm_ms = mix.get("gemm_ms") or []
    gemm_avg = statistics.mean(gemm_ms) if gemm_ms else None
    flops_launch = 2.0 * n3 * nv ** 5  # one of the three W_vvvv.t3 strings
    hbm, bf16, bf16_sus, src = peaks()
    peak_useful = bf16_sus / 3.0  # three bf16 products per FP64-equivalent flop
    achieved = flops_launch / (gemm_avg * 1e-3) / 1e12 if gemm_avg else None
    traffic = profile_traffic("gemm_split3_wvvvv_nocc%d_nvir%d" % (no, nv))

    value = ranks.job_seconds_per_iteration(mix["ms_total"], args.steps, world)  # whole job, replicas
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mix["ms_per_step"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 storage; " + args.precision + " products, f32 accumulate", "data": DATA,
        "config": {"workload": "rccsdt_t3_half_iteration", "nocc": no, "nvir": nv, "n_blocks": n3,
                   "shape_of": "benzene cc-pVDZ, 6 C1s frozen" if (no, nv) == HEADLINE else "custom",
                   "terms": "r1r2_add_t3_tri_ + intermediates_t3_add_t3_tri feedback, compute_r3_tri (W_vvvo.t2, "
                            "W_vooo.t2, F_vv.t3, OO W_ovov/W_ovvo/F_oo/W_oooo.t3, W_vvvv.t3), P3_full, divide, "
                            "update, norms, unified DIIS (%d slots)" % DIIS_SPACE,
                   "precision": args.precision, "l2": "inputs larger than L2 (t3 %.2f GB)" % (n3 * nv ** 3 * 8e-9),
                   "parallelism": "replicas" if world > 1 else "single"},
        "fp64_path_s_per_iter": f64["ms_per_step"] / 1e3 if f64 else None,
        "speedup_vs_fp64": f64["ms_per_step"] / mix["ms_per_step"] if f64 else None,
        "device_status_ok": mix["status_ok"] and (f64["status_ok"] if f64 else True),
        "t3_finite": mix["t3_finite"],
        "wvvvv_gemm_pipeline": mix.get("wvvvv_gemm_pipeline"),
        "s_gemm_tiles": mix.get("s_gemm_tiles"),
        "roofline": {"kernel": "dcc::k_gemm_split3<0> (W_vvvv.t3 string)", "bound": "tensor",
                     "achieved": achieved, "peak": peak_useful, "unit": "TFLOP/s",
                     "frac": (achieved / peak_useful) if achieved else None,
                     "peak_note": "bf16 dense %s sustained %.1f TF/s / 3 products (of %s)" % (src, bf16_sus, src),
                     "flops_per_launch": flops_launch, "launch_ms": gemm_avg, "traffic": traffic},
        "cpu_baseline": cpu,
        "e2e": {"value": ranks.job_seconds_per_iteration(e2e_ms, e2e_steps, world), "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "path": "dcc.backend.update_amps_rccsdt_tri_ + run_diis_t3, host numpy intermediates and t1/t2, "
                        "T3 resident"},
        "gpu_launches": mix["launches_per_step"] * args.steps,
        "library_launches_per_step": mix["library_launches_per_step"],
        "clocks": clk.summary(),
    }
    line.update(extras)
    # algorithmic FP64-equivalent flops of one step, counted from the reference's einsum strings per
    # canonical block (W_vvvv.t3 6 nv^5, W_vvvo.t2 + F_vv.t3 18 nv^4, OO batch ~24 no nv^4, W_vooo.t2
    # 12 no nv^3) plus the feedback's two nv^4-per-ordered-block strings (4 no^3 nv^4)
    step_flops = n3 * (6.0 * nv ** 5 + 18.0 * nv ** 4 + 24.0 * no * nv ** 4 + 12.0 * no * nv ** 3) \
        + 4.0 * no ** 3 * nv ** 4
    line["step_algorithmic_flops"] = step_flops
    line["mixed_step_tflops"] = step_flops / (mix["ms_per_step"] * 1e-3) / 1e12
    if f64:
        line["fp64_step_tflops"] = step_flops / (f64["ms_per_step"] * 1e-3) / 1e12
        pk = extras.get("fp64_tf32_gemm_peaks")
        if pk:
            line["fp64_step_frac_of_measured_fp64_peak"] = line["fp64_step_tflops"] / pk["fp64_tflops"]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
