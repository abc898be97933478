"""Generate tests/golden/ref_drivers.npz by running the reference's own Python
drivers on seeded inputs.

Every contraction of the triples / quadruples path lives in the reference's
Python (distr_cc/rccsdt.py, rccsdt_q.py, rccsdtq.py, diis.py), which imports
PySCF and mpi4py.  Neither is installed here, so tests/ref_standins.py puts
one-rank stand-ins for both into sys.modules; the reference's C helpers are
compiled from the reference sources by oracle/Makefile and placed where the
reference's loader looks for them (build/distr_cc.so next to a copy of the
package, distr_cc/_lib.py:19).  The functions below then run unmodified:

  compute_r3_tri                    distr_cc/rccsdt.py:368-433 (+ OO :435-732)
  r1r2_add_t3_tri_                  distr_cc/rccsdt.py:253-321
  intermediates_t3_add_t3_tri       distr_cc/rccsdt.py:323-366
  update_amps_rccsdt_tri_ + run_diis_t3, four iterations of the loop of
                                    distr_cc/rccsdt.py:1103-1142 with the
                                    lower-order PySCF steps replayed
  kernel ((Q), all tasks and split into jobs)   distr_cc/rccsdt_q.py:227
  compute_r4_tri / r2_add_t4_tri_ / r3_add_t4_tri_   distr_cc/rccsdtq.py:471-1349
  DIIS.update                       distr_cc/diis.py:105-177

Run from the repository root with the reference checkout's path:

    python tests/golden/make_ref_fixtures.py <path-to-reference>

(or set DCC_REFERENCE).  Inputs follow the benchmark distributions at small
sizes; every input and output is stored, so the fixtures need nothing else.
"""
from __future__ import annotations

import itertools
import os
import shutil
import subprocess
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "ref_drivers.npz")
sys.path.insert(0, os.path.join(ROOT, "tests"))
import ref_standins as S  # noqa: E402


# ----------------------------------------------------------------- inputs

def sym8(g):
    perms = [(0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2), (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0),
             (3, 2, 1, 0)]
    return sum(g.transpose(p) for p in perms) / 8.0


def symmetric_t3(no, nv, rng, scale=1e-3):
    full = rng.standard_normal((no,) * 3 + (nv,) * 3) * scale
    return sum(full.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3))) / 6.0


def canonical(U, no):
    return np.ascontiguousarray(np.stack([U[i, j, k] for i in range(no) for j in range(i, no)
                                          for k in range(j, no)]))


def physicist(no, nv, rng):
    """<pq|rs> = (pr|qs) of an 8-fold symmetric N(0, 0.1) ERI tensor, and its slices."""
    nmo = no + nv
    eri = sym8(rng.standard_normal((nmo,) * 4) * 0.1)
    g = np.ascontiguousarray(eri.transpose(0, 2, 1, 3))
    o, v = slice(0, no), slice(no, nmo)
    sl = {"W_vvvv": g[v, v, v, v], "W_vvvo": g[v, v, v, o], "W_vooo": g[v, o, o, o], "W_ovov": g[o, v, o, v],
          "W_ovvo": g[o, v, v, o], "W_oooo": g[o, o, o, o]}
    return g, {k: np.ascontiguousarray(a) for k, a in sl.items()}


def energies(no, nv, rng):
    eo = np.sort(rng.uniform(-1.5, -0.3, no))
    ev = np.sort(rng.uniform(0.1, 3.0, nv))
    return eo, ev


def t2_of(no, nv, rng):
    t2 = rng.standard_normal((no, no, nv, nv)) * 1e-2
    return np.ascontiguousarray((t2 + t2.transpose(1, 0, 3, 2)) * 0.5)


def fock_blocks(eo, ev, rng):
    no, nv = len(eo), len(ev)
    cv = rng.standard_normal((nv, nv)) * 1e-2
    co = rng.standard_normal((no, no)) * 1e-2
    return np.diag(ev) + 0.5 * (cv + cv.T), np.diag(eo) + 0.5 * (co + co.T)


def t3_imds(no, nv, rng):
    eo, ev = energies(no, nv, rng)
    _, w = physicist(no, nv, rng)
    F_vv, F_oo = fock_blocks(eo, ev, rng)
    d = dict(w, F_vv=F_vv, F_oo=F_oo)
    return eo, ev, d


# ----------------------------------------------------------------- reference

def load_reference(ref_dir):
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "REF_SRC=%s" % os.path.join(ref_dir, "src")],
                   check=True)
    so = os.path.join(ROOT, "oracle", "_ref", "libdistr_cc_ref.so")
    tmp = tempfile.mkdtemp(prefix="dcc_ref_")
    shutil.copytree(os.path.join(ref_dir, "distr_cc"), os.path.join(tmp, "distr_cc"))
    os.makedirs(os.path.join(tmp, "build"))
    shutil.copy(so, os.path.join(tmp, "build", "distr_cc.so"))
    S.install(so)
    sys.path.insert(0, tmp)
    import distr_cc.diis as md
    import distr_cc.distribute_t3 as d3
    import distr_cc.distribute_t4 as d4
    import distr_cc.rccsdt as m3
    import distr_cc.rccsdt_q as mq
    import distr_cc.rccsdtq as m4
    return types.SimpleNamespace(m3=m3, mq=mq, m4=m4, md=md, d3=d3, d4=d4)


def make_cc(no, nv, batch_size=100, **kw):
    cc = types.SimpleNamespace(nocc=no, nmo=no + nv, einsum_backend="numpy", comm=S.OneRankComm(), rank=0, size=1,
                               batch_size=batch_size, stdout=sys.stdout, verbose=0, level_shift=0.0, nvir_diis=None,
                               max_memory=64000, diis=True, diis_space=6, diis_start_cycle=0,
                               diis_start_energy_diff=1e9, allow_python_fallback=False, unique_tamps_map=None)
    cc.build_unique_tamps_map = lambda: S.build_unique_tamps_map(cc)
    for k, v in kw.items():
        setattr(cc, k, v)
    return cc


def imds_of(ref, d):
    im = ref.m3._IMDS()
    for k, v in d.items():
        setattr(im, k, np.array(v, copy=True))
    return im


# ----------------------------------------------------------------- cases

def case_r3(ref, out, tag, no, nv, batch_size, seed, woooo_noise=0.0):
    rng = np.random.default_rng(seed)
    eo, ev, d = t3_imds(no, nv, rng)
    if woooo_noise:
        d["W_oooo"] = d["W_oooo"] + woooo_noise * rng.standard_normal(d["W_oooo"].shape)
    t2 = t2_of(no, nv, rng)
    t3 = canonical(symmetric_t3(no, nv, rng), no)
    cc = make_cc(no, nv, batch_size)
    dt3 = ref.d3.DistributedT3IJK(no, nv, cc.comm, batch_size=batch_size)
    r3 = ref.m3.compute_r3_tri(cc, imds_of(ref, d), t2, (dt3, t3.copy()))
    for k, v in d.items():
        out["%s/%s" % (tag, k)] = v
    out[tag + "/t2"], out[tag + "/t3"], out[tag + "/r3"] = t2, t3, r3
    out[tag + "/shape"] = np.array([no, nv, batch_size])


def case_feedback(ref, out, tag, no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    t1_eris = rng.standard_normal((nmo,) * 4) * 0.1
    t1_fock = rng.standard_normal((nmo, nmo)) * 0.1
    t3 = canonical(symmetric_t3(no, nv, rng, 1.0), no)
    r1, r2 = rng.standard_normal((no, nv)), rng.standard_normal((no, no, nv, nv))
    Wo, Wv = rng.standard_normal((nv, no, no, no)), rng.standard_normal((nv, nv, nv, no))
    cc = make_cc(no, nv)
    dt3 = ref.d3.DistributedT3IJK(no, nv, cc.comm)
    im = imds_of(ref, dict(t1_fock=t1_fock, t1_eris=t1_eris, W_vooo=Wo, W_vvvo=Wv))
    r1o, r2o = ref.m3.r1r2_add_t3_tri_(cc, im, r1.copy(), r2.copy(), (dt3, t3))
    ref.m3.intermediates_t3_add_t3_tri(cc, im, (dt3, t3))
    for k, v in dict(t1_eris=t1_eris, t1_fock=t1_fock, t3=t3, r1_in=r1, r2_in=r2, W_vooo_in=Wo, W_vvvo_in=Wv,
                     r1=r1o, r2=r2o, W_vooo=im.W_vooo, W_vvvo=im.W_vvvo).items():
        out["%s/%s" % (tag, k)] = v
    out[tag + "/shape"] = np.array([no, nv])


def update_inputs(no, nv, seed):
    """Arrays of one T3 half-iteration: the lower-order replay and the starting amplitudes."""
    rng = np.random.default_rng(seed)
    nmo = no + nv
    eo, ev, d = t3_imds(no, nv, rng)
    a = dict(d)
    a["mo_energy"] = np.concatenate([eo, ev])
    a["t1_fock"] = rng.standard_normal((nmo, nmo)) * 0.05
    a["t1_eris"] = rng.standard_normal((nmo,) * 4) * 0.05
    a["r1_lower"] = rng.standard_normal((no, nv)) * 1e-3
    r2 = rng.standard_normal((no, no, nv, nv)) * 1e-3
    a["r2_lower"] = r2  # r2 += r2.transpose(1, 0, 3, 2) happens inside update_amps
    a["t1"] = rng.standard_normal((no, nv)) * 1e-2
    a["t2"] = t2_of(no, nv, rng)
    a["t3"] = canonical(symmetric_t3(no, nv, rng), no)
    return a


def case_update(ref, out, tag, no, nv, seed, niter=4, nvir_diis=None, diis_space=3):
    """niter iterations of update_amps_rccsdt_tri_ followed by run_diis_t3 (the loop body of
    distr_cc/rccsdt.py:1103-1121) with the lower-order steps replayed from fixed arrays."""
    a = update_inputs(no, nv, seed)
    cc = make_cc(no, nv, batch_size=7, nvir_diis=nvir_diis, diis_space=diis_space)
    cc.unique_tamps_map = S.build_unique_tamps_map(cc)
    S.LowerOrderReplay(a, no).bind(ref.m3)
    eris = ref.m3._PhysicistsERIs()
    eris.mo_energy = a["mo_energy"]
    dt3 = ref.d3.DistributedT3IJK(no, nv, cc.comm, batch_size=7)
    tamps = [a["t1"].copy(), a["t2"].copy(), (dt3, a["t3"].copy())]
    adiis = ref.m3.make_mpi_diis(cc)
    for k, v in a.items():
        out["%s/%s" % (tag, k)] = v
    for it in range(niter):
        res_norm = ref.m3.update_amps_rccsdt_tri_(cc, tamps, eris)
        normt = np.linalg.norm(res_norm)
        out["%s/it%d/res_norm" % (tag, it)] = np.array(res_norm)
        out["%s/it%d/t3_pre" % (tag, it)] = tamps[2][1].copy()
        tamps, update_norm = ref.m3.run_diis_t3(cc, tamps, tamps[2][1], it, normt, 0.0, adiis, res_norm=res_norm,
                                                return_update_norm=True)
        out["%s/it%d/t1" % (tag, it)] = tamps[0].copy()
        out["%s/it%d/t2" % (tag, it)] = tamps[1].copy()
        out["%s/it%d/t3" % (tag, it)] = tamps[2][1].copy()
        out["%s/it%d/update_norm" % (tag, it)] = np.array(update_norm)
    out[tag + "/shape"] = np.array([no, nv, niter, -1 if nvir_diis is None else nvir_diis, diis_space])


def case_q(ref, out, tag, no, nv, blks, seed, n_jobs=3):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    eo, ev = energies(no, nv, rng)
    g, _ = physicist(no, nv, rng)
    t1 = rng.standard_normal((no, nv)) * 1e-2
    t2 = t2_of(no, nv, rng) * 10.0
    t3 = canonical(symmetric_t3(no, nv, rng, 1e-2), no)
    out[tag + "/pppp"], out[tag + "/mo_energy"] = g, np.concatenate([eo, ev])
    out[tag + "/t1"], out[tag + "/t2"], out[tag + "/t3"] = t1, t2, t3
    for blk in blks:
        for job in [None] + list(range(n_jobs)):
            cc = make_cc(no, nv)
            eris = types.SimpleNamespace(pppp=g.copy(), mo_energy=np.concatenate([eo, ev]))
            dt3 = ref.d3.DistributedT3IJK(no, nv, cc.comm)
            tamps = [t1, t2, (dt3, t3.copy())]
            kw = {} if job is None else dict(job_idx=job, n_jobs=n_jobs)
            e = ref.mq.kernel(cc, eris=eris, tamps=tamps, blksize=blk, comm=cc.comm, log_redistribution=False, **kw)
            key = "%s/e_blk%d" % (tag, blk) if job is None else "%s/e_blk%d_job%d" % (tag, blk, job)
            out[key] = np.array(e, dtype=np.float64)
    out[tag + "/shape"] = np.array([no, nv, n_jobs] + list(blks))


def case_t4(ref, out, tag, no, nv, seed, batch_size=5):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    eo, ev, d = t3_imds(no, nv, rng)
    t1_eris = sym8(rng.standard_normal((nmo,) * 4) * 0.1).transpose(0, 2, 1, 3).copy()
    t1_fock = rng.standard_normal((nmo, nmo)) * 0.1
    t2 = t2_of(no, nv, rng)
    t3 = symmetric_t3(no, nv, rng)
    full = rng.standard_normal((no,) * 4 + (nv,) * 4) * 1e-4
    t4f = sum(full.transpose(p + tuple(4 + x for x in p)) for p in itertools.permutations(range(4))) / 24.0
    cc = make_cc(no, nv, batch_size)
    dt4 = ref.d4.DistributedT4IJKL(no, nv, cc.comm)
    local = [tuple(int(x) for x in q[:4]) for q in dt4.iter_local_ijkl()]
    t4 = np.ascontiguousarray(np.stack([t4f[q] for q in local]))
    im = imds_of(ref, dict(d, t1_eris=t1_eris, t1_fock=t1_fock))
    r2_in = rng.standard_normal((no, no, nv, nv)) * 1e-3
    r3_in = rng.standard_normal((no,) * 3 + (nv,) * 3) * 1e-3
    r2 = ref.m4.r2_add_t4_tri_(cc, im, r2_in.copy(), (dt4, t4))
    r3 = ref.m4.r3_add_t4_tri_(cc, im, r3_in.copy(), (dt4, t4))
    r4 = ref.m4.compute_r4_tri(cc, imds_of(ref, dict(d, t1_eris=t1_eris, t1_fock=t1_fock)), t2, t3, (dt4, t4))
    for k, v in dict(d, t1_eris=t1_eris, t1_fock=t1_fock, t2=t2, t3=t3, t4=t4, r2_in=r2_in, r3_in=r3_in, r2=r2,
                     r3=r3, r4=r4, ijkl=np.array(local, dtype=np.int32)).items():
        out["%s/%s" % (tag, k)] = v
    out[tag + "/shape"] = np.array([no, nv, batch_size])


def case_diis(ref, out, tag, n, space, nvec, seed):
    rng = np.random.default_rng(seed)
    adiis = ref.md.DIIS(dev=None, space=space, comm=S.OneRankComm())
    x = rng.standard_normal(n)
    xs, outs, dn = [], [], []
    for it in range(nvec):
        x = 0.6 * x + 0.1 * rng.standard_normal(n)
        xs.append(x.copy())
        outs.append(adiis.update(x.copy()))
        dn.append(np.nan if adiis.last_delta_norm_sq is None else adiis.last_delta_norm_sq)
    out[tag + "/x"], out[tag + "/xnew"], out[tag + "/delta_norm_sq"] = np.array(xs), np.array(outs), np.array(dn)
    out[tag + "/shape"] = np.array([n, space, nvec])


def main():
    ref_dir = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DCC_REFERENCE")
    if not ref_dir:
        sys.exit("usage: make_ref_fixtures.py <path-to-reference>  (or set DCC_REFERENCE)")
    ref = load_reference(ref_dir)
    out = {}
    case_r3(ref, out, "r3a", 4, 6, 7, seed=101)
    case_r3(ref, out, "r3b", 3, 5, 4, seed=102, woooo_noise=0.05)
    case_r3(ref, out, "r3c", 2, 9, 100, seed=103)
    case_feedback(ref, out, "fb", 4, 6, seed=201)
    case_update(ref, out, "upd", 3, 5, seed=301)
    case_update(ref, out, "updnd", 3, 6, seed=302, nvir_diis=4)
    case_q(ref, out, "q", 3, 7, (2, 3), seed=401)
    case_q(ref, out, "q4", 4, 6, (4,), seed=402, n_jobs=2)
    case_t4(ref, out, "t4", 4, 5, seed=501)
    case_diis(ref, out, "diis", 300, 3, 6, seed=601)
    np.savez_compressed(OUT, **out)
    print("wrote %s: %d arrays, %.1f kB" % (OUT, len(out), os.path.getsize(OUT) / 1024))


if __name__ == "__main__":
    main()
