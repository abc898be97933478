"""TEST ORACLE ONLY -- the reference's CPU path of one T3 half-iteration of
RCCSDT, timed on a bounded sample, for bench.py's CPU baseline.

What one iteration of the reference does on the T3 side (distr_cc/rccsdt.py),
per canonical block (i <= j <= k) of one rank holding every block:

  r1r2_add_t3_tri_            :253-321  take + P3_422 + r1 einsums; for every
                                        distinct ordering take + P3_201 + 3 r2 einsums
  intermediates_t3_add_t3_tri :323-366  every ordering: take + P3_201 + 2 W einsums
  compute_r3_tri              :368-433  6 W_vvvo.t2, 6 W_vooo.t2, 3 F_vv.t3,
                                        3 W_vvvv.t3 einsums
  OO batch                    :435-614  per (source block, target block) pair the
                                        einsums of the matching cases, on the
                                        source's transpose-add / triple-sym forms
  F_oo / W_oooo prefactors    :616-732  Python loop over (source, target) pairs
                                        + 6 dense 'pq,pabc->qabc' GEMMs
  P3_full, divide, norms,
  t3 += r3                    :947-971
  run_diis_t3                 :1026-1067 one unified DIIS update over the vector

Per-target work is timed on one target block of each occupied case
(i<j<k, i=j<k, i<j=k, i=j=k) and weighted by how many blocks have that case;
work that is global to the iteration is timed on a slice and scaled: the
source-block preparation (transpose-add, triple-sym) on a few sources, the
prefactor loop on a tenth of its sources, the dense prefactor GEMMs on a
slice of their columns (they are compute-bound, so time scales with the
columns), and the DIIS update on a slice of the vector (memory-bound, so time
scales with its length).  The C helpers are the reference's own
(oracle/_ref, OpenMP) when they were compiled here, else the oracle's C
restatement; the einsums are numpy (BLAS, all host threads), as the
reference's numpy einsum backend runs them.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

from .oracle import Oracle, Reference, reference_available

_vp = ctypes.c_void_p


def _p(a):
    return a.ctypes.data_as(_vp)


class _Helpers:
    """take / P3 / transpose-add / triple-sym through the reference C library (or the oracle's)."""

    def __init__(self):
        self.ref = reference_available()
        self.lib = Reference() if self.ref else Oracle()

    def p3(self, blk, nv, pattern, alpha=1.0, beta=0.0):
        if self.ref:
            self.lib.t3_single_spin_summation_inplace_(_p(blk), nv, pattern.encode(), alpha, beta)
        else:
            self.lib.t3_spin_sum(blk, nv, pattern, alpha, beta)

    def take(self, t3, loc, i, j, k, no, nv, out):
        if self.ref:
            self.lib.take_t3_ijk_single_(_p(t3), _p(out), _p(loc), i, j, k, no, nv)
        else:
            out[...] = self.lib.take_t3(t3, loc, i, j, k, no, nv)[0]

    def transpose_add(self, src, nv):
        out = np.empty_like(src)
        if self.ref:
            self.lib.t3_transpose_add_(_p(src), _p(out), nv)
            return out
        return self.lib.t3_transpose_add(src, nv)

    def triple_sym(self, src, nv):
        if self.ref:
            b = [np.empty_like(src) for _ in range(3)]
            self.lib.t3_spin_summation_triple_sym_(_p(src), _p(b[0]), _p(b[1]), _p(b[2]), nv)
            return b
        return self.lib.t3_triple_sym(src, nv)


def _perms(i, j, k):
    if i < j < k:
        return [(i, j, k), (i, k, j), (j, i, k), (j, k, i), (k, i, j), (k, j, i)]
    if i == j < k:
        return [(i, j, k), (i, k, j), (k, i, j)]
    if i < j == k:
        return [(i, j, k), (j, i, k), (j, k, i)]
    return [(i, j, k)]


class T3StepCPU:
    """Inputs of one T3 half-iteration at (nocc, nvir) on the host, seeded (values do not
    change the time of the dense work; the case structure is that of the reference)."""

    def __init__(self, nocc, nvir, seed=0):
        rng = np.random.default_rng(seed)
        no, nv = nocc, nvir
        self.no, self.nv = no, nv
        self.trip = [(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)]
        self.n3 = len(self.trip)
        self.pos = {t: q for q, t in enumerate(self.trip)}
        self.loc = np.arange(self.n3, dtype=np.int64)
        r = lambda *s, sc=0.1: rng.standard_normal(s) * sc  # noqa: E731
        self.W_vvvv, self.W_vvvo, self.W_vooo = r(nv, nv, nv, nv), r(nv, nv, nv, no), r(nv, no, no, no)
        self.W_ovov, self.W_ovvo, self.W_oooo = r(no, nv, no, nv), r(no, nv, nv, no), r(no, no, no, no)
        self.F_vv, self.F_oo = np.diag(rng.uniform(0.1, 3.0, nv)), np.diag(rng.uniform(-1.5, -0.3, no))
        self.t2 = r(no, no, nv, nv, sc=1e-2)
        self.t1_fock, self.t1_eris_oovv = r(no + nv, no + nv), r(no, no, nv, nv)
        self.t1_eris_vovv, self.t1_eris_ooov = r(nv, no, nv, nv), r(no, no, no, nv)
        self.t3 = rng.standard_normal((self.n3, nv, nv, nv)) * 1e-3
        self.eia = rng.uniform(-4.5, -0.4, (no, nv))
        self.h = _Helpers()
        # one target block of each occupied case, and how many blocks share it
        cases = {}
        for t in self.trip:
            i, j, k = t
            key = (i < j, j < k)
            cases.setdefault(key, []).append(t)
        self.sample = [(v[len(v) // 2], len(v)) for v in cases.values()]
        self._src_forms = (self.h.transpose_add(self.t3[0], nv), self.h.triple_sym(self.t3[0], nv))

    # ------------------------------------------------------------------ per target
    def _target(self, i, j, k):
        """All per-block work of target (i, j, k) in one iteration; returns its r3."""
        no, nv, h, e = self.no, self.nv, self.h, lambda s, a, b: np.einsum(s, a, b, optimize=True)
        t3, W3, Wo, F, t2 = self.t3, self.W_vvvo, self.W_vooo, self.F_vv, self.t2
        q = self.pos[(i, j, k)]
        tmp = np.empty((nv, nv, nv))
        # feedback: r1 (P3_422) and, for every ordering, r2 and W (P3_201)
        h.take(t3, self.loc, i, j, k, no, nv, tmp)
        h.p3(tmp, nv, "P3_422")
        r1 = np.zeros((no, nv))
        E = self.t1_eris_oovv
        r1[i] += 0.5 * e('bc,abc->a', E[j, k], tmp) + 0.5 * e('cb,acb->a', E[j, k], tmp)
        r1[j] += 0.5 * e('bc,bac->a', E[i, k], tmp) + 0.5 * e('cb,cab->a', E[i, k], tmp)
        r1[k] += 0.5 * e('bc,bca->a', E[i, j], tmp) + 0.5 * e('cb,cba->a', E[i, j], tmp)
        r2 = np.zeros((no, no, nv, nv))
        Wv = np.zeros((nv, nv, nv, no))
        Wvo = np.zeros((nv, no, no, no))
        for (pi, pj, pk) in _perms(i, j, k):
            for _ in range(2):  # the r2 pass and the W pass each take and symmetrize again
                h.take(t3, self.loc, pi, pj, pk, no, nv, tmp)
                h.p3(tmp, nv, "P3_201")
            r2[pj, pk] += 0.5 * e("a,abc->bc", self.t1_fock[pi, no:], tmp)
            r2[pj, pk] += e("cad,dba->bc", self.t1_eris_vovv[:, pi], tmp)
            r2[pj] -= e("la,abc->lbc", self.t1_eris_ooov[pk, pi], tmp)
            Wvo[:, :, pj, pk] += e('mde,ead->am', E[:, pi], tmp)
            Wv[:, :, :, pj] -= e('de,eba->abd', E[pk, pi], tmp)
        # compute_r3_tri per-block part
        r = e('abd,dc->abc', W3[..., j], t2[i, k])
        r += e('acd,db->abc', W3[..., k], t2[i, j])
        r += e('bad,dc->abc', W3[..., i], t2[j, k])
        r += e('bcd,da->abc', W3[..., k], t2[j, i])
        r += e('cad,db->abc', W3[..., i], t2[k, j])
        r += e('cbd,da->abc', W3[..., j], t2[k, i])
        r -= e('al,lbc->abc', Wo[:, :, i, j], t2[:, k])
        r -= e('al,lcb->abc', Wo[:, :, i, k], t2[:, j])
        r -= e('bl,lac->abc', Wo[:, :, j, i], t2[:, k])
        r -= e('bl,lca->abc', Wo[:, :, j, k], t2[:, i])
        r -= e('cl,lab->abc', Wo[:, :, k, i], t2[:, j])
        r -= e('cl,lba->abc', Wo[:, :, k, j], t2[:, i])
        r += e('ad,dbc->abc', F, t3[q])
        r += e('bd,adc->abc', F, t3[q])
        r += e('cd,abd->abc', F, t3[q])
        # OO batch: every source block whose cases match this target (distr_cc/rccsdt.py:538-596);
        # a source's transpose-add / triple-sym forms are made once per source for all targets
        # (timed in _sources), so here one prepared set stands in for each source's
        Wov, Wvo2 = self.W_ovov, self.W_ovvo
        T2, V = self._src_forms
        for (o0, o1, o2) in self.trip:
            m3 = [j == o0 and k == o1, o1 != o2 and j == o0 and k == o2, o0 != o1 and j == o1 and k == o2]
            m4 = [i == o0 and k == o1, o1 != o2 and i == o0 and k == o2, o0 != o1 and i == o1 and k == o2]
            m5 = [i == o0 and j == o1, o1 != o2 and i == o0 and j == o2, o0 != o1 and i == o1 and j == o2]
            if not any(m3 + m4 + m5):
                continue
            src = t3[self.pos[(o0, o1, o2)]]
            ls = (o2, o1, o0)
            for part, (occ, m) in enumerate(((i, m3), (j, m4), (k, m5))):
                for cs in range(3):
                    if m[cs]:
                        l = ls[cs]
                        r -= e('bd,dca->abc', Wov[l, :, occ, :], src)
                        r -= 0.5 * e('ad,dcb->abc', Wov[l, :, occ, :], T2)
                        r -= e('cd,bda->abc', Wov[l, :, occ, :], src)
                        r += 0.5 * e('ad,bcd->abc', Wvo2[l, :, :, occ], V[cs])
        # W_vvvv.t3
        r += e('abde,dec->abc', self.W_vvvv, t3[q])
        r += e('acde,dbe->abc', self.W_vvvv, t3[q])
        r += e('bcde,ade->abc', self.W_vvvv, t3[q])
        # P3_full, divide, norm, update
        r = np.ascontiguousarray(r)
        h.p3(r, nv, "P3_full", -1.0 / 6.0, 1.0)
        r /= self.eia[i][:, None, None] + self.eia[j][None, :, None] + self.eia[k][None, None, :]
        float(np.vdot(r, r))
        t3[q] += r
        return r

    # ------------------------------------------------------------------ global parts
    def _prefactors(self, frac=10):
        """The F_oo / W_oooo prefactor loop (distr_cc/rccsdt.py:627-723) over 1/frac of the
        source blocks; returns seconds scaled to all of them."""
        pf = np.zeros((6, self.n3, self.n3))
        Wq, Fo = self.W_oooo, self.F_oo
        src = self.trip[::frac]
        t0 = time.perf_counter()
        for idx, (o0, o1, o2) in enumerate(src):
            for q, (i, j, k) in enumerate(self.trip):
                if k == o2:
                    pf[0, idx, q] += Wq[o0, o1, i, j]
                if o1 != o2 and k == o1:
                    pf[1, idx, q] += Wq[o0, o2, i, j]
                    pf[3, idx, q] += Wq[o2, o0, i, j]
                if o0 != o1 and k == o2:
                    pf[2, idx, q] += Wq[o1, o0, i, j]
                if o0 != o1 and k == o0:
                    pf[4, idx, q] += Wq[o1, o2, i, j]
                    if o1 != o2:
                        pf[5, idx, q] += Wq[o2, o1, i, j]
                if j == o2:
                    pf[1, idx, q] += Wq[o0, o1, i, k]
                if o1 != o2 and j == o1:
                    pf[0, idx, q] += Wq[o0, o2, i, k]
                    pf[5, idx, q] += Wq[o2, o0, i, k]
                if o0 != o1 and j == o2:
                    pf[4, idx, q] += Wq[o1, o0, i, k]
                if o0 != o1 and j == o0:
                    pf[2, idx, q] += Wq[o1, o2, i, k]
                    if o1 != o2:
                        pf[3, idx, q] += Wq[o2, o1, i, k]
                if i == o2:
                    pf[3, idx, q] += Wq[o0, o1, j, k]
                if o1 != o2 and i == o1:
                    pf[2, idx, q] += Wq[o0, o2, j, k]
                    pf[4, idx, q] += Wq[o2, o0, j, k]
                if o0 != o1 and i == o2:
                    pf[5, idx, q] += Wq[o1, o0, j, k]
                if o0 != o1 and i == o0:
                    pf[0, idx, q] += Wq[o1, o2, j, k]
                    if o1 != o2:
                        pf[1, idx, q] += Wq[o2, o1, j, k]
                if j == o0 and k == o1:
                    pf[3, idx, q] -= Fo[o2, i]
                if o1 != o2 and j == o0 and k == o2:
                    pf[2, idx, q] -= Fo[o1, i]
                if o0 != o1 and j == o1 and k == o2:
                    pf[0, idx, q] -= Fo[o0, i]
                if i == o0 and k == o1:
                    pf[1, idx, q] -= Fo[o2, j]
                if o1 != o2 and i == o0 and k == o2:
                    pf[0, idx, q] -= Fo[o1, j]
                if o0 != o1 and i == o1 and k == o2:
                    pf[2, idx, q] -= Fo[o0, j]
                if i == o0 and j == o1:
                    pf[0, idx, q] -= Fo[o2, k]
                if o1 != o2 and i == o0 and j == o2:
                    pf[1, idx, q] -= Fo[o1, k]
                if o0 != o1 and i == o1 and j == o2:
                    pf[4, idx, q] -= Fo[o0, k]
        return (time.perf_counter() - t0) * self.n3 / len(src)

    def _prefactor_gemms(self, frac=32):
        """The six dense 'pq,pabc->qabc' GEMMs (distr_cc/rccsdt.py:726-731) on 1/frac of
        their columns; seconds scaled to all columns."""
        nv3 = self.nv ** 3
        cols = max(1, nv3 // frac)
        pf = np.random.default_rng(1).standard_normal((self.n3, self.n3))
        src = np.ascontiguousarray(self.t3.reshape(self.n3, nv3)[:, :cols])
        t0 = time.perf_counter()
        for _ in range(6):
            out = pf.T @ src
        del out
        return (time.perf_counter() - t0) * nv3 / cols

    def _sources(self, nsrc=4):
        """transpose-add + triple-sym of every source block (distr_cc/rccsdt.py:531-532),
        timed on nsrc of them; seconds scaled to all."""
        t0 = time.perf_counter()
        for q in range(nsrc):
            src = self.t3[q * (self.n3 // nsrc)]
            self.h.transpose_add(src, self.nv)
            self.h.triple_sym(src, self.nv)
        return (time.perf_counter() - t0) * self.n3 / nsrc

    def _diis(self, space=6, frac=16):
        """One unified DIIS update (distr_cc/diis.py:105-177) with `space` filled slots over
        1/frac of the T3 vector; seconds scaled to the whole vector."""
        n = self.t3.size // frac
        rng = np.random.default_rng(2)
        xs = [rng.standard_normal(n) for _ in range(space)]
        es = [rng.standard_normal(n) for _ in range(space)]
        x, xprev = rng.standard_normal(n), rng.standard_normal(n)
        t0 = time.perf_counter()
        err = x - xprev
        row = [float(np.dot(err, ei)) for ei in es]
        c = np.linalg.solve(np.eye(space) + 1e-3 * np.ones((space, space)), np.array(row))
        xnew = np.zeros(n)
        for ci, xi in zip(c, xs):
            xnew += xi * ci
        d = xnew - xprev
        float(np.dot(d, d))
        return (time.perf_counter() - t0) * frac

    def step(self):
        """Seconds of one full T3 half-iteration, extrapolated from the sample; and a
        description of the sample."""
        per_target = 0.0
        for (i, j, k), count in self.sample:
            t0 = time.perf_counter()
            self._target(i, j, k)
            per_target += (time.perf_counter() - t0) * count
        total = per_target + self._sources() + self._prefactors() + self._prefactor_gemms() + self._diis()
        return total


def describe(nocc, nvir):
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    return ("%d of %d canonical blocks timed (one per occupied case i<j<k, i=j<k, i<j=k, i=j=k, weighted by "
            "the case counts): feedback, compute_r3_tri per-block einsums, the matching OO-batch einsums, "
            "W_vvvv.t3, P3_full/divide/update; global parts on slices scaled linearly: source transpose-add + "
            "triple-sym (4 blocks), F_oo/W_oooo prefactor loop (1/10 of sources), dense prefactor GEMMs (1/32 "
            "of columns), DIIS update (1/16 of the vector, 6 slots)" % (4 if nocc >= 3 else nocc, n3))
