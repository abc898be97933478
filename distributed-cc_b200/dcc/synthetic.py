"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (no molecule, no integral engine needed):

  orbital energies  e_occ ~ U[-1.5, -0.3], e_vir ~ U[0.1, 3.0]
  t2                N(0, 1e-2), symmetrised t2[i,j,a,b] = t2[j,i,b,a]
  ERIs (pq|rs)      N(0, 0.1) averaged over the 8-fold permutational symmetry
  t3                N(0, 1e-3), symmetrised over the simultaneous permutations
                    of (i,j,k) and (a,b,c), stored as canonical i<=j<=k blocks
  intermediates     the physicist ERI slices <pq|rs> = (pr|qs):
                    W_vvvv = <ab|cd>, W_vvvo = <ab|ci>, W_vooo = <ai|jk>,
                    W_ovov = <ia|jb>, W_ovvo = <ia|bj>, W_oooo = <ij|kl>;
                    F_vv, F_oo = diag(e) + symmetric N(0, 1e-2) coupling

Everything is generated on the given device with a torch generator seeded
from `seed`, so GPU benchmark inputs of several GB are made in seconds.
"""
from __future__ import annotations

import itertools

import torch

f64 = torch.float64


class Inputs:
    pass


def _sym8(g):
    """Average of the 8 permutations of (pq|rs) that leave real ERIs invariant."""
    perms = [(0, 1, 2, 3), (1, 0, 2, 3), (0, 1, 3, 2), (1, 0, 3, 2), (2, 3, 0, 1), (3, 2, 0, 1), (2, 3, 1, 0),
             (3, 2, 1, 0)]
    out = torch.zeros_like(g)
    for p in perms:
        out += g.permute(p)
    return out / 8.0


def canonical_ijk(nocc):
    return [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]


def symmetric_t3_blocks(nocc, nvir, gen, device, scale=1e-3):
    """Canonical blocks of a T3 with t[P(ijk), P(abc)] = t[ijk, abc]."""
    full = torch.randn((nocc,) * 3 + (nvir,) * 3, dtype=f64, device=device, generator=gen) * scale
    sym = torch.zeros_like(full)
    for p in itertools.permutations(range(3)):
        sym += full.permute(p + tuple(3 + x for x in p))
    sym /= 6.0
    del full
    idx = torch.tensor(canonical_ijk(nocc), device=device)
    out = sym[idx[:, 0], idx[:, 1], idx[:, 2]].contiguous()
    del sym
    return out


def make_inputs(nocc, nvir, seed=0, device="cuda", with_t3=True):
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    no, nv = nocc, nvir
    nmo = no + nv
    d = Inputs()
    d.nocc, d.nvir = no, nv
    d.e_occ = (torch.rand(no, dtype=f64, device=device, generator=gen) * 1.2 - 1.5).sort().values
    d.e_vir = (torch.rand(nv, dtype=f64, device=device, generator=gen) * 2.9 + 0.1).sort().values
    t2 = torch.randn(no, no, nv, nv, dtype=f64, device=device, generator=gen) * 1e-2
    d.t2 = ((t2 + t2.permute(1, 0, 3, 2)) * 0.5).contiguous()
    eri = _sym8(torch.randn(nmo, nmo, nmo, nmo, dtype=f64, device=device, generator=gen) * 0.1)
    o, v = slice(0, no), slice(no, nmo)
    phys = lambda p, q, r, s: eri[p, r, q, s].permute(0, 2, 1, 3).contiguous()  # <pq|rs> = (pr|qs)  # noqa: E731
    d.W_vvvv = phys(v, v, v, v)
    d.W_vvvo = phys(v, v, v, o)
    d.W_vooo = phys(v, o, o, o)
    d.W_ovov = phys(o, v, o, v)
    d.W_ovvo = phys(o, v, v, o)
    d.W_oooo = phys(o, o, o, o)
    d.eris_vvoo = phys(v, v, o, o)
    d.eris_vooo = d.W_vooo
    d.eris_vvvo = d.W_vvvo
    d.eris_ovvo = d.W_ovvo
    d.eris_ovov = d.W_ovov
    d.eris_oooo = d.W_oooo
    d.eris_vvvv = d.W_vvvv
    del eri
    cv = torch.randn(nv, nv, dtype=f64, device=device, generator=gen) * 1e-2
    co = torch.randn(no, no, dtype=f64, device=device, generator=gen) * 1e-2
    d.F_vv = (torch.diag(d.e_vir) + 0.5 * (cv + cv.t())).contiguous()
    d.F_oo = (torch.diag(d.e_occ) + 0.5 * (co + co.t())).contiguous()
    d.eia = (d.e_occ[:, None] - d.e_vir[None, :]).contiguous()
    if with_t3:
        d.t3 = symmetric_t3_blocks(no, nv, gen, device)
    d.ijk = torch.tensor(canonical_ijk(no), dtype=torch.int32, device=device)
    return d


def to_numpy(d):
    """Host copies of every tensor attribute (for the oracle)."""
    out = Inputs()
    for k, v in vars(d).items():
        setattr(out, k, v.detach().cpu().numpy() if isinstance(v, torch.Tensor) else v)
    return out


def make_t4_inputs(nocc, nvir, seed=0, device="cuda"):
    """Inputs of one T4 update (compute_r4_tri and the steps after it) with the
    distributions above: the full ERI tensor <pq|rs> as the t1-dressed `eris`, the
    physicist slices as the W intermediates, a full T3 [nocc^3, nvir^3] and the stored
    T4 blocks [n4, nvir^4] (i<=j<=k<=l without the zero-rule blocks), both invariant
    under simultaneous permutations of occupied and virtual indices (t3 N(0, 1e-3),
    t4 N(0, 1e-4) before symmetrisation); `ijkl` lists the stored quadruples (int32)."""
    from .t4_residual import stored_quadruples
    d = make_inputs(nocc, nvir, seed=seed, device=device, with_t3=False)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed + 1)
    no, nv = nocc, nvir
    nmo = no + nv
    eri = _sym8(torch.randn(nmo, nmo, nmo, nmo, dtype=f64, device=device, generator=gen) * 0.1)
    d.eris = eri.permute(0, 2, 1, 3).contiguous()
    del eri
    full = torch.randn((no,) * 3 + (nv,) * 3, dtype=f64, device=device, generator=gen) * 1e-3
    t3 = torch.zeros_like(full)
    for p in itertools.permutations(range(3)):
        t3 += full.permute(p + tuple(3 + x for x in p))
    d.t3 = (t3 / 6.0).contiguous()
    del full, t3
    full = torch.randn((no,) * 4 + (nv,) * 4, dtype=f64, device=device, generator=gen) * 1e-4
    t4 = torch.zeros_like(full)
    for p in itertools.permutations(range(4)):
        t4 += full.permute(p + tuple(4 + x for x in p))
    del full
    quads = stored_quadruples(no)
    rows = torch.tensor([((i * no + j) * no + k) * no + l for i, j, k, l in quads], device=device)
    d.t4 = (t4.view(no ** 4, -1)[rows] / 24.0).view((len(quads),) + (nv,) * 4).contiguous()
    del t4
    d.ijkl = torch.tensor(quads, dtype=torch.int32, device=device)
    return d
