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
