"""The "cuda" einsum backend: the drop-in that routes the reference driver's
triples / quadruples hot path onto this library (distr_cc/rccsdt.py,
distr_cc/rccsdt_q.py, distr_cc/rccsdtq.py).

`install(rccsdt_module, rccsdt_q_module, rccsdtq_module)` wraps the reference's
hot functions

    r1r2_add_t3_tri_(mycc, imds, r1, r2, t3)          distr_cc/rccsdt.py:253
    intermediates_t3_add_t3_tri(mycc, imds, t3)        distr_cc/rccsdt.py:323
    compute_r3_tri(mycc, imds, t2, t3)                 distr_cc/rccsdt.py:368
    rccsdt_q.kernel(mycc, eris, tamps, blksize, comm)  distr_cc/rccsdt_q.py:227
    compute_r4_tri(mycc, imds, t2, t3, t4)             distr_cc/rccsdtq.py:834
    r2_add_t4_tri_(mycc, imds, r2, t4)                 distr_cc/rccsdtq.py:471
    r3_add_t4_tri_(mycc, imds, r3, t4)                 distr_cc/rccsdtq.py:577

so that, when `mycc.einsum_backend == "cuda"` (set through the reference's
own RCCSDT.set_einsum_backend, distr_cc/rccsdt.py:1255), they run on the GPU
with the reference's argument meaning and return values; any other backend
string calls the original.  The GPU path is one rank only: a communicator of
size > 1 raises.  When mpi4py is absent, `SingleRankComm` stands in for
MPI.COMM_WORLD.  Host numpy arrays cross to the device on entry and back on
exit; the per-shape GPU objects (buffers, splits) are cached on `mycc`.
"""
from __future__ import annotations

import numpy as np
import torch

f64 = torch.float64
BACKEND = "cuda"


class SingleRankComm:
    """The part of an MPI communicator the reference's one-rank path uses."""

    rank, size = 0, 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def bcast(self, obj, root=0):
        return obj

    def Barrier(self):
        return None

    def Allreduce(self, sendbuf, recvbuf=None, op=None):
        # MPI.IN_PLACE or (send, recv) at one rank: recv = send
        if recvbuf is not None and not isinstance(sendbuf, (str, type(None))) and sendbuf is not recvbuf:
            try:
                np.copyto(recvbuf, sendbuf)
            except TypeError:
                pass
        return None

    def allreduce(self, obj, op=None):
        return obj


def comm_size(mycc):
    comm = getattr(mycc, "comm", None)
    return 1 if comm is None else int(comm.Get_size())


def require_single_rank(mycc):
    if comm_size(mycc) != 1:
        raise RuntimeError('einsum backend "cuda" runs on one rank; got a communicator of size %d' % comm_size(mycc))


def uses_cuda(mycc):
    return getattr(mycc, "einsum_backend", None) == BACKEND


def _dev(a, device):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=f64, device=device)


class _Inputs:
    pass


def _ijk(nocc, device):
    from .synthetic import canonical_ijk
    return torch.tensor(canonical_ijk(nocc), dtype=torch.int32, device=device)


def _state(mycc):
    st = getattr(mycc, "_dcc_state", None)
    if st is None:
        st = {}
        mycc._dcc_state = st
    return st


def precision_of(mycc):
    return getattr(mycc, "dcc_precision", "bf16x3")


def compute_r3_tri(mycc, imds, t2, t3):
    """r3 for the canonical blocks (distr_cc/rccsdt.py:368-433, OO terms :435-732) on the GPU."""
    from . import t3_residual
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc, nvir = mycc.nocc, mycc.nmo - mycc.nocc
    _, t3_local = t3
    st = _state(mycc)
    key = ("r3", nocc, nvir, precision_of(mycc))
    if key not in st:
        st[key] = t3_residual.T3Residual(nocc, nvir, precision_of(mycc), dev, with_oo=True)
    res = st[key]
    d = _Inputs()
    for name in ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo"):
        setattr(d, name, _dev(getattr(imds, name), dev))
    d.t2 = _dev(t2, dev)
    d.ijk = _ijk(nocc, dev)
    r3 = res.compute(d, _dev(t3_local, dev))
    if not res.status_ok():
        raise RuntimeError("a bounded wait in a GPU kernel gave up (timeout)")
    return r3.cpu().numpy()


def r1r2_add_t3_tri_(mycc, imds, r1, r2, t3):
    """distr_cc/rccsdt.py:253-321 on the GPU; r1, r2 updated in place and returned."""
    from . import t3_feedback
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc = mycc.nocc
    _, t3_local = t3
    dt3 = _dev(t3_local, dev)
    eris = _dev(imds.t1_eris, dev)
    d1, d2 = _dev(r1, dev), _dev(r2, dev)
    t3_feedback.r1_add_t3_(d1, eris, dt3, _ijk(nocc, dev), nocc)
    X = t3_feedback.p3_201_all(dt3, nocc)
    t3_feedback.r2_add_t3_(d2, _dev(imds.t1_fock, dev), eris, X, nocc)
    r1[...] = d1.cpu().numpy()
    r2[...] = d2.cpu().numpy()
    return r1, r2


def intermediates_t3_add_t3_tri(mycc, imds, t3):
    """distr_cc/rccsdt.py:323-366 on the GPU; imds.W_vooo, imds.W_vvvo updated in place."""
    from . import t3_feedback
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc = mycc.nocc
    _, t3_local = t3
    X = t3_feedback.p3_201_all(_dev(t3_local, dev), nocc)
    Wo, Wv = _dev(imds.W_vooo, dev), _dev(imds.W_vvvo, dev)
    t3_feedback.intermediates_t3_add_(Wo, Wv, _dev(imds.t1_eris, dev), X, nocc)
    imds.W_vooo[...] = Wo.cpu().numpy()
    imds.W_vvvo[...] = Wv.cpu().numpy()
    return imds


def q_kernel(mycc, eris=None, tamps=None, blksize=4, comm=None, job_idx=0, n_jobs=1, log_redistribution=False):
    """(e_q_bracket, e_q_paren) of distr_cc/rccsdt_q.py:227 on the GPU, one rank: every task,
    or with n_jobs > 1 the tasks of job `job_idx` (the reference's contiguous slice of its task
    order, distr_cc/rccsdt_q.py:359-366), whose energies add up over the jobs."""
    from . import rccsdt_q
    if comm is not None and int(comm.Get_size()) != 1:
        raise RuntimeError('einsum backend "cuda" runs on one rank')
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc, nmo = mycc.nocc, mycc.nmo
    if eris is None:
        eris = mycc.ao2mo(mycc.mo_coeff)
    tamps = tamps if tamps is not None else mycc.tamps
    _, t2, t3 = tamps
    dt3, t3_local = t3
    # T3 already in the ABC layout (prepare_tamps_for_q, distr_cc/rccsdt_q.py:58-66)
    is_abc = dt3 is not None and hasattr(dt3, "abc_to_global_idx")
    p = eris.pppp
    o, v = slice(0, nocc), slice(nocc, nmo)
    er = {"vvvo": p[v, v, v, o], "vooo": p[v, o, o, o], "vvoo": p[v, v, o, o], "ovvo": p[o, v, v, o],
          "ovov": p[o, v, o, v], "vvvv": p[v, v, v, v], "oooo": p[o, o, o, o]}
    er = {k: _dev(a, dev) for k, a in er.items()}
    nvir = nmo - nocc
    t2q = t2 if t2.shape == (nvir, nvir, nocc, nocc) else np.ascontiguousarray(np.transpose(t2, (2, 3, 0, 1)))
    e = np.asarray(eris.mo_energy)
    t3d = _dev(t3_local, dev)
    return rccsdt_q.q_energy(er, _dev(t2q, dev), None if is_abc else t3d, _dev(e[:nocc], dev), _dev(e[nocc:], dev),
                             nocc, nvir, blksize, precision_of(mycc), job_idx=job_idx, n_jobs=n_jobs,
                             t3_abc=t3d if is_abc else None)


# imds fields compute_r4_tri releases on return (distr_cc/rccsdtq.py:899-1349)
_R4_RELEASED = ("W_vvvo", "W_vooo", "W_oovvvo", "W_ovovvo", "W_ooooov", "W_oooovv", "W_oovvvv", "t1_eris", "F_vv",
                "W_vvvv", "F_oo", "W_oooo", "W_ovvo", "W_ovov")


def compute_r4_tri(mycc, imds, t2, t3, t4):
    """r4_local of distr_cc/rccsdtq.py:834 (with its OO batch, :1062) on the GPU, one rank:
    t2 [i,j,a,b], t3 the full [i,j,k,a,b,c], t4 = (dt4, t4_local) with every stored block local."""
    from . import t4_residual
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc = mycc.nocc
    t4_local = _t4_local(mycc, t4)
    quads = t4_residual.stored_quadruples(nocc)
    d = lambda a: _dev(a, dev)  # noqa: E731
    r4 = torch.zeros((len(quads),) + tuple(t4_local.shape[1:]), dtype=f64, device=dev)
    t4_residual.compute_r4_tri_(r4, d(imds.t1_eris), d(imds.F_vv), d(imds.W_vvvo), d(imds.W_vooo), d(imds.W_vvvv),
                                d(imds.W_oooo), d(imds.W_ovov), d(t2), d(t3), d(t4_local), nocc,
                                precision_of(mycc), F_oo=d(imds.F_oo), W_ovvo=d(imds.W_ovvo))
    out = r4.cpu().numpy()
    for name in _R4_RELEASED:
        if hasattr(imds, name):
            setattr(imds, name, None)
    return out


def _t4_local(mycc, t4):
    from . import t4_residual
    dt4, t4_local = t4
    quads = t4_residual.stored_quadruples(mycc.nocc)
    local = [tuple(int(x) for x in q[:4]) for q in dt4.iter_local_ijkl()] if hasattr(dt4, "iter_local_ijkl") \
        else quads
    if local != quads or len(t4_local) != len(quads):
        raise RuntimeError('einsum backend "cuda" needs every stored T4 block local, in stored order')
    return t4_local


def r2_add_t4_tri_(mycc, imds, r2, t4):
    """distr_cc/rccsdtq.py:471-575 on the GPU, one rank: r2 += the T4 part, in place."""
    from . import t4_residual
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    t4_local = _t4_local(mycc, t4)
    r = _dev(r2, dev)
    t4_residual.r2_add_t4_(r, _dev(t4_local, dev), _dev(imds.t1_eris, dev), mycc.nocc, precision_of(mycc))
    r2[...] = r.cpu().numpy()
    return r2


def r3_add_t4_tri_(mycc, imds, r3, t4):
    """distr_cc/rccsdtq.py:577-683 on the GPU, one rank: r3 (full) += the T4 part, in place."""
    from . import t4_residual
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    t4_local = _t4_local(mycc, t4)
    r = _dev(r3, dev)
    t4_residual.r3_add_t4_(r, _dev(t4_local, dev), _dev(imds.t1_fock, dev), _dev(imds.t1_eris, dev), mycc.nocc,
                           precision_of(mycc))
    r3[...] = r.cpu().numpy()
    return r3


_ROUTES = {"r1r2_add_t3_tri_": r1r2_add_t3_tri_, "intermediates_t3_add_t3_tri": intermediates_t3_add_t3_tri,
           "compute_r3_tri": compute_r3_tri}
_R4_ROUTES = {"compute_r4_tri": None, "r2_add_t4_tri_": r2_add_t4_tri_, "r3_add_t4_tri_": r3_add_t4_tri_}


HOST_EINSUM = "numpy"


def _host_einsum(orig):
    """The module's _einsum(backend, subscripts, *operands, out=, alpha=, beta=) with the
    backend string "cuda" read as HOST_EINSUM: the reference code this library does not route
    (the lower-order equations and the other intermediates) keeps running on the host."""
    def einsum(backend, *args, **kw):
        return orig(HOST_EINSUM if backend == BACKEND else backend, *args, **kw)
    einsum._dcc_wrapped = True
    einsum.__name__ = getattr(orig, "__name__", "_einsum")
    einsum.__doc__ = orig.__doc__
    return einsum


def install(rccsdt_module, rccsdt_q_module=None, rccsdtq_module=None, host_einsum_modules=()):
    """Route the reference's hot functions to the GPU when mycc.einsum_backend == "cuda".
    Every given module's `_einsum` (the reference modules bind PySCF's at import,
    distr_cc/rccsdt.py:27; pass pyscf.cc.rccsdt in host_einsum_modules for PySCF's own
    lower-order code) reads "cuda" as the host backend.  Idempotent; returns the names it
    wrapped."""
    wrapped = []
    for mod in (rccsdt_module, rccsdt_q_module, rccsdtq_module) + tuple(host_einsum_modules):
        orig = getattr(mod, "_einsum", None) if mod is not None else None
        if orig is not None and not getattr(orig, "_dcc_wrapped", False):
            mod._einsum = _host_einsum(orig)
            wrapped.append("%s._einsum" % getattr(mod, "__name__", "module"))
    for name, fn in _ROUTES.items():
        orig = getattr(rccsdt_module, name, None)
        if orig is None or getattr(orig, "_dcc_wrapped", False):
            continue

        def wrapper(mycc, *args, _orig=orig, _fn=fn, **kw):
            return _fn(mycc, *args, **kw) if uses_cuda(mycc) else _orig(mycc, *args, **kw)

        wrapper._dcc_wrapped = True
        wrapper.__name__ = name
        wrapper.__doc__ = orig.__doc__
        setattr(rccsdt_module, name, wrapper)
        wrapped.append(name)
    if rccsdt_q_module is not None:
        orig = getattr(rccsdt_q_module, "kernel", None)
        if orig is not None and not getattr(orig, "_dcc_wrapped", False):
            def qwrap(mycc, *args, _orig=orig, **kw):
                return q_kernel(mycc, *args, **kw) if uses_cuda(mycc) else _orig(mycc, *args, **kw)
            qwrap._dcc_wrapped = True
            qwrap.__name__ = "kernel"
            rccsdt_q_module.kernel = qwrap
            wrapped.append("rccsdt_q.kernel")
    if rccsdtq_module is not None:
        for name, fn in _R4_ROUTES.items():
            fn = compute_r4_tri if fn is None else fn
            orig = getattr(rccsdtq_module, name, None)
            if orig is None or getattr(orig, "_dcc_wrapped", False):
                continue

            def r4wrap(mycc, *args, _orig=orig, _fn=fn, **kw):
                return _fn(mycc, *args, **kw) if uses_cuda(mycc) else _orig(mycc, *args, **kw)
            r4wrap._dcc_wrapped = True
            r4wrap.__name__ = name
            r4wrap.__doc__ = orig.__doc__
            setattr(rccsdtq_module, name, r4wrap)
            wrapped.append("rccsdtq." + name)
    return wrapped
