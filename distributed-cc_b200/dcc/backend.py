"""The "cuda" einsum backend: the drop-in that routes the reference driver's
triples / quadruples hot path onto this library (distr_cc/rccsdt.py,
distr_cc/rccsdt_q.py, distr_cc/rccsdtq.py).

`install(rccsdt_module, rccsdt_q_module, rccsdtq_module)` wraps the reference's
hot functions

    update_amps_rccsdt_tri_(mycc, tamps, eris)         distr_cc/rccsdt.py:890
    run_diis_t3(mycc, tamps, t3_local, ...)            distr_cc/rccsdt.py:1026
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
MPI.COMM_WORLD.

T3 stays in HBM across an iteration and across iterations.  The routed
update_amps_rccsdt_tri_ (and RCCSDT.update_amps_, the class attribute the
reference's kernel calls) uploads t3_local once and puts a `DeviceT3Local`
in its place in `tamps`; the feedback, the residual, the update and the
unified DIIS then all work on that device array, and each iteration moves
over the host link only the intermediates the host-side lower-order code
produced (the slices of them the T3 path reads), r1/r2's T3 parts and two
norms.  `DeviceT3Local` reads back to numpy on demand (`np.asarray`,
indexing), so code outside the path that inspects t3_local still works.
The single-function routes (compute_r3_tri and the feedback) take either
kind of t3_local and keep the reference's host return values.  The
per-shape GPU objects (buffers, splits) are cached on `mycc`.
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


class _Transfer:
    """Bytes the routes moved between host and device since the last reset (host-link traffic
    of the drop-in path)."""

    def __init__(self):
        self.reset()

    def reset(self):
        self.h2d = 0
        self.d2h = 0


TRANSFER = _Transfer()


class _Staging:
    """Page-locked host buffers for the uploads of the drop-in routes.  A numpy array (any
    positive strides, e.g. a slice of the dressed ERIs) is gathered into a pinned buffer by
    torch's multi-threaded CPU copy and reaches the device by an asynchronous copy at the
    link's speed; a buffer is reused once the copy that last read it has completed.  Arrays
    above `limit` bytes (the one-time upload of T3) go through the pageable path."""

    limit = 1 << 30

    def __init__(self):
        self.bufs = []  # [pinned uint8 tensor, event of its last copy or None]

    def _buffer(self, nbytes):
        for b in self.bufs:
            if b[0].numel() >= nbytes and (b[1] is None or b[1].query()):
                return b
        b = [torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, pin_memory=True), None]
        self.bufs.append(b)
        return b

    def upload(self, a, device, stream=None):
        out = torch.empty(a.shape, dtype=f64, device=device)
        if out.device.type != "cuda":
            return out.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        if a.nbytes > self.limit or a.size == 0 or any(st < 0 for st in a.strides):
            src = torch.from_numpy(np.ascontiguousarray(a))
            if stream is None:
                out.copy_(src)
            else:
                with torch.cuda.stream(stream):
                    out.copy_(src, non_blocking=True)
            return out
        b = self._buffer(a.nbytes)
        host = b[0][:a.nbytes].view(f64).view(a.shape)
        host.copy_(torch.from_numpy(a))
        s = stream if stream is not None else torch.cuda.current_stream(out.device)
        with torch.cuda.stream(s):
            out.copy_(host, non_blocking=True)
            b[1] = torch.cuda.Event()
            b[1].record(s)
        return out


_STAGING = _Staging()


def _dev(a, device):
    if isinstance(a, DeviceT3Local):
        return a.tensor
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=f64)
    a = np.asarray(a, dtype=np.float64)
    TRANSFER.h2d += a.nbytes
    return _STAGING.upload(a, device)


def _dev_async(a, device, state):
    """A numpy array copied to the device on a side stream (counted in TRANSFER): returns the
    device tensor and leaves in state the event that marks its arrival.  The call returns once
    the bytes are in page-locked memory, while kernels already enqueued on the compute stream
    keep running."""
    if isinstance(a, (torch.Tensor, DeviceT3Local)):
        t = _dev(a, device)
        ev = torch.cuda.Event()
        ev.record()
        state["upload_ready"] = ev
        return t
    a = np.asarray(a, dtype=np.float64)
    TRANSFER.h2d += a.nbytes
    side = state.get("upload_stream")
    if side is None:
        side = state["upload_stream"] = torch.cuda.Stream(device=device)
    out = _STAGING.upload(a, device, stream=side)
    out.record_stream(side)
    ev = torch.cuda.Event()
    ev.record(side)
    state["upload_ready"] = ev
    return out


def _host(t):
    """A device tensor read back to a numpy array (counted in TRANSFER)."""
    a = t.cpu().numpy()
    TRANSFER.d2h += a.nbytes
    return a


class DeviceT3Local:
    """t3_local kept in device memory: [n_local_blocks, nvir, nvir, nvir] FP64 in the
    canonical order of the reference's one-rank distribution.  Reads back to a numpy array
    through np.asarray / indexing."""

    def __init__(self, tensor):
        self.tensor = tensor

    shape = property(lambda self: tuple(self.tensor.shape))
    ndim = property(lambda self: self.tensor.dim())
    size = property(lambda self: self.tensor.numel())
    nbytes = property(lambda self: self.tensor.numel() * 8)
    dtype = np.dtype(np.float64)

    def __len__(self):
        return self.tensor.shape[0]

    def __array__(self, dtype=None, copy=None):
        a = self.tensor.cpu().numpy()
        return a if dtype is None else a.astype(dtype)

    def __getitem__(self, idx):
        return self.tensor[idx].cpu().numpy()

    def numpy(self):
        return self.tensor.cpu().numpy()


class _Inputs:
    pass


def _ijk(nocc, device):
    from .synthetic import canonical_ijk
    return torch.tensor(canonical_ijk(nocc), dtype=torch.int32, device=device)


def _t3_local(mycc, t3):
    """t3_local of (dt3, t3_local), checked to hold every canonical block in canonical order
    (the one-rank layout the kernels index by position; a checkpoint written with another
    block order must be loaded through dcc.checkpoint, which reorders)."""
    from .synthetic import canonical_ijk
    dt3, t3_local = t3
    want = canonical_ijk(mycc.nocc)
    if dt3 is not None and hasattr(dt3, "iter_local_ijk"):
        local = [(int(i), int(j), int(k), int(q)) for i, j, k, q in dt3.iter_local_ijk()]
        if [x[:3] for x in local] != want or any(q != n for n, (_, _, _, q) in enumerate(local)):
            raise RuntimeError('einsum backend "cuda" needs every canonical T3 block local, in canonical order')
    if len(t3_local) != len(want):
        raise RuntimeError('einsum backend "cuda" needs every canonical T3 block local, in canonical order')
    return t3_local


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
    t3_local = _t3_local(mycc, t3)
    it = _iteration(mycc)
    d = _Inputs()
    for name in _T3_IMDS:
        setattr(d, name, _dev(getattr(imds, name), dev))
        setattr(imds, name, None)  # released as the reference releases them (distr_cc/rccsdt.py:406-428, 602-603)
    d.t2 = _dev(t2, dev)
    d.ijk = it.ijk
    it._X = None
    r3 = it.res.compute(d, _dev(t3_local, dev))
    if not it.status_ok():
        raise RuntimeError("a bounded wait in a GPU kernel gave up (timeout)")
    return _host(r3)


def r1r2_add_t3_tri_(mycc, imds, r1, r2, t3):
    """distr_cc/rccsdt.py:253-321 on the GPU; r1, r2 updated in place and returned."""
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    it = _iteration(mycc)
    sl = _feedback_slices(mycc, imds, dev)
    dr1, dr2 = it.feedback_r1r2(_dev(_t3_local(mycc, t3), dev), sl["fock_ov"], sl["oovv"], sl["vovv"], sl["ooov"])
    r1 += _host(dr1)
    r2 += _host(dr2)
    return r1, r2


def intermediates_t3_add_t3_tri(mycc, imds, t3):
    """distr_cc/rccsdt.py:323-366 on the GPU; imds.W_vooo, imds.W_vvvo updated in place."""
    from . import t3_feedback, t3_residual
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc = mycc.nocc
    it = _iteration(mycc)
    t3d = _dev(_t3_local(mycc, t3), dev)
    # X is rebuilt here: this route may be called on its own, with a T3 other than the last one
    # (unpacked into a temporary of the residual's U type, so the residual's U is left alone)
    nv = t3d.shape[1]
    U = torch.empty((nocc ** 3, nv, nv, nv), dtype=it.res.udtype, device=t3d.device)
    t3_residual.unpack_all_(t3d, U, nocc, nv)
    it._X = t3_feedback.p3_201_all(t3d, nocc, U=U, out=it.res.S)
    del U
    it._dW = None
    sl = _feedback_slices(mycc, imds, dev)
    Wo, Wv = _dev(imds.W_vooo, dev), _dev(imds.W_vvvo, dev)
    it.feedback_w(Wo, Wv, sl["oovv"])
    imds.W_vooo[...] = _host(Wo)
    imds.W_vvvo[...] = _host(Wv)
    return imds


_T3_IMDS = ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")


def _iteration(mycc):
    """The cached device state of the T3 half-iteration for mycc's shape and precision."""
    from .t3_iteration import T3Iteration
    st = _state(mycc)
    nocc, nvir = mycc.nocc, mycc.nmo - mycc.nocc
    key = ("t3it", nocc, nvir, precision_of(mycc))
    if key not in st:
        for k in [k for k in st if isinstance(k, tuple) and k[0] == "t3it"]:
            del st[k]  # one shape at a time: the buffers are tens of GB at the large shapes
        st[key] = T3Iteration(nocc, nvir, precision_of(mycc), getattr(mycc, "dcc_device", "cuda"))
    return st[key]


def _feedback_slices(mycc, imds, dev):
    """Upload the slices of the dressed Fock matrix and ERIs the T3 feedback reads (cached per
    imds object, so the two feedback passes of one iteration upload them once)."""
    from . import t3_feedback
    st = _state(mycc)
    cached = st.get("fb_slices")
    if cached is not None and cached[0] is imds.t1_eris:
        return cached[1]
    sl = t3_feedback.eris_slices(imds.t1_eris, imds.t1_fock, mycc.nocc)
    sl = {k: _dev(v, dev) for k, v in sl.items()}
    st["fb_slices"] = (imds.t1_eris, sl)
    return sl


def _t3_device(mycc, tamps):
    """The resident device T3 of tamps[2]: uploaded once (and put back into tamps as a
    DeviceT3Local) when it is still a host array."""
    dt3, t3_local = tamps[2]
    t3_local = _t3_local(mycc, (dt3, t3_local))
    if isinstance(t3_local, DeviceT3Local):
        return t3_local.tensor
    T = _dev(t3_local, getattr(mycc, "dcc_device", "cuda")).clone()
    tamps[2] = (dt3, DeviceT3Local(T))
    return T


def update_amps_rccsdt_tri_(mycc, tamps, eris, mod):
    """update_amps_rccsdt_tri_ (distr_cc/rccsdt.py:890-977) with T3 resident on the GPU.

    The lower-order steps are the ones `mod` (the reference module the route is installed
    in) imports from PySCF and run on the host as in the reference: update_t1_fock_eris,
    intermediates_t1t2, compute_r1r2, r1r2_divide_e_, intermediates_t3.  Every T3 step
    (feedback into r1/r2 and W_vooo/W_vvvo, compute_r3_tri, P3_full, the divide, the norms,
    t3 += r3) runs on the device.  Returns res_norm = [|r1|, |r2|, |r3|] and sets
    mycc._last_t3_residual_norm_sq / _last_t3_active_residual_norm_sq as the reference does."""
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nocc, nvir = mycc.nocc, mycc.nmo - mycc.nocc
    t1, t2, _ = tamps
    T = _t3_device(mycc, tamps)
    it = _iteration(mycc)
    mo_energy = np.asarray(eris.mo_energy)
    imds = mod._IMDS()
    mod.update_t1_fock_eris(mycc, imds, t1, eris)
    mod.intermediates_t1t2(mycc, imds, t2)
    r1, r2 = mod.compute_r1r2(mycc, imds, t2)
    sl = _feedback_slices(mycc, imds, dev)
    dr1, dr2 = it.feedback_r1r2(T, sl["fock_ov"], sl["oovv"], sl["vovv"], sl["ooov"])
    r1 += _host(dr1)
    r2 += _host(dr2)
    r2 += r2.transpose(1, 0, 3, 2)
    mod.r1r2_divide_e_(mycc, r1, r2, mo_energy)
    res_norm = [np.linalg.norm(r1), np.linalg.norm(r2)]
    t1 += r1
    t2 += r2
    mod.intermediates_t3(mycc, imds, t2)
    d = _Inputs()
    for name in _T3_IMDS:
        if name != "W_vvvv":
            setattr(d, name, _dev(getattr(imds, name), dev))
    it.feedback_w(d.W_vooo, d.W_vvvo, sl["oovv"])
    W_vvvv = imds.W_vvvv
    imds = None
    _state(mycc).pop("fb_slices", None)
    d.t2 = _dev(t2, dev)
    d.ijk = it.ijk

    def wvvvv_ready():
        # the largest intermediate (nvir^4) comes in while the device runs every other term
        # of the residual; it is needed only by the W_vvvv.t3 GEMMs at the end
        d.W_vvvv = _dev_async(W_vvvv, dev, _state(mycc))
        return _state(mycc)["upload_ready"]

    d.W_vvvv = None
    it.residual(d, T, wvvvv_ready=wvvvv_ready)
    eia = mo_energy[:nocc, None] - mo_energy[None, nocc:] - getattr(mycc, "level_shift", 0.0)
    nd = mod.resolve_nvir_diis(mycc, nvir) if hasattr(mod, "resolve_nvir_diis") else nvir
    norms = _host(it.update(T, _dev(eia, dev), nvir_active=nd))
    if not it.status_ok():
        raise RuntimeError("a bounded wait in a GPU kernel gave up (timeout)")
    mycc._last_t3_residual_norm_sq = float(norms[0])
    mycc._last_t3_active_residual_norm_sq = float(norms[1]) if nd < nvir else float(norms[0])
    res_norm.append(np.sqrt(float(norms[0])))
    return res_norm


def run_diis_t3(mycc, tamps, t3_local, istep, normt, de, adiis_t3, res_norm=None, return_update_norm=False,
                mod=None):
    """run_diis_t3 (distr_cc/rccsdt.py:1026-1067) with the T3 part of the unified vector
    on the GPU: the packed unique T1/T2 (the reference's pack/unpack of `mod`, host side)
    and the resident T3 go through one device DIIS update (dcc.diis.DIIS, the reference's
    distr_cc/diis.py algorithm); `adiis_t3` (the reference's DIIS object) supplies the
    space and receives last_delta_norm_sq for the update norm."""
    if not (adiis_t3 and istep >= mycc.diis_start_cycle and abs(de) < mycc.diis_start_energy_diff):
        if return_update_norm:
            update_norm = float(normt) if res_norm is None else \
                np.sqrt(max(sum(float(x) * float(x) for x in res_norm), 0.0))
            return tamps, update_norm
        return tamps
    require_single_rank(mycc)
    dev = getattr(mycc, "dcc_device", "cuda")
    nvir = mycc.nmo - mycc.nocc
    t1, t2, _ = tamps
    T = _t3_device(mycc, tamps)
    it = _iteration(mycc)
    scale = 1.0 / np.sqrt(mycc.size if hasattr(mycc, "size") else 1)
    nd = mod.resolve_nvir_diis(mycc, nvir)
    lower = _dev(mod.pack_unique_replicated_tamps(mycc, (t1, t2), scale=scale), dev)
    adiis_t3.last_delta_norm_sq = it.diis_update(lower, T, adiis_t3.space, key=adiis_t3, nvir_diis=nd)
    (t1n, t2n), _ = mod.unpack_unique_replicated_tamps(mycc, _host(lower), (t1, t2), scale=scale)
    tamps[0], tamps[1] = t1n, t2n
    if not return_update_norm:
        return tamps
    update_norm = mod._max_t_diis_update_norm(mycc, res_norm, normt, adiis_t3, nd, nvir,
                                              '_last_t3_residual_norm_sq', '_last_t3_active_residual_norm_sq')
    return tamps, update_norm


def q_kernel(mycc, eris=None, tamps=None, blksize=4, comm=None, job_idx=0, n_jobs=1, log_redistribution=False):
    """(e_q_bracket, e_q_paren) of distr_cc/rccsdt_q.py:227 on the GPU, one rank: every task,
    or with n_jobs > 1 the tasks of job `job_idx` (the reference's contiguous slice of its task
    order, distr_cc/rccsdt_q.py:359-366), whose energies add up over the jobs."""
    from . import rccsdt_q
    if comm is None:
        # the reference falls back to mycc.comm, then MPI.COMM_WORLD (distr_cc/rccsdt_q.py:233-234)
        comm = getattr(mycc, "comm", None)
        if comm is None:
            try:
                from mpi4py import MPI
                comm = MPI.COMM_WORLD
            except ImportError:
                comm = None
    if comm is not None and int(comm.Get_size()) != 1:
        raise RuntimeError('einsum backend "cuda" runs on one rank; got a communicator of size %d'
                           % int(comm.Get_size()))
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
    out = _host(r4)
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
    r2[...] = _host(r)
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
    r3[...] = _host(r)
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


_MOD_ROUTES = {"update_amps_rccsdt_tri_": update_amps_rccsdt_tri_, "run_diis_t3": run_diis_t3}
# RCCSDT class attributes bound to those functions at class creation (distr_cc/rccsdt.py:1266, 1271)
_CLASS_ROUTES = {"update_amps_": "update_amps_rccsdt_tri_", "run_diis_t3": "run_diis_t3"}


def _wrap(name, orig, fn):
    def wrapper(mycc, *args, **kw):
        return fn(mycc, *args, **kw) if uses_cuda(mycc) else orig(mycc, *args, **kw)
    wrapper._dcc_wrapped = True
    wrapper.__name__ = name
    wrapper.__doc__ = orig.__doc__
    return wrapper


def install(rccsdt_module, rccsdt_q_module=None, rccsdtq_module=None, host_einsum_modules=()):
    """Route the reference's hot functions to the GPU when mycc.einsum_backend == "cuda".
    Every given module's `_einsum` (the reference modules bind PySCF's at import,
    distr_cc/rccsdt.py:27; pass pyscf.cc.rccsdt in host_einsum_modules for PySCF's own
    lower-order code) reads "cuda" as the host backend.  update_amps_rccsdt_tri_ and
    run_diis_t3 are routed both as module functions and as the RCCSDT class attributes the
    reference's kernel calls (mycc.update_amps_, mycc.run_diis_t3); the routed versions take
    the module's own lower-order functions, so PySCF's code keeps running on the host.
    Idempotent; returns the names it wrapped."""
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
        setattr(rccsdt_module, name, _wrap(name, orig, fn))
        wrapped.append(name)
    for name, fn in _MOD_ROUTES.items():
        orig = getattr(rccsdt_module, name, None)
        if orig is None or getattr(orig, "_dcc_wrapped", False):
            continue

        def bound(mycc, *args, _fn=fn, **kw):
            return _fn(mycc, *args, mod=rccsdt_module, **kw)
        setattr(rccsdt_module, name, _wrap(name, orig, bound))
        wrapped.append(name)
    cls = getattr(rccsdt_module, "RCCSDT", None)
    if cls is not None:
        for attr, fname in _CLASS_ROUTES.items():
            orig = cls.__dict__.get(attr)
            if orig is None or getattr(orig, "_dcc_wrapped", False):
                continue
            setattr(cls, attr, getattr(rccsdt_module, fname))
            wrapped.append("RCCSDT." + attr)
    if rccsdt_q_module is not None:
        orig = getattr(rccsdt_q_module, "kernel", None)
        if orig is not None and not getattr(orig, "_dcc_wrapped", False):
            rccsdt_q_module.kernel = _wrap("kernel", orig, q_kernel)
            wrapped.append("rccsdt_q.kernel")
    if rccsdtq_module is not None:
        for name, fn in _R4_ROUTES.items():
            fn = compute_r4_tri if fn is None else fn
            orig = getattr(rccsdtq_module, name, None)
            if orig is None or getattr(orig, "_dcc_wrapped", False):
                continue
            setattr(rccsdtq_module, name, _wrap(name, orig, fn))
            wrapped.append("rccsdtq." + name)
    return wrapped
