"""Stand-ins that let the reference's own Python drivers run in one process
without MPI or PySCF, and the lower-order replay that feeds them.

Test infrastructure only.  Two users:

* tests/golden/make_ref_fixtures.py imports the reference modules
  (distr_cc/rccsdt.py, rccsdt_q.py, rccsdtq.py, diis.py) with these modules
  placed in sys.modules and runs their hot functions to write the fixtures;
* the GPU route tests install this library's drop-in routes into a
  namespace that carries the same lower-order replay, so both sides see the
  same intermediates.

What stands in for what:

  mpi4py.MPI          a communicator of one rank (Allreduce / Alltoall(v) copy
                      the send buffer, bcast / allreduce return their argument)
  pyscf.lib.logger    silent loggers with the reference's timer signatures
  pyscf.cc.rccsdt     _einsum(backend, subscripts, *ops, out, alpha, beta):
                      out = alpha * einsum + beta * out (out may be a view);
                      t3_spin_summation_inplace_: the reference's own per-block
                      t3_single_spin_summation_inplace_ (compiled from the
                      reference C sources) applied to every block
  pyscf.cc.rccsdt_highm.t3_spin_summation   the same, out of place
  pyscf lib t4_add_   t4 += r4 elementwise
  lower-order PySCF   update_t1_fock_eris / intermediates_t1t2 / compute_r1r2 /
                      intermediates_t3 replay stored arrays (LowerOrderReplay);
                      r1r2_divide_e_ divides by the orbital-energy
                      denominators; the unique T1/T2 map keeps every t1 element
                      and the i <= j pairs of t2 (restore_t_ fills t2[j, i] =
                      t2[i, j].T), which is what RHF amplitudes with
                      t2[ijab] = t2[jiba] need.

None of these is on the product path.
"""
from __future__ import annotations

import ctypes
import sys
import time
import types

import numpy as np


# --------------------------------------------------------------------------- MPI

class _Op:
    def __init__(self, name):
        self.name = name


class _Datatype:
    def Create_contiguous(self, n):
        return _Datatype()

    def Commit(self):
        return self

    def Free(self):
        return None


class OneRankComm:
    """The communicator calls the reference makes, for one rank."""

    rank, size = 0, 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def bcast(self, obj, root=0):
        return obj

    def Barrier(self):
        return None

    def allreduce(self, obj, op=None):
        return obj

    @staticmethod
    def _buf(spec):
        return spec[0] if isinstance(spec, (list, tuple)) else spec

    def Allreduce(self, sendbuf, recvbuf=None, op=None):
        if sendbuf is _IN_PLACE or recvbuf is None:
            return None
        np.copyto(np.asarray(self._buf(recvbuf)), np.asarray(self._buf(sendbuf)))
        return None

    def Alltoall(self, sendbuf, recvbuf):
        np.copyto(np.asarray(self._buf(recvbuf)), np.asarray(self._buf(sendbuf)))

    def Alltoallv(self, sendspec, recvspec):
        s, r = np.asarray(sendspec[0]).reshape(-1), np.asarray(recvspec[0]).reshape(-1)
        r[:s.size] = s

    def Allgather(self, sendbuf, recvbuf):
        np.copyto(np.asarray(self._buf(recvbuf)).reshape(-1), np.asarray(self._buf(sendbuf)).reshape(-1))

    def allgather(self, obj):
        return [obj]

    def gather(self, obj, root=0):
        return [obj]


_IN_PLACE = object()


def _mpi_module():
    mpi4py = types.ModuleType("mpi4py")
    mpi = types.ModuleType("mpi4py.MPI")
    mpi.COMM_WORLD = OneRankComm()
    mpi.Comm = OneRankComm
    mpi.SUM, mpi.MAX, mpi.MIN = _Op("sum"), _Op("max"), _Op("min")
    mpi.IN_PLACE = _IN_PLACE
    mpi.DOUBLE = _Datatype()
    mpi.INT64_T = _Datatype()
    mpi.THREAD_SINGLE, mpi.THREAD_FUNNELED, mpi.THREAD_SERIALIZED, mpi.THREAD_MULTIPLE = 0, 1, 2, 3
    mpi.Query_thread = lambda: 3
    mpi.Wtime = time.perf_counter

    class Request:
        @staticmethod
        def Waitall(reqs):
            return None

        @staticmethod
        def Testany(reqs):
            return None
    mpi.Request = Request
    mpi4py.MPI = mpi
    return mpi4py, mpi


# --------------------------------------------------------------------------- PySCF

class _Logger:
    def __init__(self, stdout=None, verbose=0):
        self.stdout, self.verbose = stdout, verbose

    def _t(self, *a, **k):
        return (time.process_time(), time.perf_counter())

    timer = timer_debug1 = _t

    def _n(self, *a, **k):
        return None

    info = debug = debug1 = debug2 = note = warn = error = _n


def einsum_standin(backend, subscripts, *operands, out=None, alpha=1.0, beta=0.0):
    """pyscf.cc.rccsdt._einsum as the reference uses it: out = alpha*einsum + beta*out."""
    res = np.einsum(subscripts, *operands, optimize=True)
    if out is None:
        return alpha * res if alpha != 1.0 else res
    if beta == 0.0:
        out[...] = alpha * res
    else:
        out[...] = beta * out + alpha * res
    return out


class _RefC:
    """The reference's t3_single_spin_summation_inplace_ from the library the reference sources compile to."""

    def __init__(self, so_path):
        self.lib = ctypes.CDLL(so_path)
        f = self.lib.t3_single_spin_summation_inplace_
        f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_char_p, ctypes.c_double, ctypes.c_double]
        f.restype = None

    def p3(self, block, nvir, pattern, alpha, beta):
        assert block.dtype == np.float64 and block.flags["C_CONTIGUOUS"]
        self.lib.t3_single_spin_summation_inplace_(block.ctypes.data_as(ctypes.c_void_p), int(nvir),
                                                   pattern.encode(), float(alpha), float(beta))


def _pyscf_modules(refc):
    pyscf = types.ModuleType("pyscf")
    lib = types.ModuleType("pyscf.lib")
    logger = types.ModuleType("pyscf.lib.logger")
    logger.Logger = _Logger
    logger.new_logger = lambda *a, **k: _Logger()
    logger.process_clock, logger.perf_counter = time.process_time, time.perf_counter
    logger.QUIET, logger.ERROR, logger.WARN, logger.NOTE, logger.INFO = 0, 1, 2, 3, 4
    logger.DEBUG, logger.DEBUG1, logger.DEBUG2 = 5, 6, 7
    for name in ("info", "debug", "debug1", "debug2", "note", "warn", "error"):
        setattr(logger, name, lambda *a, **k: None)
    logger.timer = logger.timer_debug1 = lambda *a, **k: (time.process_time(), time.perf_counter())
    lib.logger = logger
    lib.current_memory = lambda: (0.0, 0.0)
    lib.num_threads = lambda *a: 1

    def prange(start, stop, step):
        for p0 in range(start, stop, step):
            yield p0, min(p0 + step, stop)
    lib.prange = prange

    class _CcsdtLib:
        @staticmethod
        def t4_add_(t4p, r4p, nocc4, nvir):
            n = int(nocc4.value) * int(nvir.value) ** 4
            t4 = np.ctypeslib.as_array(ctypes.cast(t4p, ctypes.POINTER(ctypes.c_double)), shape=(n,))
            r4 = np.ctypeslib.as_array(ctypes.cast(r4p, ctypes.POINTER(ctypes.c_double)), shape=(n,))
            t4 += r4
    lib.load_library = lambda name: _CcsdtLib()
    diis = types.ModuleType("pyscf.lib.diis")

    class DIIS:
        pass
    diis.DIIS = DIIS
    lib.diis = diis
    pyscf.lib = lib
    config = types.ModuleType("pyscf.__config__")
    pyscf.__config__ = config

    cc = types.ModuleType("pyscf.cc")
    rccsdt = types.ModuleType("pyscf.cc.rccsdt")
    rccsdt._einsum = einsum_standin
    rccsdt.format_size = lambda n: "%d B" % int(n)

    def t3_spin_summation_inplace_(A, nblocks, nvir, pattern, alpha=1.0, beta=0.0):
        flat = A.reshape(-1, nvir, nvir, nvir)
        for b in range(int(nblocks)):
            blk = np.ascontiguousarray(flat[b])
            refc.p3(blk, nvir, pattern, alpha, beta)
            flat[b] = blk
        return A
    rccsdt.t3_spin_summation_inplace_ = t3_spin_summation_inplace_

    class _IMDS:
        def __init__(self):
            for name in ("t1_fock", "t1_eris", "F_oo", "F_vv", "W_oooo", "W_ovvo", "W_ovov", "W_vooo", "W_vvvo",
                         "W_vvvv"):
                setattr(self, name, None)
    rccsdt._IMDS = _IMDS

    class _PhysicistsERIs:
        pass
    rccsdt._PhysicistsERIs = _PhysicistsERIs
    for name in ("update_t1_fock_eris", "energy_rhf", "intermediates_t1t2", "compute_r1r2", "r1r2_divide_e_",
                 "intermediates_t3", "amplitudes_to_vector_rhf", "vector_to_amplitudes_rhf", "_ao2mo_rcc",
                 "dump_flags", "_finalize"):
        setattr(rccsdt, name, _unavailable(name))
    rccsdt.build_unique_tamps_map_rhf = build_unique_tamps_map
    rccsdt.restore_t_ = restore_t_
    cc.rccsdt = rccsdt

    highm = types.ModuleType("pyscf.cc.rccsdt_highm")

    def t3_spin_summation(A, B, nblocks, nvir, pattern, alpha=1.0, beta=0.0):
        fa, fb = A.reshape(-1, nvir, nvir, nvir), B.reshape(-1, nvir, nvir, nvir)
        for b in range(int(nblocks)):
            blk = np.array(fa[b], copy=True)  # out of place: A stays as it is
            refc.p3(blk, nvir, pattern, alpha, 0.0)
            fb[b] = blk + beta * fb[b] if beta != 0.0 else blk
        return B
    highm.t3_spin_summation = t3_spin_summation
    for name in ("t3_perm_symmetrize_inplace_", "purify_tamps_", "r1r2_add_t3_", "intermediates_t3_add_t3",
                 "compute_r3", "r3_divide_e_"):
        setattr(highm, name, _unavailable(name))
    cc.rccsdt_highm = highm

    ccsd = types.ModuleType("pyscf.cc.ccsd")

    class CCSDBase:
        pass
    ccsd.CCSDBase = CCSDBase
    cc.ccsd = ccsd
    pyscf.cc = cc
    mp = types.ModuleType("pyscf.mp")
    mp2 = types.ModuleType("pyscf.mp.mp2")
    for name in ("get_nocc", "get_nmo", "get_frozen_mask", "get_e_hf"):
        setattr(mp2, name, _unavailable(name))
    mp.mp2 = mp2
    pyscf.mp = mp
    return {"pyscf": pyscf, "pyscf.lib": lib, "pyscf.lib.logger": logger, "pyscf.lib.diis": diis,
            "pyscf.__config__": config, "pyscf.cc": cc, "pyscf.cc.rccsdt": rccsdt,
            "pyscf.cc.rccsdt_highm": highm, "pyscf.cc.ccsd": ccsd, "pyscf.mp": mp, "pyscf.mp.mp2": mp2}


def _unavailable(name):
    def f(*a, **k):
        raise RuntimeError("%s is PySCF code that is not available here; replay it instead" % name)
    f.__name__ = name
    return f


def install(ref_so_path):
    """Put the MPI and PySCF stand-ins into sys.modules (replacing nothing that exists)."""
    refc = _RefC(ref_so_path)
    mpi4py, mpi = _mpi_module()
    mods = {"mpi4py": mpi4py, "mpi4py.MPI": mpi}
    mods.update(_pyscf_modules(refc))
    for name, mod in mods.items():
        sys.modules.setdefault(name, mod)
    return refc


# ------------------------------------------------------- unique T1/T2 map (RHF)

def build_unique_tamps_map(mycc=None, nocc=None):
    """[t1 map, t2 map]: index tuples over the occupied indices (every i; pairs i <= j)."""
    nocc = mycc.nocc if nocc is None else nocc
    i1 = (np.arange(nocc),)
    iu, ju = np.triu_indices(nocc)
    return [[i1], [(iu, ju)]]


def restore_t_(t, nocc, order=1, do_tri=False, unique_tamps_map=None):
    """Fill the non-unique T2 pairs: t2[j, i] = t2[i, j].T for i < j."""
    if order == 2:
        for i in range(nocc):
            for j in range(i + 1, nocc):
                t[j, i] = t[i, j].T
    return t


# ------------------------------------------------------------ lower-order replay

class LowerOrderReplay:
    """The PySCF lower-order steps of update_amps_rccsdt_tri_ (distr_cc/rccsdt.py:908-935)
    replayed from stored arrays: the dressed Fock / ERIs, r1 and r2 before their T3 part,
    and the T3 intermediates.  `bind(namespace)` sets the five functions on a module or a
    namespace the way the reference module imports them from pyscf.cc.rccsdt."""

    NAMES = ("update_t1_fock_eris", "intermediates_t1t2", "compute_r1r2", "r1r2_divide_e_", "intermediates_t3")
    T3_IMDS = ("F_vv", "F_oo", "W_vvvo", "W_vooo", "W_vvvv", "W_ovov", "W_ovvo", "W_oooo")

    def __init__(self, arrays, nocc, level_shift=0.0):
        self.a = {k: np.asarray(v) for k, v in arrays.items()}
        self.nocc, self.level_shift = nocc, level_shift

    def update_t1_fock_eris(self, mycc, imds, t1, eris):
        imds.t1_fock = self.a["t1_fock"].copy()
        imds.t1_eris = self.a["t1_eris"].copy()
        return imds

    def intermediates_t1t2(self, mycc, imds, t2):
        return imds

    def compute_r1r2(self, mycc, imds, t2):
        return self.a["r1_lower"].copy(), self.a["r2_lower"].copy()

    def r1r2_divide_e_(self, mycc, r1, r2, mo_energy):
        nocc = self.nocc
        eia = mo_energy[:nocc, None] - mo_energy[None, nocc:] - self.level_shift
        r1 /= eia
        r2 /= eia[:, None, :, None] + eia[None, :, None, :]
        return r1, r2

    def intermediates_t3(self, mycc, imds, t2):
        for name in self.T3_IMDS:
            setattr(imds, name, self.a[name].copy())
        return imds

    def bind(self, ns):
        for name in self.NAMES:
            setattr(ns, name, getattr(self, name))
        return ns


# -------------------------------- the unique-amplitude packing of distr_cc/_runtime.py

def pack_unique_replicated_tamps(mycc, tamps, scale=1.0):
    """distr_cc/_runtime.py:151-165 over the RHF unique map above."""
    umap = mycc.unique_tamps_map
    chunks = []
    for i, t in enumerate(tamps):
        idx = (*umap[i][0], *[slice(None)] * (i + 1))
        chunk = np.asarray(t[idx]).reshape(-1)
        chunks.append(chunk * scale if scale != 1.0 else chunk)
    return np.concatenate(chunks)


def unpack_unique_replicated_tamps(mycc, vector, template_tamps, scale=1.0):
    """distr_cc/_runtime.py:167-187 over the RHF unique map above."""
    umap = mycc.unique_tamps_map
    vector = np.asarray(vector).reshape(-1)
    out, offset = [], 0
    for i, template in enumerate(template_tamps):
        order = i + 1
        t = np.zeros_like(template)
        idx = (*umap[i][0], *[slice(None)] * order)
        shape = t[idx].shape
        size = int(np.prod(shape))
        block = vector[offset:offset + size].reshape(shape)
        t[idx] = block / scale if scale != 1.0 else block
        restore_t_(t, mycc.nocc, order=order)
        out.append(t)
        offset += size
    return out, offset


# ------------------------------------- the DIIS helpers of distr_cc/_runtime.py, rccsdt.py

def norm_sq_from_norms(norms):
    """distr_cc/_runtime.py:87-88."""
    return sum(float(n) * float(n) for n in norms)


def resolve_nvir_diis(mycc, nvir):
    """distr_cc/_runtime.py:121-128."""
    nd = getattr(mycc, "nvir_diis", None)
    return nvir if nd is None else min(int(nd), nvir)


def _safe_update_norm(norm_sq):
    return np.sqrt(max(float(norm_sq), 0.0))


def _max_t_diis_update_norm(mycc, res_norm, normt, adiis, nvir_diis, nvir, total_attr, active_attr):
    """distr_cc/rccsdt.py:990-999 (with _safe_update_norm, :979-980)."""
    delta = getattr(adiis, "last_delta_norm_sq", None)
    if delta is None:
        return float(normt) if res_norm is None else _safe_update_norm(norm_sq_from_norms(res_norm))
    delta = float(delta)
    if nvir_diis < nvir:
        total = float(getattr(mycc, total_attr, res_norm[-1] * res_norm[-1]))
        active = float(getattr(mycc, active_attr, total))
        delta += max(total - active, 0.0)
    return _safe_update_norm(delta)


class IMDS:
    """pyscf.cc.rccsdt._IMDS: a bag of intermediates."""


def route_module(replay):
    """A namespace carrying what the routed update_amps_rccsdt_tri_ / run_diis_t3 take from the
    reference module they are installed in: the lower-order replay, _IMDS and the DIIS
    helpers above."""
    ns = types.SimpleNamespace(_IMDS=IMDS, resolve_nvir_diis=resolve_nvir_diis,
                               pack_unique_replicated_tamps=pack_unique_replicated_tamps,
                               unpack_unique_replicated_tamps=unpack_unique_replicated_tamps,
                               _max_t_diis_update_norm=_max_t_diis_update_norm,
                               norm_sq_from_norms=norm_sq_from_norms)
    return replay.bind(ns)


class CanonicalT3Dist:
    """One rank holding every canonical block in canonical order (the reference's
    DistributedT3IJK at one rank)."""

    def __init__(self, nocc):
        self.local_triples = [(i, j, k) for i in range(nocc) for j in range(i, nocc) for k in range(j, nocc)]

    def iter_local_ijk(self):
        for q, (i, j, k) in enumerate(self.local_triples):
            yield i, j, k, q


class StoredT4Dist:
    """One rank holding the listed stored T4 blocks in that order."""

    def __init__(self, ijkl):
        self.local_quadruples = [tuple(int(x) for x in q) for q in ijkl]

    def iter_local_ijkl(self):
        for q, (i, j, k, l) in enumerate(self.local_quadruples):
            yield i, j, k, l, q
