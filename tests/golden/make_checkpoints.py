"""Generate tests/golden/checkpoints/ with the reference's own checkpoint writers.

DistributedT3IJK.save_to_disk (distr_cc/distribute_t3.py:959-996) and
DistributedT4IJKL.save_to_disk (distr_cc/distribute_t4.py:903-925) are run for every
rank of a few small distributions, so the committed files are exactly what a
multi-rank reference run leaves on disk.  The reference modules import mpi4py and
pyscf.lib.logger at module level; neither is installed here, so this script puts
minimal stand-ins for both in sys.modules (a communicator with a fixed rank and
size, a no-op logger).  Run from the repository root, in a container that holds the
reference sources:

    python tests/golden/make_checkpoints.py <path-to-reference>   (or set DCC_REFERENCE)

Each case directory holds the checkpoint files and `blocks.npy`, the full
canonical-order amplitudes the ranks' files were cut from.
"""
import json
import os
import shutil
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "checkpoints")


class _Comm:
    """One rank of a communicator of `size` ranks.  The ranks are built one after the other,
    rank 0 first, so a broadcast hands every later rank what rank 0 sent last."""
    _sent = {}

    def __init__(self, rank, size):
        self._rank, self._size = rank, size

    def Get_rank(self):
        return self._rank

    def Get_size(self):
        return self._size

    def bcast(self, obj, root=0):
        if self._rank == root:
            _Comm._sent[root] = obj
            return obj
        return _Comm._sent[root]

    def Barrier(self):
        pass


def _install_stubs():
    mpi4py = types.ModuleType("mpi4py")
    mpi = types.ModuleType("mpi4py.MPI")
    mpi.COMM_WORLD = _Comm(0, 1)
    mpi.SUM, mpi.MAX, mpi.IN_PLACE = "sum", "max", None
    mpi4py.MPI = mpi
    pyscf = types.ModuleType("pyscf")
    lib = types.ModuleType("pyscf.lib")
    logger = types.ModuleType("pyscf.lib.logger")
    for name in ("info", "debug", "debug1", "note", "warn", "timer", "timer_debug1"):
        setattr(logger, name, lambda *a, **k: None)
    lib.logger = logger
    pyscf.lib = lib
    cc = types.ModuleType("pyscf.cc")
    rccsdt = types.ModuleType("pyscf.cc.rccsdt")
    rccsdt.format_size = lambda n: str(n)
    cc.rccsdt = rccsdt
    pyscf.cc = cc
    for name, mod in (("mpi4py", mpi4py), ("mpi4py.MPI", mpi), ("pyscf", pyscf), ("pyscf.lib", lib),
                      ("pyscf.lib.logger", logger), ("pyscf.cc", cc), ("pyscf.cc.rccsdt", rccsdt)):
        sys.modules.setdefault(name, mod)


def _t3_case(mod, name, nocc, nvir, size, distribution, batch_size, rng):
    d = os.path.join(OUT, name)
    os.makedirs(d)
    n3 = nocc * (nocc + 1) * (nocc + 2) // 6
    blocks = rng.standard_normal((n3, nvir, nvir, nvir))
    np.save(os.path.join(d, "blocks.npy"), blocks)
    for rank in range(size):
        dist = mod.DistributedT3IJK(nocc, nvir, _Comm(rank, size), distribution=distribution,
                                    batch_size=batch_size)
        idx = [mod.ijk_to_linear(i, j, k, nocc) for (i, j, k) in dist.local_triples]
        dist.save_to_disk(np.ascontiguousarray(blocks[idx]), os.path.join(d, "ckpt_"))


def _t4_case(mod, name, nocc, nvir, size, distribution, rng):
    d = os.path.join(OUT, name)
    os.makedirs(d)
    stored = mod.enumerate_stored_ijkl_quadruples(nocc)
    blocks = rng.standard_normal((len(stored), nvir, nvir, nvir, nvir))
    np.save(os.path.join(d, "blocks.npy"), blocks)
    pos = {q: n for n, q in enumerate(stored)}
    for rank in range(size):
        dist = mod.DistributedT4IJKL(nocc, nvir, _Comm(rank, size), distribution=distribution)
        idx = [pos[tuple(int(x) for x in q)] for q in dist.local_quadruples]
        dist.save_to_disk(np.ascontiguousarray(blocks[idx]), os.path.join(d, "ckpt_"))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DCC_REFERENCE")
    if not ref:
        sys.exit("usage: make_checkpoints.py <path-to-reference>  (or set DCC_REFERENCE)")
    _install_stubs()
    # The writers use no C helper; the reference refuses to import without its library
    # unless the Python fallback is allowed.
    os.environ["DISTR_CC_ALLOW_PYTHON_FALLBACK"] = "1"
    sys.path.insert(0, ref)
    import distr_cc.distribute_t3 as t3mod
    import distr_cc.distribute_t4 as t4mod
    if os.path.isdir(OUT):
        shutil.rmtree(OUT)
    rng = np.random.default_rng(20261203)
    _t3_case(t3mod, "t3_n1", 3, 4, 1, "balanced", None, rng)
    _t3_case(t3mod, "t3_n3_round_robin", 4, 3, 3, "round_robin", None, rng)
    _t3_case(t3mod, "t3_n2_block", 4, 3, 2, "block", None, rng)
    _t3_case(t3mod, "t3_n2_balanced_b4", 4, 3, 2, "balanced", 4, rng)
    _t4_case(t4mod, "t4_n1", 4, 3, 1, "balanced", rng)
    _t4_case(t4mod, "t4_n2_round_robin", 4, 3, 2, "round_robin", rng)
    for case in sorted(os.listdir(OUT)):
        with open(os.path.join(OUT, case, "ckpt_metadata.json")) as f:
            print(case, json.load(f))


if __name__ == "__main__":
    main()
