"""The split-precision T3 feedback plan (dcc.t3_feedback.SplitFeedback) on the CPU:
every operand split (row / contraction maps, the permuted E slices, one piece per
value of the contracted occupied index) and every per-piece GEMM with its epilogue
map emulated in numpy FP64, against the FP64 feedback strings
(distr_cc/rccsdt.py:300-316, 340-358).  Relative 1e-12."""
import numpy as np
import pytest
import torch

from dcc import contract, t3_feedback as fb
from test_maps_emulated import fmap


class _EmuSplit:
    """contract.Split with the two pieces replaced by one FP64 array (same maps, same pieces)."""

    def __init__(self, M, K=None, kind=0, device="cpu", buffers=None, pieces=None, align=8):
        ref = contract.Split(M, K, kind, device="meta", pieces=pieces, align=align)
        self.M, self.K, self.Kp, self.pieces, self.kind = ref.M, ref.K, ref.Kp, ref.pieces, kind
        self.a = np.zeros((self.M, self.Kp))

    def fill_piece(self, i, src, fm, fk):
        off, k, _ = self.pieces[i]
        # read through the maps from src's first element, over its storage
        st = src.untyped_storage()
        n = st.nbytes() // 8 - src.storage_offset()
        buf = torch.empty(0, dtype=torch.float64).set_(st, src.storage_offset(), (n,), (1,)).numpy()
        idx = fmap(fm, np.arange(self.M))[:, None] + fmap(fk, np.arange(k))[None, :]
        self.a[:, off:off + k] = buf[idx]
        return self

    def fill(self, src, fm, fk):
        return self.fill_piece(0, src, fm, fk)


def _emu_gemm(A, B, C, frow, fcol, alpha=1.0, beta=1.0, status=None, Kp=None):
    idx = fmap(frow, np.arange(A.M))[:, None] + fmap(fcol, np.arange(B.M))[None, :]
    assert len(np.unique(idx)) == idx.size
    flat = C.view(-1).numpy()
    # beta = 0 overwrites without reading C (BLAS semantics, as the kernel's epilogue)
    flat[idx] = alpha * (A.a @ B.a.T) + (beta * flat[idx] if beta != 0.0 else 0.0)
    return status


def _emu_gemm_range(A, B, C, frow, fcol, alpha, beta, status, col0, ncol):
    assert col0 % 64 == 0 and ncol % 64 == 0
    idx = fmap(frow, np.arange(A.M))[:, None] + fmap(fcol, np.arange(B.M))[None, :]
    flat = C.view(-1).numpy()
    flat[idx] = alpha * (A.a[:, col0:col0 + ncol] @ B.a[:, col0:col0 + ncol].T) + \
        (beta * flat[idx] if beta != 0.0 else 0.0)
    return status


class _EmuContract:
    KIND, padded_k, lin, three, _KBLK = contract.KIND, staticmethod(contract.padded_k), \
        staticmethod(contract.lin), staticmethod(contract.three), contract._KBLK
    Split = _EmuSplit
    gemm_ = staticmethod(_emu_gemm)
    gemm_range_ = staticmethod(_emu_gemm_range)


@pytest.mark.parametrize("no,nv", [(3, 5), (4, 6), (5, 4)])
def test_split_feedback_maps(no, nv):
    rng = np.random.default_rng(no * nv)
    nmo = no + nv
    g = torch.from_numpy(rng.standard_normal((nmo,) * 4))
    X = torch.from_numpy(rng.standard_normal((no, no, no, nv, nv, nv)))
    sl = {k: v.contiguous() for k, v in fb.eris_slices(g, None, no).items()}
    sfb = fb.SplitFeedback(no, nv, "bf16x3", device="cpu")
    assert all(len(p[0]) == no for p in sfb.plans.values())  # one piece per x
    sfb.c = _EmuContract
    r2 = torch.zeros(no, no, nv, nv, dtype=torch.float64)
    Wo = torch.zeros(nv, no, no, no, dtype=torch.float64)
    Wv = torch.zeros(nv, nv, nv, no, dtype=torch.float64)
    sfb.run(X, sl, {"r2": r2, "W_vooo": Wo, "W_vvvo": Wv})
    e = torch.einsum
    o, v = slice(0, no), slice(no, None)
    want_r2 = e('cxad,xyzdba->yzbc', g[v, o, v, v], X) - e('zxla,xyzabc->ylbc', g[o, o, o, v], X)
    E = g[o, o, v, v]
    want_wo = e('mxde,xyzead->amyz', E, X)
    want_wv = -e('zxde,xyzeba->abdy', E, X)
    for got, want in ((r2, want_r2), (Wo, want_wo), (Wv, want_wv)):
        np.testing.assert_allclose(got.numpy(), want.numpy(), rtol=0, atol=1e-12 * want.abs().max().item())


@pytest.mark.parametrize("no,nv", [(3, 5), (4, 7), (5, 4)])
def test_r1_without_v_pass(oracle, no, nv):
    """r1's T3 part (distr_cc/rccsdt.py:262-296) from t3 directly: the permutations of V =
    P3_422(t3) moved onto the ERI slices, three batched GEMMs over t3 (no library call, so it
    runs here on CPU tensors), against the oracle's literal per-block loop.  1e-12 relative."""
    import itertools
    from oracle import feedback_ref
    rng = np.random.default_rng(no * 10 + nv)
    nmo = no + nv
    g = rng.standard_normal((nmo,) * 4) * 0.1
    fock = rng.standard_normal((nmo, nmo)) * 0.1
    full = rng.standard_normal((no,) * 3 + (nv,) * 3)
    U = sum(full.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3))) / 6
    t3 = np.stack([U[i, j, k] for i in range(no) for j in range(i, no) for k in range(j, no)])
    ijk = np.array([(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)], dtype=np.int32)
    r1, r2 = rng.standard_normal((no, nv)), rng.standard_normal((no, no, nv, nv))
    want, _ = feedback_ref.r1r2_add_t3_ref(fock, g, r1.copy(), r2.copy(), t3, no, oracle)
    got = torch.from_numpy(r1.copy())
    fb.r1_add_t3_(got, torch.from_numpy(g), torch.from_numpy(t3), torch.from_numpy(ijk), no)
    np.testing.assert_allclose(got.numpy(), want, rtol=0, atol=1e-12 * np.abs(want).max())
