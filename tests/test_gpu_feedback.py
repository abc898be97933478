"""T3 -> r1, r2, W_vooo, W_vvvo feedback on the GPU against the oracle's
literal per-block restatement (distr_cc/rccsdt.py:253-366).  FP64: 1e-11
relative to the largest entry."""
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import t3_feedback
    from oracle import feedback_ref
    return t3_feedback, feedback_ref


def _inputs(no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    g = rng.standard_normal((nmo,) * 4) * 0.1
    fock = rng.standard_normal((nmo, nmo)) * 0.1
    full = rng.standard_normal((no,) * 3 + (nv,) * 3)
    U = sum(full.transpose(p + tuple(3 + x for x in p)) for p in itertools.permutations(range(3))) / 6
    t3 = np.stack([U[i, j, k] for i in range(no) for j in range(i, no) for k in range(j, no)])
    ijk = np.array([(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)], dtype=np.int32)
    return g, fock, t3, ijk, rng


@pytest.mark.parametrize("no,nv", [(3, 5), (4, 10)])
def test_r1_r2(mods, oracle, no, nv):
    fb, ref = mods
    g, fock, t3, ijk, rng = _inputs(no, nv, nv)
    r1, r2 = rng.standard_normal((no, nv)), rng.standard_normal((no, no, nv, nv))
    w1, w2 = ref.r1r2_add_t3_ref(fock, g, r1, r2, t3, no, oracle)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    d1, d2, dg, dt3 = dev(r1), dev(r2), dev(g), dev(t3)
    fb.r1_add_t3_(d1, dg, dt3, dev(ijk), no)
    X = fb.p3_201_all(dt3, no)
    fb.r2_add_t3_(d2, dev(fock), dg, X, no)
    np.testing.assert_allclose(d1.cpu().numpy(), w1, rtol=0, atol=1e-11 * np.abs(w1).max())
    np.testing.assert_allclose(d2.cpu().numpy(), w2, rtol=0, atol=1e-11 * np.abs(w2).max())


@pytest.mark.parametrize("no,nv", [(3, 5), (4, 10)])
def test_intermediates(mods, oracle, no, nv):
    fb, ref = mods
    g, fock, t3, ijk, rng = _inputs(no, nv, 3 + nv)
    Wo, Wv = rng.standard_normal((nv, no, no, no)), rng.standard_normal((nv, nv, nv, no))
    w1, w2 = ref.intermediates_t3_add_ref(g, Wo, Wv, t3, no, oracle)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    dWo, dWv, dt3 = dev(Wo), dev(Wv), dev(t3)
    X = fb.p3_201_all(dt3, no)
    fb.intermediates_t3_add_(dWo, dWv, dev(g), X, no)
    np.testing.assert_allclose(dWo.cpu().numpy(), w1, rtol=0, atol=1e-11 * np.abs(w1).max())
    np.testing.assert_allclose(dWv.cpu().numpy(), w2, rtol=0, atol=1e-11 * np.abs(w2).max())
