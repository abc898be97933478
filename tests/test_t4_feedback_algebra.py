"""The full-space T4 -> r2 / r3 feedback strings (dcc.t4_residual.r2_add_t4_ / r3_add_t4_)
against the oracle's literal per-block restatement of r2_add_t4_tri_ / r3_add_t4_tri_
(distr_cc/rccsdtq.py:471-683), on the CPU with the oracle's P4 symmetrizers: every
case weight of the reference (1, 1/2, 1/4) and every ordering."""
import numpy as np
import pytest
import torch

from dcc import t4_residual as tr
from oracle import t4_ref


def _inputs(no, nv, seed):
    rng = np.random.default_rng(seed)
    nmo = no + nv
    quads = t4_ref.stored_quadruples(no)
    return (rng.standard_normal((len(quads),) + (nv,) * 4) * 0.01, rng.standard_normal((nmo,) * 4) * 0.1,
            rng.standard_normal((nmo, nmo)) * 0.1, rng.standard_normal((no, no, nv, nv)),
            rng.standard_normal((no,) * 3 + (nv,) * 3))


def _spin(oracle, nv):
    def f(A, pattern):
        a = A.numpy()
        oracle.t4_spin_sum(a, a.size // nv ** 4, nv, pattern, 1.0, 0.0)
        return A
    return f


@pytest.mark.parametrize("no,nv", [(4, 3), (5, 2), (6, 3)])
def test_r2_add_t4(oracle, no, nv):
    t4, eris, fock, r2, _ = _inputs(no, nv, no + 10 * nv)
    want = t4_ref.r2_add_t4_tri_ref(r2, t4, eris, no, oracle)
    got = tr.r2_add_t4_(torch.from_numpy(r2.copy()), torch.from_numpy(t4), torch.from_numpy(eris), no,
                        spin4=_spin(oracle, nv))
    np.testing.assert_allclose(got.numpy(), want, rtol=1e-12, atol=1e-14 * np.abs(want).max())


@pytest.mark.parametrize("no,nv", [(4, 3), (5, 2), (6, 3)])
def test_r3_add_t4(oracle, no, nv):
    t4, eris, fock, _, r3 = _inputs(no, nv, 3 * no + nv)
    want = t4_ref.r3_add_t4_tri_ref(r3, t4, fock, eris, no, oracle)
    got = tr.r3_add_t4_(torch.from_numpy(r3.copy()), torch.from_numpy(t4), torch.from_numpy(fock),
                        torch.from_numpy(eris), no, spin4=_spin(oracle, nv))
    np.testing.assert_allclose(got.numpy(), want, rtol=1e-12, atol=1e-14 * np.abs(want).max())
