"""Hand-written adjoint of the T3 residual (dcc.adjoint) on the GPU:
  * forward equals the torch.einsum reference (tests/adjoint_ref.py);
  * every gradient equals autograd through that FP64 reference (t3 gradients
    projected onto stabilizer-symmetric blocks; pair-symmetric W_oooo);
  * central finite differences (h = 1e-5) of <lam, r3> along 64 random
    directions in all inputs at once equal <grad, direction>;
  * the split-precision backward agrees with FP64 to the split accuracy.
nocc=6, nvir=40 (the adjoint-check size, seeded synthetic inputs) and a small case."""
import itertools

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from adjoint_ref import r3_torch  # noqa: E402


@pytest.fixture(scope="module")
def adj():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import adjoint
    return adjoint


def _inputs(no, nv, seed):
    from dcc import synthetic
    d = synthetic.make_inputs(no, nv, seed=seed)
    W = d.W_oooo
    d.W_oooo = 0.5 * (W + W.permute(1, 0, 3, 2))
    return [d.t2, d.t3, d.F_vv, d.F_oo, d.W_vvvo, d.W_vooo, d.W_vvvv, d.W_ovov, d.W_ovvo, d.W_oooo], d


def _sym_dir(x, i, d, adjoint, g):
    v = torch.randn(x.shape, dtype=torch.float64, device="cuda", generator=g)
    if i == 1:
        v = adjoint.stab_project(v, d.ijk)
    if i == 9:
        v = 0.5 * (v + v.permute(1, 0, 3, 2))
    return v


@pytest.mark.parametrize("no,nv", [(3, 6), (6, 40)])
def test_adjoint_vs_autograd_and_fd(adj, no, nv):
    xs, d = _inputs(no, nv, seed=no + nv)
    g = torch.Generator(device="cuda").manual_seed(1)
    lam = torch.randn(d.t3.shape, dtype=torch.float64, device="cuda", generator=g)
    # forward
    r = adj.t3_residual_fn(*xs, "fp64")
    ref = r3_torch(*xs)
    assert float((r - ref).abs().max()) <= 1e-11 * float(ref.abs().max())
    # hand-written backward vs autograd through the FP64 einsum reference
    xa = [x.clone().requires_grad_(True) for x in xs]
    (lam * adj.t3_residual_fn(*xa, "fp64")).sum().backward()
    xr = [x.clone().requires_grad_(True) for x in xs]
    (lam * r3_torch(*xr)).sum().backward()
    for i, (a, b) in enumerate(zip(xa, xr)):
        want = b.grad
        if i == 1:
            want = adj.stab_project(want, d.ijk)
        scale = float(want.abs().max())
        assert float((a.grad - want).abs().max()) <= 1e-10 * scale, i
    # central finite differences along 64 random directions (all inputs at once)
    h = 1e-5
    f = lambda ys: float((lam * adj.t3_residual_fn(*ys, "fp64")).sum())  # noqa: E731
    for _ in range(64 if no == 6 else 16):
        vs = [_sym_dir(x, i, d, adj, g) for i, x in enumerate(xs)]
        fd = (f([x + h * v for x, v in zip(xs, vs)]) - f([x - h * v for x, v in zip(xs, vs)])) / (2 * h)
        an = sum(float((a.grad * v).sum()) for a, v in zip(xa, vs))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-8), (fd, an)


def test_split_backward(adj):
    xs, d = _inputs(4, 40, seed=9)
    g = torch.Generator(device="cuda").manual_seed(2)
    lam = torch.randn(d.t3.shape, dtype=torch.float64, device="cuda", generator=g)
    grads = {}
    for prec in ("fp64", "bf16x3"):
        xa = [x.clone().requires_grad_(True) for x in xs]
        (lam * adj.t3_residual_fn(*xa, prec)).sum().backward()
        grads[prec] = [x.grad for x in xa]
    for a, b in zip(grads["bf16x3"], grads["fp64"]):
        assert float((a - b).abs().max()) <= 1e-4 * float(b.abs().max())
