"""Hand-written adjoint of the (Q) energies (dcc.q_adjoint) on the GPU:
  * the forward equals the torch restatement of the task loop
    (tests/q_adjoint_ref.py), relative 1e-11;
  * every gradient (t2, t3, the seven integral slices) equals autograd through
    that FP64 torch reference (t3 gradients projected onto stabilizer-symmetric
    blocks), relative 1e-10 of the largest entry, at nocc=3 / nvir=7;
  * central finite differences (h = 1e-5) of g_b [Q] + g_p (Q) along 64 random
    directions in all inputs at once equal <grad, direction> to 1e-6 relative,
    at nocc=6 / nvir=40 (the adjoint-check size, seeded synthetic inputs)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from q_adjoint_ref import q_energy_torch  # noqa: E402
from test_q_oracle import _inputs  # noqa: E402

NAMES = ("vvvo", "vooo", "vvoo", "ovvo", "ovov", "vvvv", "oooo")


@pytest.fixture(scope="module")
def qa():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dcc import q_adjoint
    return q_adjoint


def _canonical(T, no):
    ijk = [(i, j, k) for i in range(no) for j in range(i, no) for k in range(j, no)]
    return np.stack([T[:, :, :, i, j, k] for i, j, k in ijk])


def _args(er, t2, t3, eo, ev):
    return [t2, t3] + [er[k] for k in NAMES] + [eo, ev]


def test_q_adjoint_vs_autograd(qa):
    from dcc.adjoint import stab_project
    from dcc.synthetic import canonical_ijk
    no, nv, blk = 3, 7, 3
    er, t2, T, eo, ev = _inputs(no, nv, 23)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    xs = _args({k: dev(v) for k, v in er.items()}, dev(t2), dev(_canonical(T, no)), dev(eo), dev(ev))
    gvec = torch.tensor([0.7, -1.3], dtype=torch.float64, device="cuda")
    xa = [x.clone().requires_grad_(i < 9) for i, x in enumerate(xs)]
    out = qa.q_energy_fn(*xa, blksize=blk)
    (gvec * out).sum().backward()
    xr = [x.clone().requires_grad_(i < 9) for i, x in enumerate(xs)]
    ref = q_energy_torch(dict(zip(NAMES, xr[2:9])), xr[0], xr[1], xr[9], xr[10], blk)
    o, rf = out.detach(), [float(ref[0].detach()), float(ref[1].detach())]
    assert abs(float(o[0]) - rf[0]) <= 1e-11 * abs(rf[0])
    assert abs(float(o[1]) - rf[1]) <= 1e-11 * abs(rf[1])
    (gvec[0] * ref[0] + gvec[1] * ref[1]).backward()
    ijk = torch.tensor(canonical_ijk(no), dtype=torch.int32, device="cuda")
    for i in range(9):
        want = xr[i].grad
        if i == 1:
            want = stab_project(want, ijk)
        scale = float(want.abs().max())
        assert scale > 0
        assert float((xa[i].grad - want).abs().max()) <= 1e-10 * scale, i


def test_q_adjoint_finite_differences(qa):
    from dcc import synthetic
    from dcc.adjoint import stab_project
    no, nv, blk = 6, 40, 10
    d = synthetic.make_inputs(no, nv, seed=31)
    er = {"vvvo": d.W_vvvo, "vooo": d.W_vooo, "vvoo": d.eris_vvoo, "ovvo": d.W_ovvo, "ovov": d.W_ovov,
          "vvvv": d.W_vvvv, "oooo": d.W_oooo}
    xs = _args(er, d.t2.permute(2, 3, 0, 1).contiguous(), d.t3, d.e_occ, d.e_vir)
    gvec = torch.tensor([0.4, 1.1], dtype=torch.float64, device="cuda")
    xa = [x.clone().requires_grad_(i < 9) for i, x in enumerate(xs)]
    (gvec * qa.q_energy_fn(*xa, blksize=blk)).sum().backward()
    g = torch.Generator(device="cuda").manual_seed(3)

    def f(ys):
        return float((gvec * qa.q_energy_fn(*ys, blksize=blk)).sum())

    h = 1e-5
    for _ in range(64):
        vs = []
        for i, x in enumerate(xs):
            if i >= 9:
                vs.append(torch.zeros_like(x))
                continue
            v = torch.randn(x.shape, dtype=torch.float64, device="cuda", generator=g) * float(x.abs().max())
            vs.append(stab_project(v, d.ijk) if i == 1 else v)
        fd = (f([x + h * v for x, v in zip(xs, vs)]) - f([x - h * v for x, v in zip(xs, vs)])) / (2 * h)
        an = sum(float((a.grad * v).sum()) for a, v in zip(xa[:9], vs[:9]))
        assert abs(fd - an) <= 1e-6 * max(abs(an), 1e-8), (fd, an)
