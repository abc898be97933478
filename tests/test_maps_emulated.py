"""The address maps the residual drivers hand to dcc_split_operand and
dcc_gemm_split3, checked on the CPU: the split, the GEMM and the epilogue
scatter are emulated in numpy with the same three-digit map arithmetic the
kernels use, and compared with numpy einsums of the terms they implement."""
import numpy as np

from dcc import contract as c


def fmap(f, m):
    R1, R2, S0, S1, S2 = f
    m = np.asarray(m, dtype=np.int64)
    return (m // (R1 * R2)) * S0 + ((m // R2) % R1) * S1 + (m % R2) * S2


def split(src, M, K, fm, fk):
    return src.ravel()[fmap(fm, np.arange(M))[:, None] + fmap(fk, np.arange(K))[None, :]]


def gemm(A, B, C, fr, fc, alpha, beta):
    idx = fmap(fr, np.arange(A.shape[0]))[:, None] + fmap(fc, np.arange(B.shape[0]))[None, :]
    assert len(np.unique(idx)) == idx.size  # the epilogue map never writes an element twice
    flat = C.ravel()
    flat[idx] = alpha * (A @ B.T) + beta * flat[idx]


NO, NV = 3, 4
e = np.einsum


def test_oo_maps():
    no, nv = NO, NV
    rng = np.random.default_rng(1)
    Wov, Wvo = rng.standard_normal((no, nv, no, nv)), rng.standard_normal((no, nv, nv, no))
    U = rng.standard_normal((no, no, no, nv, nv, nv))
    G2 = (-0.5 * (Wov + Wvo.transpose(0, 1, 3, 2))).transpose(2, 1, 0, 3).copy()
    ref = (-e('lbid,jkldca->ijkabc', Wov, U) + e('iald,jkldcb->ijkabc', G2, U) + e('iald,jklbdc->ijkabc', G2, U)
           - e('lcid,jklbda->ijkabc', Wov, U) + e('ladi,jklbcd->ijkabc', Wvo, U))
    n3v = nv ** 3
    Z = np.zeros(no ** 3 * n3v)
    zr = lambda xs: c.two(nv, no * no * n3v, xs)  # noqa: E731
    zc = lambda ys, zs: c.three(nv, nv, n3v, ys, zs)  # noqa: E731
    ur = lambda ys, zs: c.three(nv, nv, no * n3v, ys, zs)  # noqa: E731
    wov = (c.two(nv, nv, no * nv), c.two(nv, nv * no * nv, 1))
    g2 = (c.lin(no * nv), c.lin(1))
    wvo = (c.two(nv, 1, nv * no), c.two(nv, nv * nv * no, no))
    K, M, N = no * nv, no * nv, no * no * nv * nv
    B0 = split(U, N, K, ur(nv, 1), c.two(nv, n3v, nv * nv))
    gemm(split(Wov, M, K, *wov), B0, Z, zr(nv), zc(1, nv * nv), -1.0, 0.0)
    gemm(split(G2, M, K, *g2), B0, Z, zr(nv * nv), zc(1, nv), 1.0, 1.0)
    B1 = split(U, N, K, ur(nv * nv, 1), c.two(nv, n3v, nv))
    gemm(split(G2, M, K, *g2), B1, Z, zr(nv * nv), zc(nv, 1), 1.0, 1.0)
    gemm(split(Wov, M, K, *wov), B1, Z, zr(1), zc(nv, nv * nv), -1.0, 1.0)
    B2 = split(U, N, K, ur(nv * nv, nv), c.two(nv, n3v, 1))
    gemm(split(Wvo, M, K, *wvo), B2, Z, zr(nv * nv), zc(nv, 1), 1.0, 1.0)
    np.testing.assert_allclose(Z.reshape(ref.shape), ref, rtol=0, atol=1e-12)


def test_xy_maps():
    no, nv = NO, NV
    rng = np.random.default_rng(2)
    Wvvvo, Wvooo = rng.standard_normal((nv, nv, nv, no)), rng.standard_normal((nv, no, no, no))
    t2 = rng.standard_normal((no, no, nv, nv))
    N = no * no * nv
    X = np.zeros(no * nv * nv * N)
    gemm(split(Wvvvo, no * nv * nv, nv, c.two(nv * nv, 1, nv * no), c.lin(no)),
         split(t2, no * no * nv, nv, c.two(nv, nv * nv, 1), c.lin(nv)), X, c.lin(N), c.lin(1), 1.0, 0.0)
    gemm(split(Wvooo, no * no * nv, no, c.three(no, nv, no, 1, no ** 3), c.lin(no * no)),
         split(t2, no * nv * nv, no, c.lin(1), c.lin(no * nv * nv)), X,
         c.three(no, nv, no * nv, nv * nv * N, nv * N), c.three(nv, nv, nv, N, 1), -1.0, 1.0)
    ref = e('abdj,ikdc->jabikc', Wvvvo, t2) - e('alij,lkbc->jabikc', Wvooo, t2)
    np.testing.assert_allclose(X.reshape(ref.shape), ref, rtol=0, atol=1e-12)


def test_wvvvv_maps():
    nv, nb = NV, 5
    rng = np.random.default_rng(3)
    W, t3 = rng.standard_normal((nv,) * 4), rng.standard_normal((nb, nv, nv, nv))
    r = np.zeros(t3.size)
    Ws = split(W, nv * nv, nv * nv, c.lin(nv * nv), c.lin(1))
    for am, ak, er, ec in c.wvvvv_maps(nv):
        gemm(split(t3, nb * nv, nv * nv, am, ak), Ws, r, er, ec, 1.0, 1.0)
    ref = e('abde,qdec->qabc', W, t3) + e('acde,qdbe->qabc', W, t3) + e('bcde,qade->qabc', W, t3)
    np.testing.assert_allclose(r.reshape(ref.shape), ref, rtol=0, atol=1e-12)
