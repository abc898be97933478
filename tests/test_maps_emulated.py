"""The address maps the residual drivers hand to dcc_split_operand and
dcc_gemm_split3, checked on the CPU: the split, the GEMM and the epilogue
scatter are emulated in numpy with the same three-digit map arithmetic the
kernels use, and compared with numpy einsums of the terms they implement."""
import numpy as np

from dcc import contract as c


def fmap(f, m):
    R1, R2, R3, S0, S1, S2, S3 = c.as4(f)
    m = np.asarray(m, dtype=np.int64)
    return (m // (R1 * R2 * R3)) * S0 + ((m // (R2 * R3)) % R1) * S1 + ((m // R3) % R2) * S2 + (m % R3) * S3


def split(src, M, K, fm, fk):
    return src.ravel()[fmap(fm, np.arange(M))[:, None] + fmap(fk, np.arange(K))[None, :]]


def gemm(A, B, C, fr, fc, alpha, beta):
    idx = fmap(fr, np.arange(A.shape[0]))[:, None] + fmap(fc, np.arange(B.shape[0]))[None, :]
    assert len(np.unique(idx)) == idx.size  # the epilogue map never writes an element twice
    flat = C.ravel()
    # beta = 0 overwrites without reading C, as the kernel's epilogue does
    flat[idx] = alpha * (A @ B.T) + (beta * flat[idx] if beta != 0.0 else 0.0)


NO, NV = 3, 4
e = np.einsum


def split_pieces(srcs, M, pieces, Kp):
    """Emulated K-concatenated Split: piece i = (offset, K_i, width) filled from srcs[i] = (src, fm, fk)."""
    A = np.zeros((M, Kp))
    for (off, k, _), (src, fm, fk) in zip(pieces, srcs):
        A[:, off:off + k] = split(src, M, k, fm, fk)
    return A


def test_s_plan_maps():
    """The GEMMs of t3_residual.s_plan build S = X + T1 + T2 + T5/2 in S's layout."""
    import torch
    from dcc import t3_residual as tr
    no, nv = NO, NV
    rng = np.random.default_rng(1)
    Wvvvo, t2 = rng.standard_normal((nv, nv, nv, no)), rng.standard_normal((no, no, nv, nv))
    Wov, Wvo = rng.standard_normal((no, nv, no, nv)), rng.standard_normal((no, nv, nv, no))
    U = rng.standard_normal((no, no, no, nv, nv, nv))
    G2 = -0.5 * (Wov + Wvo.transpose(0, 1, 3, 2))  # [l,a,i,d]
    ref = (e('abdj,ikdc->ijkabc', Wvvvo, t2) - e('lbid,jkldca->ijkabc', Wov, U) + e('laid,jkldcb->ijkabc', G2, U)
           + 0.5 * e('ladi,jklbcd->ijkabc', Wvo, U))
    src = {"W_vvvo": Wvvvo, "t2": t2, "W_ovov": Wov, "Wvo_half": 0.5 * Wvo, "U": U,
           "G2": G2.transpose(2, 1, 0, 3).copy()}
    plan = tr.s_plan(no, nv)
    S = np.full(ref.size, np.nan)
    K = no * nv
    shapes = {"x": (no * nv * nv, no * no * nv, [nv]), "oo": (no * nv, no * no * nv * nv, [K, K])}
    ops = {}
    for key, (M, N, pieces) in shapes.items():
        sp = c.Split(M, kind=0, device="cpu", pieces=pieces)
        ent = plan[key]
        A = split_pieces([(src[n], fm, fk) for n, fm, fk in ent["a"]], M, sp.pieces, sp.Kp)
        B = split_pieces([(src[n], fm, fk) for n, fm, fk in ent["b"]], N, sp.pieces, sp.Kp)
        ops[key] = (A, B)
        if key == "x":
            S[:] = 0.0  # beta = 0 of the first GEMM overwrites S
        gemm(A, B, S, *ent["out"], ent["alpha"], ent["beta"])
    t1 = plan["t1"]
    sp = c.Split(no * nv, K, 0, device="cpu")
    A = split_pieces([(src[n], fm, fk) for n, fm, fk in t1["a"]], no * nv, sp.pieces, sp.Kp)
    B = ops["oo"][1][:, :sp.Kp]  # leading columns of the T2/T5 U operand
    gemm(A, B, S, *t1["out"], t1["alpha"], t1["beta"])
    del torch
    np.testing.assert_allclose(S.reshape(ref.shape), ref, rtol=0, atol=1e-12)


def test_y_strides():
    """Y[(i,j,a),(k,b,c)] read through T3Residual.y_strides is Y[ijk][abc]."""
    no, nv = NO, NV
    rng = np.random.default_rng(2)
    Wvooo, t2 = rng.standard_normal((nv, no, no, no)), rng.standard_normal((no, no, nv, nv))
    Y = (Wvooo.transpose(2, 3, 0, 1).reshape(no * no * nv, no) @ t2.transpose(1, 2, 3, 0).reshape(no * nv * nv, no).T)
    Ny = no * nv * nv
    st = (no * nv * Ny, nv * Ny, nv * nv, Ny, nv, 1)
    ref = e('alij,lkbc->ijkabc', Wvooo, t2)
    idx = np.indices(ref.shape).reshape(6, -1)
    got = Y.ravel()[sum(idx[m] * st[m] for m in range(6))]
    np.testing.assert_allclose(got, ref.ravel(), rtol=0, atol=1e-13)


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


def test_einsum_into_maps():
    """contract.einsum_into's digit grouping: the split and epilogue maps it builds,
    emulated in numpy, reproduce torch.einsum for (Q)-style strings, including
    sliced (non-contiguous) operands and a strided output."""
    import torch
    rng = np.random.default_rng(4)
    no, nv = 2, 5
    T = torch.from_numpy(rng.standard_normal((3, 4, nv, no, no, no)))
    W = torch.from_numpy(rng.standard_normal((nv, nv, nv, no)))
    V = torch.from_numpy(rng.standard_normal((nv, no, no, no)))
    t2 = torch.from_numpy(rng.standard_normal((nv, nv, no, no)))
    cases = [('cdel,abeijk->abcdijkl', W[1:3, 2:5], T), ('dmli,abcmjk->abcdijkl', V[2:5], T[:, :, 1:3]),
             ('cmki,abdmjl->abcdijkl', V[1:3], T[:, :, 2:5]), ('abef,fcjk->abcejk', W[..., 0].reshape(nv, nv, nv, 1)
                                                                  .expand(nv, nv, nv, nv)[0:2, 1:4].contiguous(), t2[:, 1:3]),
             ('mnki,abnj->abmijk', torch.from_numpy(rng.standard_normal((no,) * 4)), t2[1:4, 0:2]),
             ('acdekl,ebij->abcdijkl', torch.from_numpy(rng.standard_normal((2, 3, 2, nv, no, no))), t2[:, 1:3])]
    checked = 0
    for subs, X, Y in cases:
        ref = torch.einsum(subs, X, Y)
        base = torch.zeros(ref.numel() * 2, dtype=torch.float64)
        out = base[::2].view(ref.shape)  # every other element: a strided output
        ins, o = subs.split('->')
        xs, ys = ins.split(',')
        K = [ch for ch in xs if ch in ys]
        Mi = [ch for ch in xs if ch not in ys]
        Ni = [ch for ch in ys if ch not in xs]
        size = {ch: X.shape[xs.index(ch)] for ch in xs}
        size.update({ch: Y.shape[ys.index(ch)] for ch in ys})
        sX = {ch: X.stride(xs.index(ch)) for ch in xs}
        sY = {ch: Y.stride(ys.index(ch)) for ch in ys}
        sO = {ch: out.stride(o.index(ch)) for ch in o}
        gM, gN, gK = (c._digit_orders(Mi, size, [sX, sO]), c._digit_orders(Ni, size, [sY, sO]),
                      c._digit_orders(K, size, [sX, sY]))
        if gM is None or gN is None or gK is None:
            continue  # more than four digits: einsum_into takes the FP64 path
        checked += 1
        m, n, k = (int(np.prod([size[ch] for ch in g])) for g in (Mi, Ni, K))
        xf = X.as_strided((X.storage().size() - X.storage_offset(),), (1,)).numpy()
        yf = Y.as_strided((Y.storage().size() - Y.storage_offset(),), (1,)).numpy()
        A = xf[fmap(c._map_of(gM, 0), np.arange(m))[:, None] + fmap(c._map_of(gK, 0), np.arange(k))[None, :]]
        B = yf[fmap(c._map_of(gN, 0), np.arange(n))[:, None] + fmap(c._map_of(gK, 1), np.arange(k))[None, :]]
        gemm(A, B, base.numpy(), c._map_of(gM, 1), c._map_of(gN, 1), 1.0, 0.0)
        np.testing.assert_allclose(out.numpy(), ref.numpy(), rtol=0, atol=1e-12)
    assert checked >= 4
