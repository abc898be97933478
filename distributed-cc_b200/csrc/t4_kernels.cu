// T4 kernels: the 1 - P[4] - P[3,1] projector, P4 spin summations (single
// block, many blocks, and the (Q) form with the occupied axes inner),
// three-term transpose-add, quadruple-sym, r4 division, unpack of any
// ordering, block gather and t4 += r4.
#include <string.h>

#include "s4_orbit.cuh"

namespace dcc {

constexpr int S4_THREADS = 256;
constexpr int S4_WARPS = S4_THREADS / 32;

// One warp per (outer block, orbit): A <- beta*A + alpha*Q(A) with
// Q = (Omega-6)(Omega-2)(2 Omega^2 + 19 Omega + 48)/576 (src/rccsdtq.c:262-287).
__global__ void __launch_bounds__(S4_THREADS) k_t4_project(double *A, int64_t nouter, int nv, int64_t norb,
                                                           double alpha, double beta) {
    const int lane = threadIdx.x & 31;
    int partner[6];
    s4_partners(lane, partner);
    const int64_t n4 = (int64_t)nv * nv * nv * nv;
    const int64_t total = nouter * norb;
    for (int64_t w = (int64_t)blockIdx.x * S4_WARPS + (threadIdx.x >> 5); w < total; w += (int64_t)gridDim.x * S4_WARPS) {
        int64_t o = w / norb, r = w % norb;
        int asc[4], base[4], pos[4];
        decode_tri4(r, nv, asc);
        base[0] = asc[3]; base[1] = asc[2]; base[2] = asc[1]; base[3] = asc[0];
        int64_t off = o * n4 + s4_lane_offset(lane, base, nv, pos);
        double x = A[off];
        double x1 = dsub(omega6(x, partner), dmul(6.0, x));
        double x2 = dsub(omega6(x1, partner), dmul(2.0, x1));
        double x3 = omega6(x2, partner);
        double x4 = omega6(x3, partner);
        double y = __ddiv_rn(dadd(dadd(dmul(2.0, x4), dmul(19.0, x3)), dmul(48.0, x2)), 576.0);
        double out = dadd(dmul(beta, x), dmul(alpha, y));
        if (s4_first_holder(lane, off)) A[off] = out;
    }
}

// One warp per (outer block, orbit): A <- alpha*P(A) + beta*A.
__global__ void __launch_bounds__(S4_THREADS) k_t4_spin_sum(double *A, int64_t nouter, int n, int64_t norb,
                                                            P4Coef k) {
    const int lane = threadIdx.x & 31;
    int partner[6];
    s4_partners(lane, partner);
    const int64_t n4 = (int64_t)n * n * n * n;
    const int64_t total = nouter * norb;
    for (int64_t w = (int64_t)blockIdx.x * S4_WARPS + (threadIdx.x >> 5); w < total; w += (int64_t)gridDim.x * S4_WARPS) {
        int64_t o = w / norb, r = w % norb;
        int asc[4], base[4], pos[4];
        decode_tri4(r, n, asc);
        base[0] = asc[3]; base[1] = asc[2]; base[2] = asc[1]; base[3] = asc[0];
        int64_t off = o * n4 + s4_lane_offset(lane, base, n, pos);
        double x = A[off];
        double out = p4_apply(x, partner, k);
        if (s4_first_holder(lane, off)) A[off] = out;
    }
}

#define V4(a, b, c, d) ((((int64_t)(a) * nv + (b)) * nv + (c)) * nv + (d))

__global__ void k_t4_transpose_add(const double *src, double *dst, int nv) {
    const int64_t n4 = (int64_t)nv * nv * nv * nv;
    src += blockIdx.y * n4;  // block blockIdx.y of a batch
    dst += blockIdx.y * n4;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += (int64_t)gridDim.x * blockDim.x) {
        int d = (int)(e % nv), c = (int)((e / nv) % nv), b = (int)((e / ((int64_t)nv * nv)) % nv),
            a = (int)(e / ((int64_t)nv * nv * nv));
        dst[e] = dadd(dadd(src[e], src[V4(c, a, b, d)]), src[V4(d, a, c, b)]);
    }
}

__global__ void k_t4_quadruple_sym(const double *src, double *B0, double *B1, double *B2, double *B3, int nv) {
    const int64_t n4 = (int64_t)nv * nv * nv * nv;
    const int64_t o = blockIdx.y * n4;  // block blockIdx.y of a batch
    src += o;
    B0 += o;
    B1 += o;
    B2 += o;
    B3 += o;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += (int64_t)gridDim.x * blockDim.x) {
        int d = (int)(e % nv), c = (int)((e / nv) % nv), b = (int)((e / ((int64_t)nv * nv)) % nv),
            a = (int)(e / ((int64_t)nv * nv * nv));
        double two = dmul(2.0, src[e]);
        double bacd = src[V4(b, a, c, d)], cbad = src[V4(c, b, a, d)], dbca = src[V4(d, b, c, a)];
        double acbd = src[V4(a, c, b, d)], adcb = src[V4(a, d, c, b)], abdc = src[V4(a, b, d, c)];
        B0[e] = dsub(dsub(dsub(two, dbca), adcb), abdc);
        B1[e] = dsub(dsub(dsub(two, cbad), acbd), abdc);
        B2[e] = dsub(dsub(dsub(two, bacd), acbd), adcb);
        B3[e] = dsub(dsub(dsub(two, bacd), cbad), dbca);
    }
}

__global__ void k_r4_divide(double *r4, const double *eia, const int32_t *ijkl, int64_t nlocal, int nv) {
    const int64_t n4 = (int64_t)nv * nv * nv * nv;
    for (int64_t q = blockIdx.y; q < nlocal; q += gridDim.y) {
        const double *ei = eia + (int64_t)ijkl[4 * q] * nv, *ej = eia + (int64_t)ijkl[4 * q + 1] * nv,
                     *ek = eia + (int64_t)ijkl[4 * q + 2] * nv, *el = eia + (int64_t)ijkl[4 * q + 3] * nv;
        double *blk = r4 + q * n4;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += (int64_t)gridDim.x * blockDim.x) {
            int d = (int)(e % nv), c = (int)((e / nv) % nv), b = (int)((e / ((int64_t)nv * nv)) % nv),
                a = (int)(e / ((int64_t)nv * nv * nv));
            blk[e] = __ddiv_rn(blk[e], dadd(dadd(dadd(ei[a], ej[b]), ek[c]), el[d]));
        }
    }
}

// out[v[ax0], v[ax1], v[ax2], v[ax3]] = src[v]; loc < 0 means zero-fill.
__global__ void k_unpack_t4(const double *src, double *out, int64_t loc, int ax0, int ax1, int ax2, int ax3, int nv) {
    const int64_t n4 = (int64_t)nv * nv * nv * nv;
    const int ax[4] = {ax0, ax1, ax2, ax3};
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += (int64_t)gridDim.x * blockDim.x) {
        if (loc < 0) {
            out[e] = 0.0;
            continue;
        }
        int u[4] = {(int)(e / ((int64_t)nv * nv * nv)), (int)((e / ((int64_t)nv * nv)) % nv), (int)((e / nv) % nv),
                    (int)(e % nv)};
        // output position u came from source v with u[m] = v[ax[m]]
        int v[4];
        for (int m = 0; m < 4; m++) v[ax[m]] = u[m];
        out[e] = src[loc * n4 + V4(v[0], v[1], v[2], v[3])];
    }
}
#undef V4

__global__ void k_copy_blocks4(const double *in, double *out, const int32_t *req, const int64_t *map, int64_t nreq,
                               int64_t blk) {
    for (int64_t r = blockIdx.y; r < nreq; r += gridDim.y) {
        int64_t l = map[req[r]];
        if (l < 0) continue;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < blk; e += (int64_t)gridDim.x * blockDim.x)
            out[r * blk + e] = in[l * blk + e];
    }
}

__global__ void k_axpy1(double *t, const double *r, int64_t n) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        t[e] = dadd(t[e], r[e]);
}

static unsigned grid1d(int64_t n, int threads = 256) {
    int64_t g = (n + threads - 1) / threads;
    return (unsigned)(g < 148 * 32 ? (g ? g : 1) : 148 * 32);
}

static unsigned s4_grid(int64_t warps) {
    int64_t g = (warps + S4_WARPS - 1) / S4_WARPS;
    return (unsigned)(g < 148 * 64 ? (g ? g : 1) : 148 * 64);
}

int p4_coef(const char *pattern, double alpha, double beta, P4Coef &k) {
    if (p4_pattern(pattern, k.p)) {
        set_error("unrecognized pattern \"%s\"", pattern ? pattern : "(null)");
        return DCC_ERR_PATTERN;
    }
    k.alpha = alpha;
    k.beta = beta;
    return DCC_OK;
}

// Stable sort of (i,j,k,l): sorted values and, per input axis, its sorted slot
// (src/rccsdtq.c:931-960).
static void sort4_stable(const int64_t v[4], int64_t s[4], int ax[4]) {
    int64_t val[4] = {v[0], v[1], v[2], v[3]};
    int pos[4] = {0, 1, 2, 3};
    for (int a = 1; a < 4; a++)
        for (int b = a; b > 0 && val[b - 1] > val[b]; b--) {
            int64_t t = val[b]; val[b] = val[b - 1]; val[b - 1] = t;
            int u = pos[b]; pos[b] = pos[b - 1]; pos[b - 1] = u;
        }
    for (int m = 0; m < 4; m++) s[m] = val[m];
    for (int d = 0; d < 4; d++)
        for (int q = 0; q < 4; q++)
            if (pos[q] == d) { ax[d] = q; break; }
}

}  // namespace dcc

using namespace dcc;

extern "C" int dcc_t4_project_1_minus_p4_p31_inplace(double *A, int64_t nocc4, int64_t nvir, double alpha,
                                                     double beta, void *stream) {
    clear_error();
    DCC_REQUIRE(nocc4 >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nocc4 == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(A, DCC_ERR_NULL, "A is NULL");
    int64_t norb = binom(nvir + 3, 4);
    k_t4_project<<<s4_grid(nocc4 * norb), S4_THREADS, 0, as_stream(stream)>>>(A, nocc4, (int)nvir, norb, alpha, beta);
    return launch_status("t4_project_1_minus_p4_p31");
}

extern "C" int dcc_t4_spin_summation_inplace(double *A, int64_t nouter, int64_t ninner, const char *pattern,
                                             double alpha, double beta, void *stream) {
    clear_error();
    P4Coef k;
    int rc = p4_coef(pattern, alpha, beta, k);
    if (rc) return rc;
    DCC_REQUIRE(nouter >= 0 && ninner >= 0, DCC_ERR_SHAPE, "negative size");
    if (nouter == 0 || ninner == 0) return DCC_OK;
    DCC_REQUIRE(A, DCC_ERR_NULL, "A is NULL");
    int64_t norb = binom(ninner + 3, 4);
    k_t4_spin_sum<<<s4_grid(nouter * norb), S4_THREADS, 0, as_stream(stream)>>>(A, nouter, (int)ninner, norb, k);
    return launch_status("t4_spin_summation");
}

extern "C" int dcc_t4_transpose_add(const double *src, double *dst, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nvir == 0) return DCC_OK;
    DCC_REQUIRE(src && dst && src != dst, DCC_ERR_NULL, "NULL or aliased buffer");
    int64_t n4 = nvir * nvir * nvir * nvir;
    k_t4_transpose_add<<<grid1d(n4), 256, 0, as_stream(stream)>>>(src, dst, (int)nvir);
    return launch_status("t4_transpose_add");
}

extern "C" int dcc_t4_spin_summation_quadruple_sym(const double *src, double *B0, double *B1, double *B2, double *B3,
                                                   int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nvir == 0) return DCC_OK;
    DCC_REQUIRE(src && B0 && B1 && B2 && B3, DCC_ERR_NULL, "NULL buffer");
    int64_t n4 = nvir * nvir * nvir * nvir;
    k_t4_quadruple_sym<<<grid1d(n4), 256, 0, as_stream(stream)>>>(src, B0, B1, B2, B3, (int)nvir);
    return launch_status("t4_quadruple_sym");
}

extern "C" int dcc_t4_transpose_add_batched(const double *src, double *dst, int64_t nblocks, int64_t nvir,
                                            void *stream) {
    clear_error();
    DCC_REQUIRE(nvir >= 0 && nblocks >= 0 && nblocks < 65536, DCC_ERR_SHAPE, "bad size");
    if (nvir == 0 || nblocks == 0) return DCC_OK;
    DCC_REQUIRE(src && dst && src != dst, DCC_ERR_NULL, "NULL or aliased buffer");
    int64_t n4 = nvir * nvir * nvir * nvir;
    unsigned gx = grid1d(n4);
    gx = gx > 64 ? 64 : gx;
    k_t4_transpose_add<<<dim3(gx, (unsigned)nblocks), 256, 0, as_stream(stream)>>>(src, dst, (int)nvir);
    return launch_status("t4_transpose_add_batched");
}

extern "C" int dcc_t4_spin_summation_quadruple_sym_batched(const double *src, double *B0, double *B1, double *B2,
                                                           double *B3, int64_t nblocks, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nvir >= 0 && nblocks >= 0 && nblocks < 65536, DCC_ERR_SHAPE, "bad size");
    if (nvir == 0 || nblocks == 0) return DCC_OK;
    DCC_REQUIRE(src && B0 && B1 && B2 && B3, DCC_ERR_NULL, "NULL buffer");
    int64_t n4 = nvir * nvir * nvir * nvir;
    unsigned gx = grid1d(n4);
    gx = gx > 64 ? 64 : gx;
    k_t4_quadruple_sym<<<dim3(gx, (unsigned)nblocks), 256, 0, as_stream(stream)>>>(src, B0, B1, B2, B3, (int)nvir);
    return launch_status("t4_quadruple_sym_batched");
}

extern "C" int dcc_r4_local_tri_divide_e(double *r4_local, const double *eia, const int32_t *local_ijkl,
                                         int64_t nlocal, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nlocal >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nlocal == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(r4_local && eia && local_ijkl, DCC_ERR_NULL, "NULL buffer");
    int64_t n4 = nvir * nvir * nvir * nvir;
    unsigned gx = grid1d(n4);
    gx = gx > 64 ? 64 : gx;
    dim3 grid(gx, (unsigned)(nlocal < 65535 ? nlocal : 65535));
    k_r4_divide<<<grid, 256, 0, as_stream(stream)>>>(r4_local, eia, local_ijkl, nlocal, (int)nvir);
    return launch_status("r4_local_tri_divide_e");
}

extern "C" int dcc_unpack_t4_ijkl_single(const double *t4_local, double *t4_blk, const int64_t *ijkl_to_local_idx,
                                         int64_t i, int64_t j, int64_t k, int64_t l, int64_t nocc, int64_t nvir,
                                         void *stream) {
    clear_error();
    DCC_REQUIRE(i >= 0 && j >= 0 && k >= 0 && l >= 0 && i < nocc && j < nocc && k < nocc && l < nocc,
                DCC_ERR_SHAPE, "occupied index out of range");
    DCC_REQUIRE(t4_blk && ijkl_to_local_idx, DCC_ERR_NULL, "NULL buffer");
    int64_t v[4] = {i, j, k, l}, s[4];
    int ax[4];
    sort4_stable(v, s, ax);
    int64_t loc;
    if ((s[0] == s[1] && s[1] == s[2]) || (s[1] == s[2] && s[2] == s[3])) {
        loc = -1;  // zero-rule block: zero-fill
    } else {
        loc = ijkl_to_local_idx[ijkl_linear(s[0], s[1], s[2], s[3], nocc)];
        if (loc < 0) {
            set_error("block (%lld,%lld,%lld,%lld) is not stored", (long long)s[0], (long long)s[1],
                      (long long)s[2], (long long)s[3]);
            return DCC_ERR_NOT_LOCAL;
        }
        DCC_REQUIRE(t4_local, DCC_ERR_NULL, "t4_local is NULL");
    }
    int64_t n4 = nvir * nvir * nvir * nvir;
    k_unpack_t4<<<grid1d(n4), 256, 0, as_stream(stream)>>>(t4_local, t4_blk, loc, ax[0], ax[1], ax[2], ax[3],
                                                            (int)nvir);
    return launch_status("unpack_t4_ijkl_single");
}

extern "C" int dcc_fill_local_data_ijkl(const double *t4_local, double *send_data, const int32_t *requests,
                                        const int64_t *ijkl_to_local_idx, int64_t n_requests, int64_t nvir,
                                        void *stream) {
    clear_error();
    DCC_REQUIRE(n_requests >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (n_requests == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t4_local && send_data && requests && ijkl_to_local_idx, DCC_ERR_NULL, "NULL buffer");
    int64_t blk = nvir * nvir * nvir * nvir;
    unsigned gx = grid1d(blk);
    gx = gx > 64 ? 64 : gx;
    dim3 grid(gx, (unsigned)(n_requests < 65535 ? n_requests : 65535));
    k_copy_blocks4<<<grid, 256, 0, as_stream(stream)>>>(t4_local, send_data, requests, ijkl_to_local_idx, n_requests,
                                                        blk);
    return launch_status("fill_local_data_ijkl");
}

extern "C" int dcc_t4_add(double *t4, const double *r4, int64_t n, void *stream) {
    clear_error();
    DCC_REQUIRE(n >= 0, DCC_ERR_SHAPE, "negative size");
    if (n == 0) return DCC_OK;
    DCC_REQUIRE(t4 && r4, DCC_ERR_NULL, "NULL buffer");
    k_axpy1<<<grid1d(n), 256, 0, as_stream(stream)>>>(t4, r4, n);
    return launch_status("t4_add");
}
