// The per-block strings of compute_r4_tri (distr_cc/rccsdtq.py:862-1055) in ONE
// persistent launch over the stored T4 blocks, FP64.
//
// The reference walks its stored blocks (i<=j<=k<=l) and, for each, adds about a
// hundred strings  r4[q][a,b,c,d] += alpha W[..] . T[..]  whose operands are
// slices of full tensors at the block's occupied indices.  Every such string is a
// small GEMM over the block's virtual indices: the output letters that sit in W
// are its rows, those in T its columns, the summed letters (one or two of e, f,
// m, n) its contraction.  Here one CTA owns the output rows a in [a0, a0+na) of
// one stored block in shared memory and runs every string of a descriptor table
// over it: each thread takes 4x4 (row, column) micro-tiles of the string's GEMM,
// reads W and T through strides (operands stay in L2: at nvir ~ 11 the
// intermediates are a few MB), and adds alpha times its tile into the shared
// accumulator; one barrier separates consecutive strings, and the block is
// written once at the end.  The work and memory are those of the stored blocks
// only, and no operand is gathered or permuted in HBM.
//
// The W_ovov / W_voov strings of the OO batch (distr_cc/rccsdtq.py:1062-1349) take a
// stored SOURCE block and an occupied m per term: they run in "pair mode", once for
// every (source, m) pair that the output block's sparse pair list holds for the
// string's group (the reference's masked prefactor slots, only the nonzero ones).
// The F_oo / W_oooo prefactor strings are plain strings over the unpacked T4 of every
// ordering.
//
// A descriptor is 32 int64 (DCC_T4S_DESC_LEN; layout in include/dcc_b200.h).  Every
// string is checked in the kernel before it runs: operand indices, non-negative
// strides, letters in exactly one operand, and the largest offset it can reach
// inside its operand's element count; a string that fails is skipped and sets bit
// 2 of *status, a block whose occupied indices fall outside [0, nocc) sets bit 1, a pair
// (or pair range) that fails the same checks is skipped and sets bit 4.
#include "dcc_common.cuh"
#include "dcc_b200.h"

namespace dcc {

constexpr int T4S_THREADS = 256;
constexpr int T4S_MAXOPS = 32;
constexpr int T4S_DESC = 32;
constexpr int64_t T4S_SMEM_MAX = 200 * 1024;

struct T4StrOps {
    const double *p[T4S_MAXOPS];
    int64_t n[T4S_MAXOPS];
    int nops;
};

__device__ __forceinline__ int t4s_ostride(int x, int nv) {  // accumulator stride of output letter x
    return x == 0 ? nv * nv * nv : (x == 1 ? nv * nv : (x == 2 ? nv : 1));
}

__global__ void __launch_bounds__(T4S_THREADS, 2)
    k_t4_strings(T4StrOps ops, const int64_t *__restrict__ desc, int nstr, const int32_t *__restrict__ quads,
                 const int32_t *__restrict__ pair_off, const int32_t *__restrict__ pair_sm, int ngroups, int npairs,
                 int nocc, int nv, int na_step, int nsplit, double beta, double *__restrict__ r4, int *status) {
    extern __shared__ double acc[];
    const int q = blockIdx.x / nsplit, part = blockIdx.x % nsplit;
    const int a0 = part * na_step;
    const int na = min(na_step, nv - a0);
    const int nv3 = nv * nv * nv;
    const int nacc = na * nv3;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int e = threadIdx.x; e < nacc; e += blockDim.x) acc[e] = 0.0;
    int occ[4];
    bool occ_ok = true;
#pragma unroll
    for (int x = 0; x < 4; ++x) {
        occ[x] = quads[4 * (int64_t)q + x];
        occ_ok = occ_ok && occ[x] >= 0 && occ[x] < nocc;
    }
    if (!occ_ok) {  // uniform over the CTA
        if (threadIdx.x == 0) atomicOr(status, 1);
        return;
    }
    for (int s = 0; s < nstr; ++s) {
        __syncthreads();  // the previous string's tiles are in acc
        const int64_t *d = desc + (int64_t)s * T4S_DESC;
        const int64_t wop = d[0], top = d[1], mask = d[20], K0 = d[21], wk0 = d[22], tk0 = d[23], K1 = d[24],
                      wk1 = d[25], tk1 = d[26], rord = d[28], cord = d[29], wm = d[30], mode = d[31];
        const double alpha = __longlong_as_double((long long)d[27]);
        // ---- checks (uniform: every thread reads the same descriptor)
        bool ok = wop >= 0 && wop < ops.nops && top >= 0 && top < ops.nops && mask >= 0 && mask < 16 && K0 >= 1 &&
                  K1 >= 1 && wk0 >= 0 && tk0 >= 0 && wk1 >= 0 && tk1 >= 0 && d[10] >= 0 && d[11] >= 0 &&
                  rord >= 0 && rord < 65536 && cord >= 0 && cord < 65536 && wm >= 0 && mode >= 0 && mode <= ngroups;
        int64_t wb = 0, tb = 0, wmax = 0, tmax = 0;
        int seen_r = 0, seen_c = 0, npos_r = 0, npos_c = 0;
#pragma unroll
        for (int x = 0; x < 4; ++x) {
            const int64_t ws = d[2 + x], ts = d[6 + x], wv = d[12 + x], tv = d[16 + x];
            const bool inw = (mask >> x) & 1;
            ok = ok && ws >= 0 && ts >= 0 && wv >= 0 && tv >= 0 && (inw ? tv == 0 : wv == 0);
            wb += ws * occ[x];
            tb += ts * occ[x];
            const int ex = x == 0 ? na : nv;
            wmax += wv * (ex - 1);
            tmax += tv * (ex - 1);
            const int xr = (int)((rord >> (4 * x)) & 15) - 1, xc = (int)((cord >> (4 * x)) & 15) - 1;
            if (xr >= 0) {
                npos_r++;
                seen_r |= 1 << (xr & 7);
                ok = ok && xr < 4;
            }
            if (xc >= 0) {
                npos_c++;
                seen_c |= 1 << (xc & 7);
                ok = ok && xc < 4;
            }
        }
        // the row order lists the letters of W once each, the column order those of T
        ok = ok && seen_r == (int)mask && seen_c == (int)(15 & ~mask) && npos_r == __popc(seen_r) &&
             npos_c == __popc(seen_c);
        if (ok) {
            wb += d[10] * q + d[12] * a0;
            tb += (mode == 0 ? d[11] * q : 0) + d[16] * a0;  // pair mode: field 11 strides the source block
            wmax += wb + wk0 * (K0 - 1) + wk1 * (K1 - 1);
            tmax += tb + tk0 * (K0 - 1) + tk1 * (K1 - 1);
            ok = wmax < ops.n[wop] && tmax < ops.n[top];
        }
        if (!ok) {
            if (threadIdx.x == 0) atomicOr(status, 2);
            continue;
        }
        // ---- the string as a GEMM: rows = W's output letters in the row order (the last
        // position fastest), columns = T's in the column order
        int rext[4], cext[4], rws[4], cts[4], ros[4], cos_[4];
        int R = 1, C = 1;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int xr = (int)((rord >> (4 * p)) & 15) - 1, xc = (int)((cord >> (4 * p)) & 15) - 1;
            rext[p] = xr < 0 ? 1 : (xr == 0 ? na : nv);
            rws[p] = xr < 0 ? 0 : (int)d[12 + xr];
            ros[p] = xr < 0 ? 0 : t4s_ostride(xr, nv);
            cext[p] = xc < 0 ? 1 : (xc == 0 ? na : nv);
            cts[p] = xc < 0 ? 0 : (int)d[16 + xc];
            cos_[p] = xc < 0 ? 0 : t4s_ostride(xc, nv);
            R *= rext[p];
            C *= cext[p];
        }
        const int wk0i = (int)wk0, tk0i = (int)tk0, wk1i = (int)wk1, tk1i = (int)tk1, K0i = (int)K0, K1i = (int)K1;
        // a warp tile: Lr x Lc lanes, each lane 4 consecutive rows x 4 columns strided by Lc,
        // so a warp's loads of T cover Lc consecutive columns and its loads of W broadcast
        const int Lc = C > 64 ? 32 : (C > 32 ? 16 : (C > 16 ? 8 : (C > 8 ? 4 : (C > 4 ? 2 : 1))));
        const int Lr = 32 / Lc;
        const int lr = lane / Lc, lc = lane % Lc;
        const int nrt = (R + 4 * Lr - 1) / (4 * Lr), nct = (C + 4 * Lc - 1) / (4 * Lc);
        // pair mode: once per (source block, m) pair of group mode-1 of this block
        int p0 = 0, p1 = 1;
        if (mode > 0) {
            const int32_t *po = pair_off + (int64_t)q * (ngroups + 1) + (mode - 1);
            p0 = po[0];
            p1 = po[1];
            if (p0 < 0 || p1 < p0 || p1 > npairs) {
                if (threadIdx.x == 0) atomicOr(status, 4);
                continue;
            }
        }
        for (int pr = p0; pr < p1; ++pr) {
        int64_t wbp = wb, tbp = tb;
        if (mode > 0) {  // uniform: every thread reads the same pair
            const int src = pair_sm[2 * (int64_t)pr], m = pair_sm[2 * (int64_t)pr + 1];
            const int64_t dw = wm * m, dt = d[11] * src;
            if (src < 0 || m < 0 || m >= nocc || wmax + dw >= ops.n[wop] || tmax + dt >= ops.n[top]) {
                if (threadIdx.x == 0) atomicOr(status, 4);
                continue;
            }
            wbp += dw;
            tbp += dt;
        }
        const double *W = ops.p[wop] + wbp;
        const double *T = ops.p[top] + tbp;
        for (int tile = warp; tile < nrt * nct; tile += T4S_THREADS / 32) {
            const int r0 = (tile / nct) * 4 * Lr + lr * 4, c0 = (tile % nct) * 4 * Lc + lc;
            int wo[4], to[4], oR[4], oC[4];
            bool rv[4], cv[4];
            int dg[4];  // digits of row r0 (position p), then stepped by one row at a time
            {
                int r = r0 < R ? r0 : 0;
#pragma unroll
                for (int p = 3; p >= 0; --p) {
                    dg[p] = r % rext[p];
                    r /= rext[p];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                rv[u] = r0 + u < R;
                int o = 0, oa = 0;
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    o += rws[p] * dg[p];
                    oa += ros[p] * dg[p];
                }
                wo[u] = rv[u] ? o : 0;
                oR[u] = oa;
                bool carry = true;  // next row
#pragma unroll
                for (int p = 3; p >= 0; --p) {
                    if (carry) {
                        dg[p] += 1;
                        carry = dg[p] >= rext[p];
                        if (carry) dg[p] = 0;
                    }
                }
                int c = c0 + u * Lc;
                cv[u] = c < C;
                c = cv[u] ? c : 0;
                o = 0;
                oa = 0;
#pragma unroll
                for (int p = 3; p >= 0; --p) {
                    const int ix = c % cext[p];
                    c /= cext[p];
                    o += cts[p] * ix;
                    oa += cos_[p] * ix;
                }
                to[u] = o;
                oC[u] = oa;
            }
            double cacc[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) cacc[u][v] = 0.0;
            for (int k1 = 0; k1 < K1i; ++k1) {
                const double *Wk = W + k1 * wk1i;
                const double *Tk = T + k1 * tk1i;
                for (int k0 = 0; k0 < K0i; ++k0, Wk += wk0i, Tk += tk0i) {
                    double av[4], bv[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        av[u] = __ldg(Wk + wo[u]);
                        bv[u] = __ldg(Tk + to[u]);
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u)
#pragma unroll
                        for (int v = 0; v < 4; ++v) cacc[u][v] = fma(av[u], bv[v], cacc[u][v]);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v)
                    if (rv[u] && cv[v]) acc[oR[u] + oC[v]] += alpha * cacc[u][v];
        }
        }  // pairs: a string's micro-tiles belong to the same threads for every pair
    }
    __syncthreads();
    double *out = r4 + (int64_t)q * nv * nv3 + (int64_t)a0 * nv3;
    if (beta == 0.0) {
        for (int e = threadIdx.x; e < nacc; e += blockDim.x) out[e] = acc[e];
    } else {
        for (int e = threadIdx.x; e < nacc; e += blockDim.x) out[e] = beta * out[e] + acc[e];
    }
}

}  // namespace dcc

using namespace dcc;

extern "C" int dcc_t4_strings_rows_per_cta(int64_t nq, int64_t nvir) {
    if (nq <= 0 || nvir <= 0) return -1;
    const int64_t row = nvir * nvir * nvir * (int64_t)sizeof(double);
    const int64_t na_max = T4S_SMEM_MAX / row;
    if (na_max < 1) return -1;
    // at least ~3 CTAs per SM over the stored blocks, within the shared-memory limit
    int64_t nsplit = (3 * 148 + nq - 1) / nq;
    nsplit = nsplit < 1 ? 1 : (nsplit > nvir ? nvir : nsplit);
    int64_t na = (nvir + nsplit - 1) / nsplit;
    if (na > na_max) na = na_max;
    return (int)na;
}

extern "C" int dcc_t4_strings(const double *const *ops, const int64_t *op_numel, int nops, const int64_t *desc,
                              int nstr, const int32_t *quads, int64_t nq, const int32_t *pair_off,
                              const int32_t *pair_sm, int ngroups, int64_t npairs, int64_t nocc, int64_t nvir,
                              double beta, double *r4, int *status, void *stream) {
    clear_error();
    DCC_REQUIRE(nops >= 1 && nops <= T4S_MAXOPS, DCC_ERR_SHAPE, "1 to 32 operands");
    DCC_REQUIRE(ngroups >= 0 && ngroups < 4096 && npairs >= 0 && npairs < (1LL << 30), DCC_ERR_SHAPE,
                "bad pair lists");
    DCC_REQUIRE(ngroups == 0 || (pair_off && pair_sm), DCC_ERR_NULL, "NULL pair lists");
    DCC_REQUIRE(nstr >= 0 && nq >= 0 && nocc >= 1 && nvir >= 1 && nq < (1LL << 24) && nvir < 1024, DCC_ERR_SHAPE,
                "bad size");
    if (nq == 0) return DCC_OK;
    DCC_REQUIRE(ops && op_numel && desc && quads && r4 && status, DCC_ERR_NULL, "NULL argument");
    T4StrOps o = {};
    for (int i = 0; i < nops; ++i) {
        DCC_REQUIRE(ops[i] && op_numel[i] >= 1, DCC_ERR_NULL, "NULL or empty operand");
        DCC_REQUIRE(op_numel[i] < (1LL << 31), DCC_ERR_SHAPE, "operands must hold fewer than 2^31 elements");
        o.p[i] = ops[i];
        o.n[i] = op_numel[i];
    }
    o.nops = nops;
    const int na = dcc_t4_strings_rows_per_cta(nq, nvir);
    DCC_REQUIRE(na >= 1, DCC_ERR_SHAPE, "nvir^3 doubles exceed the shared-memory accumulator");
    const int nsplit = (int)((nvir + na - 1) / na);
    const int64_t grid = nq * nsplit;
    DCC_REQUIRE(grid < (1LL << 31), DCC_ERR_SHAPE, "too many blocks");
    const size_t smem = (size_t)na * nvir * nvir * nvir * sizeof(double);
    static_assert(T4S_SMEM_MAX <= 227 * 1024, "shared memory per CTA");
    cudaFuncSetAttribute(k_t4_strings, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T4S_SMEM_MAX);
    k_t4_strings<<<(unsigned)grid, T4S_THREADS, smem, as_stream(stream)>>>(
        o, desc, nstr, quads, pair_off, pair_sm, ngroups, (int)npairs, (int)nocc, (int)nvir, na, nsplit, beta, r4,
        status);
    return launch_status("t4_strings");
}
