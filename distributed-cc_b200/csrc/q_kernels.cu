// (Q) denominator-and-energy loop: the reference's separate division and
// factor kernels, and one fused per-task epilogue that evaluates
//   t~4 = factor(abcd) * P4_444_ijkl((t4 + z4) / D)
// and both energy dot products without writing any block back.
#include <utility>

#include "s4_orbit.cuh"

namespace dcc {

int p4_coef(const char *pattern, double alpha, double beta, P4Coef &k);

struct QRange {
    int a0, a1, b0, b1, c0, c1, d0, d1;
};

// r4[abcd][ijkl] /= D (src/rccsdt_q.c:474-588): D = ((e_i+e_j)+(e_k+e_l)) + neg,
// neg = -(((e_a+e_b)+e_c)+e_d); exact zero where |D| <= 1e-15.
__global__ void k_q_division(double *r4, const double *eo, const double *ev, QRange R, int bb, int bc, int bd, int no) {
    const int64_t n4 = (int64_t)no * no * no * no;
    const int ba_ = R.a1 - R.a0, bb_ = R.b1 - R.b0, bc_ = R.c1 - R.c0, bd_ = R.d1 - R.d0;
    const int64_t nsub = (int64_t)ba_ * bb_ * bc_ * bd_;
    for (int64_t s = blockIdx.y; s < nsub; s += gridDim.y) {
        int id = (int)(s % bd_), ic = (int)((s / bd_) % bc_), ib = (int)((s / ((int64_t)bd_ * bc_)) % bb_),
            ia = (int)(s / ((int64_t)bd_ * bc_ * bb_));
        int a = R.a0 + ia, b = R.b0 + ib, c = R.c0 + ic, d = R.d0 + id;
        double neg = -dadd(dadd(dadd(ev[a], ev[b]), ev[c]), ev[d]);
        double *blk = r4 + ((((int64_t)ia * bb + ib) * bc + ic) * bd + id) * n4;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += (int64_t)gridDim.x * blockDim.x) {
            int l = (int)(e % no), k = (int)((e / no) % no), j = (int)((e / ((int64_t)no * no)) % no),
                i = (int)(e / ((int64_t)no * no * no));
            double den = dadd(dadd(dadd(eo[i], eo[j]), dadd(eo[k], eo[l])), neg);
            blk[e] = (fabs(den) > 1e-15) ? __ddiv_rn(blk[e], den) : 0.0;
        }
    }
}

__global__ void k_q_factor(double *t4, const double *factor, int64_t nsub, int64_t n4) {
    for (int64_t s = blockIdx.y; s < nsub; s += gridDim.y) {
        double f = factor[s];
        double *blk = t4 + s * n4;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n4; e += (int64_t)gridDim.x * blockDim.x)
            blk[e] = (f == 0.0) ? 0.0 : dmul(blk[e], f);
    }
}

// factor of a virtual quadruple (distr_cc/rccsdt_q.py:410-428)
__device__ __forceinline__ double q_factor(int a, int b, int c, int d) {
    if (a < b && b < c && c < d) return 24.0;
    if ((a == b && b < c && c < d) || (a < b && b == c && c < d) || (a < b && b < c && c == d)) return 12.0;
    if (a == b && b < c && c == d) return 6.0;
    return 0.0;
}

constexpr int QE_THREADS = 256;
constexpr int QE_WARPS = QE_THREADS / 32;

// One warp per (valid abcd sub-block, ijkl orbit).  Per-CTA partial sums of
// <t~4, z4sq> and <t~4, z4> go to ws[2*cta].
__global__ void __launch_bounds__(QE_THREADS) k_q_epilogue(const double *t4, const double *z4, const double *vvoo,
                                                           const double *t2, const double *eo, const double *ev,
                                                           QRange R, int blk, int no, int nv, int64_t norb,
                                                           P4Coef k, double *ws) {
    const int lane = threadIdx.x & 31;
    int partner[6];
    s4_partners(lane, partner);
    const int64_t n4 = (int64_t)no * no * no * no;
    const int ba = R.a1 - R.a0, bb = R.b1 - R.b0, bc = R.c1 - R.c0, bd = R.d1 - R.d0;
    const int64_t nsub = (int64_t)ba * bb * bc * bd;
    const int64_t total = nsub * norb;
    const int64_t no2 = (int64_t)no * no;
    double s_br = 0.0, s_pa = 0.0;
    for (int64_t w = (int64_t)blockIdx.x * QE_WARPS + (threadIdx.x >> 5); w < total; w += (int64_t)gridDim.x * QE_WARPS) {
        int64_t s = w / norb, r = w % norb;
        int id = (int)(s % bd), ic = (int)((s / bd) % bc), ib = (int)((s / ((int64_t)bd * bc)) % bb),
            ia = (int)(s / ((int64_t)bd * bc * bb));
        int a = R.a0 + ia, b = R.b0 + ib, c = R.c0 + ic, d = R.d0 + id;
        double f = q_factor(a, b, c, d);
        if (f == 0.0) continue;  // warp-uniform: the whole sub-block contributes exactly zero
        int asc[4], base[4], pos[4];
        decode_tri4(r, no, asc);
        base[0] = asc[3]; base[1] = asc[2]; base[2] = asc[1]; base[3] = asc[0];
        int64_t off = s4_lane_offset(lane, base, no, pos);
        int64_t q = (((int64_t)ia * blk + ib) * blk + ic) * blk + id;
        int i = pos[0], j = pos[1], kk = pos[2], l = pos[3];
        double zt = z4[q * n4 + off];
        double x = dadd(t4[q * n4 + off], zt);
        double neg = -dadd(dadd(dadd(ev[a], ev[b]), ev[c]), ev[d]);
        double den = dadd(dadd(dadd(eo[i], eo[j]), dadd(eo[kk], eo[l])), neg);
        x = (fabs(den) > 1e-15) ? __ddiv_rn(x, den) : 0.0;
        double y = dmul(p4_apply(x, partner, k), f);
        if (s4_first_holder(lane, off)) {
            // disconnected vvoo x t2 product (distr_cc/rccsdt_q.py:1143-1150)
#define VO(p, q_, m, n) (((int64_t)(p) * nv + (q_)) * no2 + (int64_t)(m) * no + (n))
            double zsq = vvoo[VO(a, b, i, j)] * t2[VO(c, d, kk, l)] + vvoo[VO(a, c, i, kk)] * t2[VO(b, d, j, l)] +
                         vvoo[VO(a, d, i, l)] * t2[VO(b, c, j, kk)] + vvoo[VO(b, c, j, kk)] * t2[VO(a, d, i, l)] +
                         vvoo[VO(b, d, j, l)] * t2[VO(a, c, i, kk)] + vvoo[VO(c, d, kk, l)] * t2[VO(a, b, i, j)];
#undef VO
            s_br += y * zsq;
            s_pa += y * zt;
        }
    }
    __shared__ double red[2][QE_WARPS];
    for (int o = 16; o > 0; o >>= 1) {
        s_br += __shfl_down_sync(0xffffffffu, s_br, o);
        s_pa += __shfl_down_sync(0xffffffffu, s_pa, o);
    }
    if (lane == 0) {
        red[0][threadIdx.x >> 5] = s_br;
        red[1][threadIdx.x >> 5] = s_pa;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int t = 0; t < QE_WARPS; t++) {
            x += red[0][t];
            y += red[1][t];
        }
        ws[2 * blockIdx.x] = x;
        ws[2 * blockIdx.x + 1] = y;
    }
}

// out[0] += B/12, out[1] += P/12 + B/12, summing the partials in a fixed order.
__global__ void k_q_finish(const double *ws, int64_t n, double *out) {
    __shared__ double red[2][32];
    double x = 0.0, y = 0.0;
    for (int64_t t = threadIdx.x; t < n; t += blockDim.x) {
        x += ws[2 * t];
        y += ws[2 * t + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
        x += __shfl_down_sync(0xffffffffu, x, o);
        y += __shfl_down_sync(0xffffffffu, y, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = x;
        red[1][threadIdx.x >> 5] = y;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double B = 0.0, P = 0.0;
        for (int t = 0; t < (int)(blockDim.x >> 5); t++) {
            B += red[0][t];
            P += red[1][t];
        }
        double tb = B / 12.0;
        double tp = P / 12.0 + tb;
        out[0] += tb;
        out[1] += tp;
    }
}

// ----------------------------------------------------------------- group epilogue
//
// A task group's blocks z4 (T3-connected) and t4 (T2-connected), stored
// [i][j][k][l][ia][ib][ic][id] with the virtual quadruple fastest: one warp
// takes one ijkl orbit and 32 consecutive quadruples (lanes), so every load
// of a position is one coalesced row, and each lane holds its quadruple's 24
// orbit values in registers.  The P4 stages then read partners at compile-time
// register indices; per position the arithmetic is the task epilogue's
// expression, term for term.

// p[m] of the lexicographic permutation l of {0,1,2,3}
__host__ __device__ constexpr int perm4_at(int l, int m) {
    int avail[4] = {0, 1, 2, 3}, p[4] = {0, 0, 0, 0}, f[3] = {6, 2, 1}, n = 4;
    for (int s = 0; s < 3; s++) {
        const int q = l / f[s];
        l %= f[s];
        p[s] = avail[q];
        for (int t = q; t < n - 1; t++) avail[t] = avail[t + 1];
        n--;
    }
    p[3] = avail[0];
    return p[m];
}

// lane of the permutation l with slots of transposition s (ab, ac, ad, bc, bd, cd) swapped
__host__ __device__ constexpr int partner4(int l, int s) {
    int q[4] = {perm4_at(l, 0), perm4_at(l, 1), perm4_at(l, 2), perm4_at(l, 3)};
    const int i = (s < 3) ? 0 : (s < 5 ? 1 : 2), j = (s < 3) ? s + 1 : (s < 5 ? s - 1 : 3);
    const int t = q[i];
    q[i] = q[j];
    q[j] = t;
    int r = 0, f[3] = {6, 2, 1};
    for (int m = 0; m < 3; m++) {
        int smaller = 0;
        for (int u = m + 1; u < 4; u++) smaller += q[u] < q[m];
        r += smaller * f[m];
    }
    return r;
}

template <int S>
__device__ __forceinline__ double p4_t1_at(const double (&x)[24], const P4Coef &k) {
    constexpr int ab = partner4(S, 0), ac = partner4(S, 1), ad = partner4(S, 2);
    return dadd(dadd(dadd(dmul(k.p[0], x[S]), dmul(k.p[1], x[ab])), dmul(k.p[2], x[ac])), dmul(k.p[3], x[ad]));
}
template <int S>
__device__ __forceinline__ double p4_t2_at(const double (&t1)[24], const P4Coef &k) {
    constexpr int bc = partner4(S, 3), bd = partner4(S, 4);
    return dadd(dadd(dmul(k.p[4], t1[S]), dmul(k.p[5], t1[bc])), dmul(k.p[6], t1[bd]));
}
// R without its beta term (beta = 0 for P4_444: beta * x adds a signed zero only)
template <int S>
__device__ __forceinline__ double p4_r0_at(const double (&t2)[24], const P4Coef &k) {
    constexpr int cd = partner4(S, 5);
    return dmul(k.alpha, dadd(dmul(k.p[7], t2[S]), dmul(k.p[8], t2[cd])));
}
template <int... S>
__device__ __forceinline__ void p4_t1_all(const double (&x)[24], double (&t1)[24], const P4Coef &k,
                                          std::integer_sequence<int, S...>) {
    ((t1[S] = p4_t1_at<S>(x, k)), ...);
}
template <int... S>
__device__ __forceinline__ void p4_t2_all(const double (&t1)[24], double (&t2)[24], const P4Coef &k,
                                          std::integer_sequence<int, S...>) {
    ((t2[S] = p4_t2_at<S>(t1, k)), ...);
}
template <int... S>
__device__ __forceinline__ void p4_r0_all(const double (&t2)[24], double (&r)[24], const P4Coef &k,
                                          std::integer_sequence<int, S...>) {
    ((r[S] = p4_r0_at<S>(t2, k)), ...);
}

struct QGroup {
    int a0, b0, c0, d0, ba, bb, bc, dn;
};

constexpr int QG_THREADS = 128;
constexpr int QG_WARPS = QG_THREADS / 32;

__device__ __forceinline__ double q_load(const double *p) { return __ldcs(p); }
__device__ __forceinline__ double q_load(const float *p) { return (double)__ldcs(p); }

// vvooT / t2T: [x][p][q][y] = vvoo / t2 [x][y][p][q] (second virtual fastest).
template <typename T>
__global__ void __launch_bounds__(QG_THREADS, 4) k_q_group_epilogue(const T *t4, const T *z4, const double *vvooT,
                                                                 const double *t2T, const double *eo, const double *ev,
                                                                 QGroup g, int no, int nv, int64_t norb, P4Coef k,
                                                                 double *ws) {
    const int lane = threadIdx.x & 31;
    const int64_t V = (int64_t)g.ba * g.bb * g.bc * g.dn;
    const int64_t nchunk = (V + 31) / 32, total = norb * nchunk;
    double s_br = 0.0, s_pa = 0.0;
    for (int64_t w = (int64_t)blockIdx.x * QG_WARPS + (threadIdx.x >> 5); w < total;
         w += (int64_t)gridDim.x * QG_WARPS) {
        const int64_t r = w / nchunk, v = (w % nchunk) * 32 + lane;
        // orbit positions: lane s < 24 computes position s, then all lanes take them by shuffle
        int asc[4], base[4], pos[4];
        decode_tri4(r, no, asc);
        base[0] = asc[3];
        base[1] = asc[2];
        base[2] = asc[1];
        base[3] = asc[0];
        const int64_t my_off = s4_lane_offset(lane, base, no, pos);
        const unsigned first = __ballot_sync(0xffffffffu, s4_first_holder(lane, my_off));
        const int my_pos = pos[0] | (pos[1] << 8) | (pos[2] << 16) | (pos[3] << 24);
        double my_eo = dadd(dadd(eo[pos[0]], eo[pos[1]]), dadd(eo[pos[2]], eo[pos[3]]));
        const bool valid = v < V;
        const int64_t vv = valid ? v : 0;
        const int id = (int)(vv % g.dn), ic = (int)((vv / g.dn) % g.bc), ib = (int)((vv / ((int64_t)g.dn * g.bc)) % g.bb),
                  ia = (int)(vv / ((int64_t)g.dn * g.bc * g.bb));
        const int a = g.a0 + ia, b = g.b0 + ib, c = g.c0 + ic, d = g.d0 + id;
        const double f = valid ? q_factor(a, b, c, d) : 0.0;
        const double neg = -dadd(dadd(dadd(ev[a], ev[b]), ev[c]), ev[d]);
        double x[24], t1[24];
#pragma unroll
        for (int s = 0; s < 24; s++) {
            const int ps = __shfl_sync(0xffffffffu, my_pos, s);
            const double eos = __shfl_sync(0xffffffffu, my_eo, s);
            const int64_t off = (((int64_t)(ps & 255) * no + ((ps >> 8) & 255)) * no + ((ps >> 16) & 255)) * no +
                                (ps >> 24);
            double xv = 0.0;
            if (f != 0.0) {
                xv = dadd(q_load(t4 + off * V + vv), q_load(z4 + off * V + vv));
                const double den = dadd(eos, neg);
                xv = (fabs(den) > 1e-15) ? __ddiv_rn(xv, den) : 0.0;
            }
            x[s] = xv;
        }
        // x -> T1 (t1) -> T2 (into x) -> R (into t1): two arrays of 24 live at a time
        p4_t1_all(x, t1, k, std::make_integer_sequence<int, 24>{});
        p4_t2_all(t1, x, k, std::make_integer_sequence<int, 24>{});
        p4_r0_all(x, t1, k, std::make_integer_sequence<int, 24>{});
#pragma unroll
        for (int s = 0; s < 24; s++) {
            if (!((first >> s) & 1u)) continue;  // a repeated position counts once (warp-uniform)
            const int ps = __shfl_sync(0xffffffffu, my_pos, s);
            if (f == 0.0) continue;
            const int i = ps & 255, j = (ps >> 8) & 255, kk = (ps >> 16) & 255, l = ps >> 24;
            const int64_t off = (((int64_t)i * no + j) * no + kk) * no + l;
            const double y = dmul(t1[s], f);
#define VT(p, m, n, q_) ((((int64_t)(p) * no + (m)) * no + (n)) * nv + (q_))
            const double zsq = vvooT[VT(a, i, j, b)] * t2T[VT(c, kk, l, d)] + vvooT[VT(a, i, kk, c)] * t2T[VT(b, j, l, d)] +
                               vvooT[VT(a, i, l, d)] * t2T[VT(b, j, kk, c)] + vvooT[VT(b, j, kk, c)] * t2T[VT(a, i, l, d)] +
                               vvooT[VT(b, j, l, d)] * t2T[VT(a, i, kk, c)] + vvooT[VT(c, kk, l, d)] * t2T[VT(a, i, j, b)];
#undef VT
            s_br += y * zsq;
            s_pa += y * q_load(z4 + off * V + vv);
        }
    }
    __shared__ double red[2][QG_WARPS];
    for (int o = 16; o > 0; o >>= 1) {
        s_br += __shfl_down_sync(0xffffffffu, s_br, o);
        s_pa += __shfl_down_sync(0xffffffffu, s_pa, o);
    }
    if (lane == 0) {
        red[0][threadIdx.x >> 5] = s_br;
        red[1][threadIdx.x >> 5] = s_pa;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int t = 0; t < QG_WARPS; t++) {
            x += red[0][t];
            y += red[1][t];
        }
        ws[2 * blockIdx.x] = x;
        ws[2 * blockIdx.x + 1] = y;
    }
}

// Adjoint of the group epilogue for the cotangents (gb, gp) of ([Q], (Q)).  With
// X = (t4 + z4) / D, Y = f P(X) and  gb [Q] + gp (Q) = sum Y (gp z4 + (gb + gp) z4sq) / 12
// over the distinct positions:
//   dX = P^T(H),  H = f (gp z4 + (gb + gp) z4sq) / 12
//   gt4 = dX / D,  gz4 = dX / D + gp f P(X) / 12,  gz4sq = (gb + gp) f P(X) / 12
// P^T applies the same three stages in reverse order (each transposition is its
// own transpose); on an orbit with repeated positions the slot values stay equal
// per position, so the value at a position's first slot is the adjoint there.
// Every position of the group is written exactly once (zero where f = 0).
__global__ void __launch_bounds__(QG_THREADS) k_q_group_epilogue_adj(const double *t4, const double *z4,
                                                                     const double *vvooT, const double *t2T,
                                                                     const double *eo, const double *ev, QGroup g,
                                                                     int no, int nv, int64_t norb, P4Coef k,
                                                                     double gb, double gp, double *gt4, double *gz4,
                                                                     double *gzsq) {
    const int lane = threadIdx.x & 31;
    const int64_t V = (int64_t)g.ba * g.bb * g.bc * g.dn;
    const int64_t nchunk = (V + 31) / 32, total = norb * nchunk;
    for (int64_t w = (int64_t)blockIdx.x * QG_WARPS + (threadIdx.x >> 5); w < total;
         w += (int64_t)gridDim.x * QG_WARPS) {
        const int64_t r = w / nchunk, v = (w % nchunk) * 32 + lane;
        int asc[4], base[4], pos[4];
        decode_tri4(r, no, asc);
        base[0] = asc[3];
        base[1] = asc[2];
        base[2] = asc[1];
        base[3] = asc[0];
        const int64_t my_off = s4_lane_offset(lane, base, no, pos);
        const unsigned first = __ballot_sync(0xffffffffu, s4_first_holder(lane, my_off));
        const int my_pos = pos[0] | (pos[1] << 8) | (pos[2] << 16) | (pos[3] << 24);
        const double my_eo = dadd(dadd(eo[pos[0]], eo[pos[1]]), dadd(eo[pos[2]], eo[pos[3]]));
        const bool valid = v < V;
        const int64_t vv = valid ? v : 0;
        const int id = (int)(vv % g.dn), ic = (int)((vv / g.dn) % g.bc), ib = (int)((vv / ((int64_t)g.dn * g.bc)) % g.bb),
                  ia = (int)(vv / ((int64_t)g.dn * g.bc * g.bb));
        const int a = g.a0 + ia, b = g.b0 + ib, c = g.c0 + ic, d = g.d0 + id;
        const double f = valid ? q_factor(a, b, c, d) : 0.0;
        const double neg = -dadd(dadd(dadd(ev[a], ev[b]), ev[c]), ev[d]);
        double x[24], y[24], h[24];
#pragma unroll
        for (int s = 0; s < 24; s++) {
            const int ps = __shfl_sync(0xffffffffu, my_pos, s);
            const double eos = __shfl_sync(0xffffffffu, my_eo, s);
            const int i = ps & 255, j = (ps >> 8) & 255, kk = (ps >> 16) & 255, l = ps >> 24;
            const int64_t off = (((int64_t)i * no + j) * no + kk) * no + l;
            double xv = 0.0, hv = 0.0;
            if (f != 0.0) {
                const double zt = z4[off * V + vv];
                xv = dadd(t4[off * V + vv], zt);
                const double den = dadd(eos, neg);
                xv = (fabs(den) > 1e-15) ? __ddiv_rn(xv, den) : 0.0;
#define VT(p, m, n, q_) ((((int64_t)(p) * no + (m)) * no + (n)) * nv + (q_))
                const double zsq = vvooT[VT(a, i, j, b)] * t2T[VT(c, kk, l, d)] + vvooT[VT(a, i, kk, c)] * t2T[VT(b, j, l, d)] +
                                   vvooT[VT(a, i, l, d)] * t2T[VT(b, j, kk, c)] + vvooT[VT(b, j, kk, c)] * t2T[VT(a, i, l, d)] +
                                   vvooT[VT(b, j, l, d)] * t2T[VT(a, i, kk, c)] + vvooT[VT(c, kk, l, d)] * t2T[VT(a, i, j, b)];
#undef VT
                hv = f * (gp * zt + (gb + gp) * zsq) / 12.0;
            }
            x[s] = xv;
            h[s] = hv;
        }
        // y = P(x) (forward stages), then x <- P^T(h): R, T2, T1 in that order
        p4_t1_all(x, y, k, std::make_integer_sequence<int, 24>{});
        p4_t2_all(y, x, k, std::make_integer_sequence<int, 24>{});
        p4_r0_all(x, y, k, std::make_integer_sequence<int, 24>{});
        p4_r0_all(h, x, k, std::make_integer_sequence<int, 24>{});
        p4_t2_all(x, h, k, std::make_integer_sequence<int, 24>{});
        p4_t1_all(h, x, k, std::make_integer_sequence<int, 24>{});
#pragma unroll
        for (int s = 0; s < 24; s++) {
            if (!((first >> s) & 1u)) continue;  // warp-uniform
            const int ps = __shfl_sync(0xffffffffu, my_pos, s);
            const double eos = __shfl_sync(0xffffffffu, my_eo, s);
            if (!valid) continue;
            const int64_t off = (((int64_t)(ps & 255) * no + ((ps >> 8) & 255)) * no + ((ps >> 16) & 255)) * no +
                                (ps >> 24);
            double gx = 0.0, gy = 0.0;
            if (f != 0.0) {
                const double den = dadd(eos, neg);
                gx = (fabs(den) > 1e-15) ? x[s] / den : 0.0;
                gy = f * y[s] / 12.0;
            }
            gt4[off * V + vv] = gx;
            gz4[off * V + vv] = gx + gp * gy;
            gzsq[off * V + vv] = (gb + gp) * gy;
        }
    }
}

static unsigned q_group_grid(int64_t items) {
    int64_t g = (items + QG_WARPS - 1) / QG_WARPS;
    return (unsigned)(g < 148 * 8 ? (g ? g : 1) : 148 * 8);
}

static unsigned q_epilogue_grid(int64_t nwarps) {
    int64_t g = (nwarps + QE_WARPS - 1) / QE_WARPS;
    return (unsigned)(g < 148 * 16 ? (g ? g : 1) : 148 * 16);
}

}  // namespace dcc

using namespace dcc;

extern "C" int dcc_e_abcdijkl_division(double *r4, const double *e_occ, const double *e_vir, int64_t a0, int64_t a1,
                                       int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0, int64_t d1,
                                       int64_t blk_a, int64_t blk_b, int64_t blk_c, int64_t blk_d, int64_t nocc,
                                       void *stream) {
    clear_error();
    DCC_REQUIRE(a1 - a0 <= blk_a && b1 - b0 <= blk_b && c1 - c0 <= blk_c && d1 - d0 <= blk_d, DCC_ERR_SHAPE,
                "virtual ranges exceed the block extents");
    DCC_REQUIRE(a0 <= a1 && b0 <= b1 && c0 <= c1 && d0 <= d1 && nocc >= 0, DCC_ERR_SHAPE, "bad ranges");
    int64_t nsub = (a1 - a0) * (b1 - b0) * (c1 - c0) * (d1 - d0);
    if (nsub == 0 || nocc == 0) return DCC_OK;
    DCC_REQUIRE(r4 && e_occ && e_vir, DCC_ERR_NULL, "NULL buffer");
    int64_t n4 = nocc * nocc * nocc * nocc;
    unsigned gx = ceil_div(n4, 256);
    gx = gx > 32 ? 32 : gx;
    dim3 grid(gx, (unsigned)(nsub < 65535 ? nsub : 65535));
    QRange R{(int)a0, (int)a1, (int)b0, (int)b1, (int)c0, (int)c1, (int)d0, (int)d1};
    k_q_division<<<grid, 256, 0, as_stream(stream)>>>(r4, e_occ, e_vir, R, (int)blk_b, (int)blk_c, (int)blk_d,
                                                      (int)nocc);
    return launch_status("e_abcdijkl_division");
}

extern "C" int dcc_t4_multiply_factor(double *t4_blk, const double *factor_blk, int64_t blk_a, int64_t blk_b,
                                      int64_t blk_c, int64_t blk_d, int64_t nocc, void *stream) {
    clear_error();
    DCC_REQUIRE(blk_a >= 0 && blk_b >= 0 && blk_c >= 0 && blk_d >= 0 && nocc >= 0, DCC_ERR_SHAPE, "negative size");
    int64_t nsub = blk_a * blk_b * blk_c * blk_d, n4 = nocc * nocc * nocc * nocc;
    if (nsub == 0 || n4 == 0) return DCC_OK;
    DCC_REQUIRE(t4_blk && factor_blk, DCC_ERR_NULL, "NULL buffer");
    unsigned gx = ceil_div(n4, 256);
    gx = gx > 32 ? 32 : gx;
    dim3 grid(gx, (unsigned)(nsub < 65535 ? nsub : 65535));
    k_q_factor<<<grid, 256, 0, as_stream(stream)>>>(t4_blk, factor_blk, nsub, n4);
    return launch_status("t4_multiply_factor");
}

extern "C" size_t dcc_q_epilogue_workspace_bytes(int64_t blksize, int64_t nocc) {
    int64_t nwarps = blksize * blksize * blksize * blksize * binom(nocc + 3, 4);
    return (size_t)q_epilogue_grid(nwarps) * 2 * sizeof(double);
}

extern "C" int dcc_q_task_epilogue(const double *t4, const double *z4, const double *eris_vvoo,
                                   const double *t2_vvoo, const double *e_occ, const double *e_vir, int64_t a0,
                                   int64_t a1, int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0,
                                   int64_t d1, int64_t blksize, int64_t nocc, int64_t nvir, double *out,
                                   void *workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    DCC_REQUIRE(0 <= a0 && a0 <= a1 && a1 <= nvir && 0 <= b0 && b0 <= b1 && b1 <= nvir && 0 <= c0 && c0 <= c1 &&
                    c1 <= nvir && 0 <= d0 && d0 <= d1 && d1 <= nvir,
                DCC_ERR_SHAPE, "virtual range out of bounds");
    DCC_REQUIRE(a1 - a0 <= blksize && b1 - b0 <= blksize && c1 - c0 <= blksize && d1 - d0 <= blksize,
                DCC_ERR_SHAPE, "range longer than blksize");
    DCC_REQUIRE(t4 && z4 && eris_vvoo && t2_vvoo && e_occ && e_vir && out && workspace, DCC_ERR_NULL,
                "NULL buffer");
    size_t need = dcc_q_epilogue_workspace_bytes(blksize, nocc);
    DCC_REQUIRE(workspace_bytes >= need, DCC_ERR_WORKSPACE, "workspace needs %zu bytes, got %zu", need,
                workspace_bytes);
    P4Coef k;
    int rc = p4_coef("P4_444", 1.0, 0.0, k);
    if (rc) return rc;
    int64_t norb = binom(nocc + 3, 4);
    int64_t nwarps_grid = blksize * blksize * blksize * blksize * norb;
    unsigned grid = q_epilogue_grid(nwarps_grid);
    QRange R{(int)a0, (int)a1, (int)b0, (int)b1, (int)c0, (int)c1, (int)d0, (int)d1};
    cudaStream_t st = as_stream(stream);
    k_q_epilogue<<<grid, QE_THREADS, 0, st>>>(t4, z4, eris_vvoo, t2_vvoo, e_occ, e_vir, R, (int)blksize, (int)nocc,
                                              (int)nvir, norb, k, (double *)workspace);
    rc = launch_status("q_task_epilogue");
    if (rc) return rc;
    k_q_finish<<<1, 256, 0, st>>>((const double *)workspace, grid, out);
    return launch_status("q_task_epilogue finish");
}

extern "C" size_t dcc_q_group_epilogue_workspace_bytes(void) { return (size_t)148 * 8 * 2 * sizeof(double); }

extern "C" int dcc_q_group_epilogue(const void *t4, const void *z4, int f32, const double *vvooT,
                                    const double *t2T, const double *e_occ, const double *e_vir, int64_t a0,
                                    int64_t a1, int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0,
                                    int64_t d1, int64_t nocc, int64_t nvir, double *out, void *workspace,
                                    size_t workspace_bytes, void *stream) {
    clear_error();
    DCC_REQUIRE(0 <= a0 && a0 <= a1 && a1 <= nvir && 0 <= b0 && b0 <= b1 && b1 <= nvir && 0 <= c0 && c0 <= c1 &&
                    c1 <= nvir && 0 <= d0 && d0 <= d1 && d1 <= nvir,
                DCC_ERR_SHAPE, "virtual range out of bounds");
    DCC_REQUIRE(nocc >= 1 && nocc <= 255, DCC_ERR_SHAPE, "nocc must be in [1, 255]");
    DCC_REQUIRE(f32 == 0 || f32 == 1, DCC_ERR_SHAPE, "f32 must be 0 or 1");
    DCC_REQUIRE(t4 && z4 && vvooT && t2T && e_occ && e_vir && out && workspace, DCC_ERR_NULL, "NULL buffer");
    DCC_REQUIRE(workspace_bytes >= dcc_q_group_epilogue_workspace_bytes(), DCC_ERR_WORKSPACE,
                "workspace needs %zu bytes, got %zu", dcc_q_group_epilogue_workspace_bytes(), workspace_bytes);
    const int64_t V = (a1 - a0) * (b1 - b0) * (c1 - c0) * (d1 - d0);
    if (V == 0) return DCC_OK;
    DCC_REQUIRE(V * nocc * nocc * nocc * nocc < (1ll << 40), DCC_ERR_SHAPE, "group block too large");
    P4Coef k;
    int rc = p4_coef("P4_444", 1.0, 0.0, k);  // beta = 0: the kernel drops the beta term
    if (rc) return rc;
    const int64_t norb = binom(nocc + 3, 4);
    const unsigned grid = q_group_grid(norb * ((V + 31) / 32));
    QGroup g{(int)a0, (int)b0, (int)c0, (int)d0, (int)(a1 - a0), (int)(b1 - b0), (int)(c1 - c0), (int)(d1 - d0)};
    cudaStream_t st = as_stream(stream);
    if (f32)
        k_q_group_epilogue<float><<<grid, QG_THREADS, 0, st>>>((const float *)t4, (const float *)z4, vvooT, t2T, e_occ,
                                                               e_vir, g, (int)nocc, (int)nvir, norb, k,
                                                               (double *)workspace);
    else
        k_q_group_epilogue<double><<<grid, QG_THREADS, 0, st>>>((const double *)t4, (const double *)z4, vvooT, t2T,
                                                                e_occ, e_vir, g, (int)nocc, (int)nvir, norb, k,
                                                                (double *)workspace);
    rc = launch_status("q_group_epilogue");
    if (rc) return rc;
    k_q_finish<<<1, 256, 0, st>>>((const double *)workspace, grid, out);
    return launch_status("q_group_epilogue finish");
}

extern "C" int dcc_q_group_epilogue_adjoint(const double *t4, const double *z4, const double *vvooT,
                                            const double *t2T, const double *e_occ, const double *e_vir, int64_t a0,
                                            int64_t a1, int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0,
                                            int64_t d1, int64_t nocc, int64_t nvir, double g_bracket, double g_paren,
                                            double *gt4, double *gz4, double *gz4sq, void *stream) {
    clear_error();
    DCC_REQUIRE(0 <= a0 && a0 <= a1 && a1 <= nvir && 0 <= b0 && b0 <= b1 && b1 <= nvir && 0 <= c0 && c0 <= c1 &&
                    c1 <= nvir && 0 <= d0 && d0 <= d1 && d1 <= nvir,
                DCC_ERR_SHAPE, "virtual range out of bounds");
    DCC_REQUIRE(nocc >= 1 && nocc <= 255, DCC_ERR_SHAPE, "nocc must be in [1, 255]");
    DCC_REQUIRE(t4 && z4 && vvooT && t2T && e_occ && e_vir && gt4 && gz4 && gz4sq, DCC_ERR_NULL, "NULL buffer");
    const int64_t V = (a1 - a0) * (b1 - b0) * (c1 - c0) * (d1 - d0);
    if (V == 0) return DCC_OK;
    DCC_REQUIRE(V * nocc * nocc * nocc * nocc < (1ll << 40), DCC_ERR_SHAPE, "group block too large");
    P4Coef k;
    int rc = p4_coef("P4_444", 1.0, 0.0, k);
    if (rc) return rc;
    const int64_t norb = binom(nocc + 3, 4);
    const unsigned grid = q_group_grid(norb * ((V + 31) / 32));
    QGroup g{(int)a0, (int)b0, (int)c0, (int)d0, (int)(a1 - a0), (int)(b1 - b0), (int)(c1 - c0), (int)(d1 - d0)};
    k_q_group_epilogue_adj<<<grid, QG_THREADS, 0, as_stream(stream)>>>(t4, z4, vvooT, t2T, e_occ, e_vir, g, (int)nocc,
                                                                      (int)nvir, norb, k, g_bracket, g_paren, gt4,
                                                                      gz4, gz4sq);
    return launch_status("q_group_epilogue_adjoint");
}
