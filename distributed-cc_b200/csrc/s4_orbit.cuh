// Warp-per-orbit machinery for operators built from transpositions of four
// axes (the T4 projector 1 - P[4] - P[3,1], the P4 spin summations, and the
// P4_444 step of the (Q) loop).
//
// A warp owns one orbit of positions under S4: lane l < 24 holds the position
// base o PERM4[l] (lexicographic permutations of the four axes).  Swapping two
// slots of a lane's position lands on the position of a fixed partner lane
// (the S4 action table), whether or not the base has repeated values, so every
// stage of an operator is one shuffle per transposition and the arithmetic of
// each position is exactly the reference's per-position expression.  Lanes
// whose position repeats an earlier lane's compute identical values; only the
// first holder stores.
#pragma once

#include "dcc_common.cuh"

namespace dcc {

// slot pairs of the six transpositions, in the order ab, ac, ad, bc, bd, cd
__device__ __forceinline__ void swap_pair(int s, int &i, int &j) {
    i = (s < 3) ? 0 : (s < 5 ? 1 : 2);
    j = (s < 3) ? s + 1 : (s < 5 ? s - 1 : 3);
}

// lexicographic permutation l of {0,1,2,3}
__device__ __forceinline__ void perm4_unrank(int l, int p[4]) {
    int avail[4] = {0, 1, 2, 3};
    int f[3] = {6, 2, 1};
    int n = 4;
    for (int m = 0; m < 3; m++) {
        int q = l / f[m];
        l %= f[m];
        p[m] = avail[q];
        for (int t = q; t < n - 1; t++) avail[t] = avail[t + 1];
        n--;
    }
    p[3] = avail[0];
}

__device__ __forceinline__ int perm4_rank(const int p[4]) {
    int r = 0, f[3] = {6, 2, 1};
    for (int m = 0; m < 3; m++) {
        int smaller = 0;
        for (int t = m + 1; t < 4; t++) smaller += p[t] < p[m];
        r += smaller * f[m];
    }
    return r;
}

// partner lanes of lane `lane` under the six transpositions
__device__ __forceinline__ void s4_partners(int lane, int partner[6]) {
    int p[4];
    perm4_unrank(lane < 24 ? lane : 0, p);
    for (int s = 0; s < 6; s++) {
        int i, j, q[4] = {p[0], p[1], p[2], p[3]};
        swap_pair(s, i, j);
        int t = q[i];
        q[i] = q[j];
        q[j] = t;
        partner[s] = perm4_rank(q);
    }
}

// Non-decreasing (w0<=w1<=w2<=w3) from its lexicographic rank among n values.
__device__ __forceinline__ void decode_tri4(int64_t r, int n, int w[4]) {
    int a = 0;
    for (;; a++) {
        int64_t m = binom(n - a + 2, 3);
        if (r < m) break;
        r -= m;
    }
    int b = a;
    for (;; b++) {
        int64_t m = (int64_t)(n - b) * (n - b + 1) / 2;
        if (r < m) break;
        r -= m;
    }
    int c = b;
    for (;; c++) {
        int64_t m = n - c;
        if (r < m) break;
        r -= m;
    }
    w[0] = a;
    w[1] = b;
    w[2] = c;
    w[3] = c + (int)r;
}

// Offset of lane's position within an n^4 block for orbit base (descending).
__device__ __forceinline__ int64_t s4_lane_offset(int lane, const int base[4], int n, int pos[4]) {
    int p[4];
    perm4_unrank(lane < 24 ? lane : 0, p);
    for (int m = 0; m < 4; m++) pos[m] = base[p[m]];
    return (((int64_t)pos[0] * n + pos[1]) * n + pos[2]) * n + pos[3];
}

// Sum of the values at the six transposition partners, in the order ab..cd.
__device__ __forceinline__ double omega6(double x, const int partner[6]) {
    double s = __shfl_sync(0xffffffffu, x, partner[0]);
    for (int t = 1; t < 6; t++) s = dadd(s, __shfl_sync(0xffffffffu, x, partner[t]));
    return s;
}

struct P4Coef {
    double p[9];
    double alpha, beta;
};

// Factorised P4 operator of the reference (src/rccsdt_q.c:33-40):
//   T1(z) = p0 A(z) + p1 A(z swap ab) + p2 A(z swap ac) + p3 A(z swap ad)
//   T2(y) = p4 T1(y) + p5 T1(y swap bc) + p6 T1(y swap bd)
//   R(x)  = alpha (p7 T2(x) + p8 T2(x swap cd)) + beta A(x)
__device__ __forceinline__ double p4_apply(double x, const int partner[6], const P4Coef &k) {
    double t1 = dadd(dadd(dadd(dmul(k.p[0], x), dmul(k.p[1], __shfl_sync(0xffffffffu, x, partner[0]))),
                          dmul(k.p[2], __shfl_sync(0xffffffffu, x, partner[1]))),
                     dmul(k.p[3], __shfl_sync(0xffffffffu, x, partner[2])));
    double t2 = dadd(dadd(dmul(k.p[4], t1), dmul(k.p[5], __shfl_sync(0xffffffffu, t1, partner[3]))),
                     dmul(k.p[6], __shfl_sync(0xffffffffu, t1, partner[4])));
    return dadd(dmul(k.alpha, dadd(dmul(k.p[7], t2), dmul(k.p[8], __shfl_sync(0xffffffffu, t2, partner[5])))),
                dmul(k.beta, x));
}

// True on the first lane (of 24) holding this offset.
__device__ __forceinline__ bool s4_first_holder(int lane, int64_t off) {
    bool first = false;
    if (lane < 24) {
        unsigned peers = __match_any_sync(0x00ffffffu, (unsigned long long)off);
        first = (__ffs(peers) - 1) == lane;
    }
    return first;
}

}  // namespace dcc
