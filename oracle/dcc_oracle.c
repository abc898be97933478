/*
 * dcc_oracle.c -- TEST ORACLE ONLY.
 *
 * A plain, scalar, single-threaded C restatement of the bandwidth-bound helpers
 * of Distributed-CC's triples/quadruples path.  It is the checker that the CUDA
 * library is compared against (tests, smoke check, timed CPU baseline); nothing
 * in the shipped library links or calls it.
 *
 * Every kernel is written in an element-wise form: the value written at a
 * position is a fixed expression over the tensor values at permutations of
 * that position.  The expressions keep the operation order of the reference C
 * code built with its default flags (ISO C11, -O3, no -march=native, hence no
 * contraction of a*b+c into FMA), so results agree bit for bit with it.  This
 * file is pinned against the reference library itself by tests/test_oracle_pin.py.
 *
 * Reference behaviour restated (paths relative to the Distributed-CC project):
 *   src/rccsdt.c   : take_t3_ijk_single_ (32-129), t3_single_spin_summation_inplace_
 *                    (131-233), t3_spin_summation_triple_sym_ (245-310),
 *                    t3_transpose_add_ (320-375), fill_local_data_ijk_ (105-117),
 *                    IJK->ABC record pack/unpack (386-561)
 *   src/rccsdt_q.c : t4_spin_summation_inplace_ (33-472), e_abcdijkl_division_
 *                    (474-588), t4_multiply_factor_ (590-650),
 *                    fill_t3_from_ptr_array (655-828)
 *   src/rccsdtq.c  : t4_project_1_minus_p4_p31_inplace_ (63-308),
 *                    t4_single_spin_summation_inplace_ (316-916),
 *                    ijkl maps + unpack_t4_ijkl_single_ (918-983, 1104-1125),
 *                    t4_transpose_add_ (990-1005), t4_spin_summation_quadruple_sym_
 *                    (1018-1047), r4_local_tri_divide_e_ (1055-1088)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* pattern coefficient tables                                          */
/* ------------------------------------------------------------------ */

/* P3 patterns (src/rccsdt.c:135-152): 0 = P3_full, 1 = P3_422, 2 = P3_201 */
static int p3_coeffs(int pattern, double p[5]) {
    static const double tab[3][5] = {
        {1.0, 1.0, 1.0, 1.0, 1.0},
        {2.0, -1.0, -1.0, 2.0, -1.0},
        {2.0, -1.0, -1.0, 1.0, 0.0},
    };
    if (pattern < 0 || pattern > 2) return -1;
    memcpy(p, tab[pattern], sizeof(tab[0]));
    return 0;
}

/* P4 patterns (src/rccsdt_q.c:49-85, src/rccsdtq.c:324-350):
 * 0 = P4_full, 1 = P4_444, 2 = P4_442, 3 = P4_201 */
static int p4_coeffs(int pattern, double p[9]) {
    static const double tab[4][9] = {
        {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0},
        {2.0, -1.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0, -1.0},
        {2.0, -1.0, -1.0, -1.0, 2.0, -1.0, -1.0, 1.0, 0.0},
        {2.0, -1.0, -1.0, -1.0, 1.0, 0.0, 0.0, 1.0, 0.0},
    };
    if (pattern < 0 || pattern > 3) return -1;
    memcpy(p, tab[pattern], sizeof(tab[0]));
    return 0;
}

/* ------------------------------------------------------------------ */
/* occupied-tuple index maps                                           */
/* ------------------------------------------------------------------ */

/* lexicographic rank of a canonical i<=j<=k triple among all such triples
 * (distr_cc/distribute_t3.py:51-60) */
int64_t oracle_ijk_to_linear(int64_t i, int64_t j, int64_t k, int64_t n) {
    int64_t ni = n - i;
    int64_t before_i = (n * (n + 1) * (n + 2) - ni * (ni + 1) * (ni + 2)) / 6;
    int64_t before_j = (j - i) * (2 * n - j - i + 1) / 2;
    return before_i + before_j + (k - j);
}

static int64_t choose(int64_t n, int64_t r) {
    if (n < r || n < 0) return 0;
    int64_t v = 1;
    for (int64_t t = 0; t < r; t++) v = v * (n - t) / (t + 1);
    return v;
}

/* full triangular rank of i<=j<=k<=l (src/rccsdtq.c:924-929) */
int64_t oracle_ijkl_to_linear(int64_t i, int64_t j, int64_t k, int64_t l, int64_t n) {
    return (choose(n + 3, 4) - choose(n - i + 3, 4)) + (choose(n - i + 2, 3) - choose(n - j + 2, 3)) +
           (choose(n - j + 1, 2) - choose(n - k + 1, 2)) + (l - k);
}

/* Which of the six orderings (i,j,k) is, with the sorted triple (src/rccsdt.c:41-73).
 * Returns the case number; s[] receives the sorted triple. */
static int order_case3(int64_t i, int64_t j, int64_t k, int64_t s[3]) {
    int c;
    if (i <= j && j <= k) { s[0] = i; s[1] = j; s[2] = k; c = 0; }
    else if (i <= k && k < j) { s[0] = i; s[1] = k; s[2] = j; c = 1; }
    else if (j < i && i <= k) { s[0] = j; s[1] = i; s[2] = k; c = 2; }
    else if (k < i && i <= j) { s[0] = k; s[1] = i; s[2] = j; c = 3; }
    else if (j <= k && k < i) { s[0] = j; s[1] = k; s[2] = i; c = 4; }
    else { s[0] = k; s[1] = j; s[2] = i; c = 5; }
    return c;
}

/* axis maps of the six cases: output axis m takes input axis PERM3[c][m] */
static const int PERM3[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

/* ------------------------------------------------------------------ */
/* T3 helpers                                                          */
/* ------------------------------------------------------------------ */

/* out = T3[i,j,k,:,:,:] for any ordering of (i,j,k), read from the canonical
 * block.  Element (v0,v1,v2) of the canonical block lands at
 * (v[P[0]], v[P[1]], v[P[2]]) of the output. */
int oracle_take_t3(const double *t3_local, double *out, const int64_t *ijk_to_local, int64_t i, int64_t j,
                   int64_t k, int64_t nocc, int64_t nvir) {
    int64_t s[3];
    int cs = order_case3(i, j, k, s);
    int64_t loc = ijk_to_local[oracle_ijk_to_linear(s[0], s[1], s[2], nocc)];
    if (loc < 0) return 1;
    const double *src = t3_local + loc * nvir * nvir * nvir;
    for (int64_t v0 = 0; v0 < nvir; v0++)
        for (int64_t v1 = 0; v1 < nvir; v1++)
            for (int64_t v2 = 0; v2 < nvir; v2++) {
                int64_t v[3] = {v0, v1, v2};
                out[(v[PERM3[cs][0]] * nvir + v[PERM3[cs][1]]) * nvir + v[PERM3[cs][2]]] =
                    src[(v0 * nvir + v1) * nvir + v2];
            }
    return 0;
}

/* copy requested canonical blocks into a contiguous buffer (src/rccsdt.c:105-117) */
void oracle_gather_t3(const double *t3_local, double *out, const int32_t *requests, const int64_t *ijk_to_local,
                      int64_t nreq, int64_t nvir) {
    int64_t v3 = nvir * nvir * nvir;
    for (int64_t r = 0; r < nreq; r++) {
        int64_t loc = ijk_to_local[requests[r]];
        if (loc >= 0) memcpy(out + r * v3, t3_local + loc * v3, (size_t)v3 * sizeof(double));
    }
}

#define AT3(A, x, y, z) (A)[((x)*nv + (y)) * nv + (z)]

/* A <- beta*A + alpha*P(A) on nblk blocks of nvir^3, P one of the P3 patterns.
 * For a position u=(u0,u1,u2):
 *   T(u) = p0*A(u0,u1,u2) + p1*A(u2,u1,u0) + p2*A(u1,u0,u2)
 *   R(u) = beta*A(u) + alpha*(p3*T(u) + p4*T(u0,u2,u1))
 * and for the all-equal position (a,a,a) the reference's collapsed form
 *   R = beta*A + (alpha*(p3+p4)) * ((p0+p1+p2)*A).                         */
int oracle_t3_spin_sum(double *A, int64_t nblk, int64_t nvir, int pattern, double alpha, double beta) {
    double p[5];
    if (p3_coeffs(pattern, p)) return -1;
    const int64_t nv = nvir, n3 = nvir * nvir * nvir;
    double *src = (double *)malloc((size_t)n3 * sizeof(double));
    for (int64_t b = 0; b < nblk; b++) {
        double *blk = A + b * n3;
        memcpy(src, blk, (size_t)n3 * sizeof(double));
        for (int64_t x = 0; x < nv; x++)
            for (int64_t y = 0; y < nv; y++)
                for (int64_t z = 0; z < nv; z++) {
                    double a0 = AT3(src, x, y, z);
                    if (x == y && y == z) {
                        double t = (p[0] + p[1] + p[2]) * a0;
                        AT3(blk, x, y, z) = beta * a0 + alpha * (p[3] + p[4]) * t;
                        continue;
                    }
                    double t_u = p[0] * a0 + p[1] * AT3(src, z, y, x) + p[2] * AT3(src, y, x, z);
                    /* T at (x,z,y) */
                    double t_w = p[0] * AT3(src, x, z, y) + p[1] * AT3(src, y, z, x) + p[2] * AT3(src, z, x, y);
                    AT3(blk, x, y, z) = beta * a0 + alpha * (p[3] * t_u + p[4] * t_w);
                }
    }
    free(src);
    return 0;
}

/* B0 = 2T - T_acb - T_cba, B1 = 2T - T_bac - T_acb, B2 = B0 + T_acb - T_bac
 * in the scalar operation order of src/rccsdt.c:295-305 */
void oracle_t3_triple_sym(const double *A, double *B0, double *B1, double *B2, int64_t nvir) {
    const int64_t nv = nvir;
    for (int64_t a = 0; a < nv; a++)
        for (int64_t b = 0; b < nv; b++)
            for (int64_t c = 0; c < nv; c++) {
                double t = AT3(A, a, b, c), t_bac = AT3(A, b, a, c), t_acb = AT3(A, a, c, b),
                       t_cba = AT3(A, c, b, a);
                double two = 2.0 * t;
                double d0 = two - t_acb - t_cba;
                AT3(B0, a, b, c) = d0;
                AT3(B1, a, b, c) = two - t_bac - t_acb;
                AT3(B2, a, b, c) = d0 + t_acb - t_bac;
            }
}

/* B[a,b,c] = A[a,b,c] + A[c,a,b] */
void oracle_t3_transpose_add(const double *A, double *B, int64_t nvir) {
    const int64_t nv = nvir;
    for (int64_t a = 0; a < nv; a++)
        for (int64_t b = 0; b < nv; b++)
            for (int64_t c = 0; c < nv; c++) AT3(B, a, b, c) = AT3(A, a, b, c) + AT3(A, c, a, b);
}

/* r3[q,a,b,c] /= (eia[i,a] + eia[j,b]) + eia[k,c] for the q-th canonical triple
 * (distr_cc/rccsdt.py:734-744) */
void oracle_r3_divide(double *r3, const double *eia, const int32_t *ijk, int64_t nblk, int64_t nvir) {
    const int64_t nv = nvir;
    for (int64_t q = 0; q < nblk; q++) {
        const double *ei = eia + ijk[3 * q] * nv, *ej = eia + ijk[3 * q + 1] * nv, *ek = eia + ijk[3 * q + 2] * nv;
        double *blk = r3 + q * nv * nv * nv;
        for (int64_t a = 0; a < nv; a++)
            for (int64_t b = 0; b < nv; b++)
                for (int64_t c = 0; c < nv; c++) AT3(blk, a, b, c) /= (ei[a] + ej[b]) + ek[c];
    }
}
#undef AT3

/* ------------------------------------------------------------------ */
/* T4 helpers                                                          */
/* ------------------------------------------------------------------ */

#define AT4(A, a, b, c, d) (A)[(((a)*nv + (b)) * nv + (c)) * nv + (d)]

/* A <- alpha*P(A) + beta*A on nouter blocks of nvir^4 with the factorised
 * P4 operator (p7 + p8 P_cd)(p4 + p5 P_bc + p6 P_bd)(p0 + p1 P_ab + p2 P_ac + p3 P_ad):
 *   T1(z) = p0 A(z) + p1 A(z1,z0,z2,z3) + p2 A(z2,z1,z0,z3) + p3 A(z3,z1,z2,z0)
 *   T2(y) = p4 T1(y) + p5 T1(y0,y2,y1,y3) + p6 T1(y0,y3,y2,y1)
 *   R(x)  = alpha*(p7 T2(x) + p8 T2(x0,x1,x3,x2)) + beta*A(x)               */
static double p4_t1(const double *A, int64_t nv, const double *p, int64_t z0, int64_t z1, int64_t z2, int64_t z3) {
    return p[0] * AT4(A, z0, z1, z2, z3) + p[1] * AT4(A, z1, z0, z2, z3) + p[2] * AT4(A, z2, z1, z0, z3) +
           p[3] * AT4(A, z3, z1, z2, z0);
}
static double p4_t2(const double *A, int64_t nv, const double *p, int64_t y0, int64_t y1, int64_t y2, int64_t y3) {
    return p[4] * p4_t1(A, nv, p, y0, y1, y2, y3) + p[5] * p4_t1(A, nv, p, y0, y2, y1, y3) +
           p[6] * p4_t1(A, nv, p, y0, y3, y2, y1);
}
int oracle_t4_spin_sum(double *A, int64_t nouter, int64_t nvir, int pattern, double alpha, double beta) {
    double p[9];
    if (p4_coeffs(pattern, p)) return -1;
    const int64_t nv = nvir, n4 = nv * nv * nv * nv;
    double *src = (double *)malloc((size_t)n4 * sizeof(double));
    for (int64_t o = 0; o < nouter; o++) {
        double *blk = A + o * n4;
        memcpy(src, blk, (size_t)n4 * sizeof(double));
        for (int64_t a = 0; a < nv; a++)
            for (int64_t b = 0; b < nv; b++)
                for (int64_t c = 0; c < nv; c++)
                    for (int64_t d = 0; d < nv; d++) {
                        double u = p4_t2(src, nv, p, a, b, c, d), w = p4_t2(src, nv, p, a, b, d, c);
                        AT4(blk, a, b, c, d) = alpha * (p[7] * u + p[8] * w) + beta * AT4(src, a, b, c, d);
                    }
    }
    free(src);
    return 0;
}

/* Q = (Omega-6)(Omega-2)(2 Omega^2 + 19 Omega + 48)/576 with Omega the sum of
 * the six transpositions of the four virtual axes; A <- beta*A + alpha*Q(A).
 * Evaluated per orbit of positions under S4, in the reference's stage order:
 *   x1 = Omega x - 6x, x2 = Omega x1 - 2 x1, x3 = Omega x2, x4 = Omega x3,
 *   y = (2 x4 + 19 x3 + 48 x2)/576, out = beta x + alpha y.
 * Omega sums the six swapped positions in the order ab, ac, ad, bc, bd, cd. */
static const int SWAP_PAIRS[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
static const int PERM4[24][4] = {
    {0, 1, 2, 3}, {0, 1, 3, 2}, {0, 2, 1, 3}, {0, 2, 3, 1}, {0, 3, 1, 2}, {0, 3, 2, 1}, {1, 0, 2, 3}, {1, 0, 3, 2},
    {1, 2, 0, 3}, {1, 2, 3, 0}, {1, 3, 0, 2}, {1, 3, 2, 0}, {2, 0, 1, 3}, {2, 0, 3, 1}, {2, 1, 0, 3}, {2, 1, 3, 0},
    {2, 3, 0, 1}, {2, 3, 1, 0}, {3, 0, 1, 2}, {3, 0, 2, 1}, {3, 1, 0, 2}, {3, 1, 2, 0}, {3, 2, 0, 1}, {3, 2, 1, 0},
};

static void omega_stage(const double *x, double *y, int nbr[24][6]) {
    for (int p = 0; p < 24; p++) {
        double s = x[nbr[p][0]];
        for (int t = 1; t < 6; t++) s = s + x[nbr[p][t]];
        y[p] = s;
    }
}

void oracle_t4_project(double *A, int64_t nouter, int64_t nvir, double alpha, double beta) {
    const int64_t nv = nvir, n4 = nv * nv * nv * nv;
    for (int64_t o = 0; o < nouter; o++) {
        double *blk = A + o * n4;
        for (int64_t a = 0; a < nv; a++)
            for (int64_t b = 0; b <= a; b++)
                for (int64_t c = 0; c <= b; c++)
                    for (int64_t d = 0; d <= c; d++) {
                        int64_t base[4] = {a, b, c, d}, pos[24][4], off[24];
                        int nbr[24][6];
                        for (int p = 0; p < 24; p++) {
                            for (int m = 0; m < 4; m++) pos[p][m] = base[PERM4[p][m]];
                            off[p] = ((pos[p][0] * nv + pos[p][1]) * nv + pos[p][2]) * nv + pos[p][3];
                        }
                        /* neighbour under each swap: any slot holding the swapped position */
                        for (int p = 0; p < 24; p++)
                            for (int s = 0; s < 6; s++) {
                                int64_t t[4] = {pos[p][0], pos[p][1], pos[p][2], pos[p][3]};
                                int64_t tmp = t[SWAP_PAIRS[s][0]];
                                t[SWAP_PAIRS[s][0]] = t[SWAP_PAIRS[s][1]];
                                t[SWAP_PAIRS[s][1]] = tmp;
                                int64_t toff = ((t[0] * nv + t[1]) * nv + t[2]) * nv + t[3];
                                int q = 0;
                                while (off[q] != toff) q++;
                                nbr[p][s] = q;
                            }
                        double x[24], x1[24], x2[24], x3[24], x4[24], om[24];
                        for (int p = 0; p < 24; p++) x[p] = blk[off[p]];
                        omega_stage(x, om, nbr);
                        for (int p = 0; p < 24; p++) x1[p] = om[p] - 6.0 * x[p];
                        omega_stage(x1, om, nbr);
                        for (int p = 0; p < 24; p++) x2[p] = om[p] - 2.0 * x1[p];
                        omega_stage(x2, x3, nbr);
                        omega_stage(x3, x4, nbr);
                        for (int p = 0; p < 24; p++) {
                            double y = (2.0 * x4[p] + 19.0 * x3[p] + 48.0 * x2[p]) / 576.0;
                            blk[off[p]] = beta * x[p] + alpha * y;
                        }
                    }
    }
}

/* dst = src + src[c,a,b,d] + src[d,a,c,b] (src/rccsdtq.c:990-1005) */
void oracle_t4_transpose_add(const double *src, double *dst, int64_t nvir) {
    const int64_t nv = nvir;
    for (int64_t a = 0; a < nv; a++)
        for (int64_t b = 0; b < nv; b++)
            for (int64_t c = 0; c < nv; c++)
                for (int64_t d = 0; d < nv; d++)
                    AT4(dst, a, b, c, d) = AT4(src, a, b, c, d) + AT4(src, c, a, b, d) + AT4(src, d, a, c, b);
}

/* four P4_201 variants (src/rccsdtq.c:1018-1047) */
void oracle_t4_quadruple_sym(const double *src, double *B0, double *B1, double *B2, double *B3, int64_t nvir) {
    const int64_t nv = nvir;
    for (int64_t a = 0; a < nv; a++)
        for (int64_t b = 0; b < nv; b++)
            for (int64_t c = 0; c < nv; c++)
                for (int64_t d = 0; d < nv; d++) {
                    double two = 2.0 * AT4(src, a, b, c, d);
                    double bacd = AT4(src, b, a, c, d), cbad = AT4(src, c, b, a, d), dbca = AT4(src, d, b, c, a);
                    double acbd = AT4(src, a, c, b, d), adcb = AT4(src, a, d, c, b), abdc = AT4(src, a, b, d, c);
                    AT4(B0, a, b, c, d) = two - dbca - adcb - abdc;
                    AT4(B1, a, b, c, d) = two - cbad - acbd - abdc;
                    AT4(B2, a, b, c, d) = two - bacd - acbd - adcb;
                    AT4(B3, a, b, c, d) = two - bacd - cbad - dbca;
                }
}

/* r4[q] /= ((eia[i,a] + eia[j,b]) + eia[k,c]) + eia[l,d] (src/rccsdtq.c:1055-1088) */
void oracle_r4_divide(double *r4, const double *eia, const int32_t *ijkl, int64_t nlocal, int64_t nvir) {
    const int64_t nv = nvir;
    for (int64_t q = 0; q < nlocal; q++) {
        const double *ei = eia + ijkl[4 * q] * nv, *ej = eia + ijkl[4 * q + 1] * nv,
                     *ek = eia + ijkl[4 * q + 2] * nv, *el = eia + ijkl[4 * q + 3] * nv;
        double *blk = r4 + q * nv * nv * nv * nv;
        for (int64_t a = 0; a < nv; a++)
            for (int64_t b = 0; b < nv; b++)
                for (int64_t c = 0; c < nv; c++) {
                    double e3 = (ei[a] + ej[b]) + ek[c];
                    for (int64_t d = 0; d < nv; d++) AT4(blk, a, b, c, d) /= e3 + el[d];
                }
    }
}

/* Stable sort of (i,j,k,l): sorted values and, per output axis, the source axis
 * (src/rccsdtq.c:931-960). */
static void sort4_stable(const int64_t v[4], int64_t sorted[4], int64_t axis_from[4]) {
    int64_t val[4] = {v[0], v[1], v[2], v[3]}, pos[4] = {0, 1, 2, 3};
    for (int a = 1; a < 4; a++)
        for (int b = a; b > 0 && val[b - 1] > val[b]; b--) {
            int64_t t = val[b]; val[b] = val[b - 1]; val[b - 1] = t;
            t = pos[b]; pos[b] = pos[b - 1]; pos[b - 1] = t;
        }
    for (int m = 0; m < 4; m++) sorted[m] = val[m];
    /* axis_from[dst] = the sorted slot that came from input axis dst */
    for (int d = 0; d < 4; d++)
        for (int s = 0; s < 4; s++)
            if (pos[s] == d) { axis_from[d] = s; break; }
}

/* T4[i,j,k,l,:,:,:,:] for any ordering from the canonical stored block; the
 * zero-rule blocks (i=j=k or j=k=l after sorting) come back as zeros.
 * Returns 1 when the canonical block is not stored locally (nothing written). */
int oracle_unpack_t4(const double *t4_local, double *out, const int64_t *ijkl_to_local, int64_t i, int64_t j,
                     int64_t k, int64_t l, int64_t nocc, int64_t nvir) {
    const int64_t nv = nvir, n4 = nv * nv * nv * nv;
    int64_t in[4] = {i, j, k, l}, s[4], ax[4];
    sort4_stable(in, s, ax);
    if ((s[0] == s[1] && s[1] == s[2]) || (s[1] == s[2] && s[2] == s[3])) {
        memset(out, 0, (size_t)n4 * sizeof(double));
        return 0;
    }
    int64_t loc = ijkl_to_local[oracle_ijkl_to_linear(s[0], s[1], s[2], s[3], nocc)];
    if (loc < 0) return 1;
    const double *src = t4_local + loc * n4;
    for (int64_t a = 0; a < nv; a++)
        for (int64_t b = 0; b < nv; b++)
            for (int64_t c = 0; c < nv; c++)
                for (int64_t d = 0; d < nv; d++) {
                    int64_t v[4] = {a, b, c, d};
                    AT4(out, v[ax[0]], v[ax[1]], v[ax[2]], v[ax[3]]) = AT4(src, a, b, c, d);
                }
    return 0;
}
#undef AT4

/* ------------------------------------------------------------------ */
/* (Q) helpers                                                         */
/* ------------------------------------------------------------------ */

/* r4[abcd block][ijkl] /= D with D = ((e_i+e_j) + (e_k+e_l)) + (-(((e_a+e_b)+e_c)+e_d)),
 * set to zero where |D| <= 1e-15 (src/rccsdt_q.c:474-588) */
void oracle_e_abcdijkl_division(double *r4, const double *e_occ, const double *e_vir, int64_t a0, int64_t a1,
                                int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0, int64_t d1,
                                int64_t blk_b, int64_t blk_c, int64_t blk_d, int64_t nocc) {
    const int64_t n = nocc, n4 = n * n * n * n;
    for (int64_t a = a0; a < a1; a++)
        for (int64_t b = b0; b < b1; b++)
            for (int64_t c = c0; c < c1; c++)
                for (int64_t d = d0; d < d1; d++) {
                    double neg = -(e_vir[a] + e_vir[b] + e_vir[c] + e_vir[d]);
                    double *blk = r4 + ((((a - a0) * blk_b + (b - b0)) * blk_c + (c - c0)) * blk_d + (d - d0)) * n4;
                    for (int64_t i = 0; i < n; i++)
                        for (int64_t j = 0; j < n; j++)
                            for (int64_t k = 0; k < n; k++)
                                for (int64_t l = 0; l < n; l++) {
                                    double e = (e_occ[i] + e_occ[j]) + (e_occ[k] + e_occ[l]);
                                    double den = e + neg;
                                    double *r = blk + ((i * n + j) * n + k) * n + l;
                                    *r = (fabs(den) > 1e-15) ? *r / den : 0.0;
                                }
                }
}

/* t4[abcd][:] *= factor[abcd], exact zero where factor == 0 (src/rccsdt_q.c:590-650) */
void oracle_t4_multiply_factor(double *t4, const double *factor, int64_t ba, int64_t bb, int64_t bc, int64_t bd,
                               int64_t nocc) {
    const int64_t n4 = nocc * nocc * nocc * nocc, nab = ba * bb * bc * bd;
    for (int64_t q = 0; q < nab; q++) {
        double f = factor[q];
        double *blk = t4 + q * n4;
        if (f == 0.0) { memset(blk, 0, (size_t)n4 * sizeof(double)); continue; }
        for (int64_t x = 0; x < n4; x++) blk[x] *= f;
    }
}

/* factor of a virtual quadruple (distr_cc/rccsdt_q.py:410-428) */
double oracle_q_factor(int64_t a, int64_t b, int64_t c, int64_t d) {
    if (a < b && b < c && c < d) return 24.0;
    if ((a == b && b < c && c < d) || (a < b && b == c && c < d) || (a < b && b < c && c == d)) return 12.0;
    if (a == b && b < c && c == d) return 6.0;
    return 0.0;
}

/* lexicographic rank of a<=b<=c among all such triplets (src/rccsdt_q.c:657-665) */
int64_t oracle_abc_index(int64_t a, int64_t b, int64_t c, int64_t nvir) {
    int64_t all = nvir * (nvir + 1) * (nvir + 2) / 6;
    int64_t rem = nvir - a;
    return all - rem * (rem + 1) * (rem + 2) / 6 + (b - a) * (2 * nvir - a - b + 1) / 2 + (c - b);
}

/* Ordering case of a virtual triple (a,b,c) as chosen by the reference's three
 * c-regions (src/rccsdt_q.c:690-743); s[] receives the sorted triple. */
static int abc_case(int64_t a, int64_t b, int64_t c, int64_t s[3]) {
    int64_t lo = a < b ? a : b, hi = a < b ? b : a;
    int cs;
    if (c > hi) cs = (a <= b) ? 0 : 2;
    else if (c > lo) cs = (a <= b) ? ((b <= c) ? 0 : 1) : ((a <= c) ? 2 : 4);
    else cs = (a <= b) ? ((a <= c) ? 1 : 3) : ((b <= c) ? 4 : 5);
    switch (cs) {
    case 0: s[0] = a; s[1] = b; s[2] = c; break;
    case 1: s[0] = a; s[1] = c; s[2] = b; break;
    case 2: s[0] = b; s[1] = a; s[2] = c; break;
    case 3: s[0] = c; s[1] = a; s[2] = b; break;
    case 4: s[0] = b; s[1] = c; s[2] = a; break;
    default: s[0] = c; s[1] = b; s[2] = a; break;
    }
    return cs;
}

/* target[ia,ib,c,i,j,k] (row pitch ld_b over b) from ABC-ordered storage
 * t3_abc[g][x][y][z]; the occupied axes are permuted by the virtual ordering
 * case: element (i,j,k) of the source lands at (v[P0],v[P1],v[P2]).
 * Returns the number of virtual triples whose block is absent (missing[g]!=0). */
int64_t oracle_fill_t3_abc(double *target, int64_t a0, int64_t a1, int64_t b0, int64_t b1, int64_t nvir,
                           int64_t nocc, const double *t3_abc, const uint8_t *present, int64_t ld_b) {
    const int64_t n = nocc, n3 = n * n * n;
    int64_t missing = 0;
    for (int64_t a = a0; a < a1; a++)
        for (int64_t b = b0; b < b1; b++)
            for (int64_t c = 0; c < nvir; c++) {
                int64_t s[3];
                int cs = abc_case(a, b, c, s);
                int64_t g = oracle_abc_index(s[0], s[1], s[2], nvir);
                if (present && !present[g]) { missing++; continue; }
                const double *src = t3_abc + g * n3;
                double *dst = target + (((a - a0) * ld_b + (b - b0)) * nvir + c) * n3;
                for (int64_t i = 0; i < n; i++)
                    for (int64_t j = 0; j < n; j++)
                        for (int64_t k = 0; k < n; k++) {
                            int64_t v[3] = {i, j, k};
                            dst[(v[PERM3[cs][0]] * n + v[PERM3[cs][1]]) * n + v[PERM3[cs][2]]] =
                                src[(i * n + j) * n + k];
                        }
            }
    return missing;
}

/* IJK -> ABC layout transform at one rank (distr_cc/distribute_t3.py:1544-1642 with
 * src/rccsdt.c:411-561).  Every canonical block T_ijk[a,b,c] is shipped to
 * ABC block sigma_p(a,b,c) (when that is sorted) at occupied position
 * sigma_p(i,j,k) for the six axis maps p = 0..5; where several records hit the
 * same destination the last one in the reference's record order wins, which
 * is the largest p.  Restated here as a gather: destination (g, x,y,z) reads
 * the canonical block of sorted(x,y,z) at sigma_p^{-1}(A,B,C) for the largest
 * p with sigma_p^{-1}(x,y,z) sorted. */
void oracle_ijk_to_abc(const double *t3_ijk, double *t3_abc, int64_t nocc, int64_t nvir) {
    const int64_t n = nocc, nv = nvir, n3 = n * n * n;
    int64_t g = 0;
    for (int64_t A = 0; A < nv; A++)
        for (int64_t B = A; B < nv; B++)
            for (int64_t C = B; C < nv; C++, g++) {
                int64_t tgt[3] = {A, B, C};
                for (int64_t x = 0; x < n; x++)
                    for (int64_t y = 0; y < n; y++)
                        for (int64_t z = 0; z < n; z++) {
                            int64_t xyz[3] = {x, y, z};
                            int best = -1;
                            int64_t ijk[3] = {0, 0, 0};
                            for (int p = 0; p < 6; p++) {
                                /* sigma_p(u)[m] = u[PERM3[p][m]]; invert: w[PERM3[p][m]] = xyz[m] */
                                int64_t w[3];
                                for (int m = 0; m < 3; m++) w[PERM3[p][m]] = xyz[m];
                                if (w[0] <= w[1] && w[1] <= w[2]) {
                                    best = p;
                                    ijk[0] = w[0]; ijk[1] = w[1]; ijk[2] = w[2];
                                }
                            }
                            int64_t abc[3];
                            for (int m = 0; m < 3; m++) abc[PERM3[best][m]] = tgt[m];
                            const double *blk = t3_ijk + oracle_ijk_to_linear(ijk[0], ijk[1], ijk[2], n) * nv * nv * nv;
                            t3_abc[g * n3 + (x * n + y) * n + z] = blk[(abc[0] * nv + abc[1]) * nv + abc[2]];
                        }
            }
}
