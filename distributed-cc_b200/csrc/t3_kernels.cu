// T3 kernels: P3 spin summation, triple-sym, transpose-add, block unpack /
// gather, denominator division + update + norms, IJK->ABC transform and the
// ABC block fill of the (Q) loop.
//
// The symmetrizers use "orbit tiles": the nvir^3 block is cut into 8^3 tiles,
// and one CTA owns the set of tiles {sigma(I,J,K)} for a canonical I<=J<=K
// and every axis permutation sigma.  Every position that the permutations of
// a position in that set reach lies in the same set, so a CTA reads its tiles
// once from HBM into shared memory, evaluates each output from six shared
// loads, and writes each element once: the kernel moves exactly the
// algorithmic 2 x 8 bytes per element (in place) and needs no global scratch.
#include <stdarg.h>
#include <string.h>

#include <mutex>

#include "async_util.cuh"
#include "dcc_common.cuh"

namespace dcc {

constexpr int TE = 8;            // tile edge
constexpr int TE3 = TE * TE * TE;
constexpr int SLOT = TE * 68;    // padded tile footprint in doubles
constexpr int OT_THREADS = 256;

// Conflict-free for all six axis permutations of an 8^3 tile read by 32
// consecutive (x,y,z) in row-major order (two lanes per 8-byte bank pair).
__device__ __forceinline__ int sidx(int x, int y, int z) { return x * 68 + y * 8 + ((z + y) & 7); }

// (t0 <= t1 <= t2) from its lexicographic rank among n tile indices.
__device__ __forceinline__ void decode_tri3(int64_t r, int n, int &t0, int &t1, int &t2) {
    int a = 0;
    for (;; a++) {
        int64_t m = (int64_t)(n - a) * (n - a + 1) / 2;
        if (r < m) break;
        r -= m;
    }
    int b = a;
    for (;; b++) {
        int64_t m = n - b;
        if (r < m) break;
        r -= m;
    }
    t0 = a;
    t1 = b;
    t2 = b + (int)r;
}

struct OrbitSet {
    int nslot;
    int tile[6][3];
    int nbr[6][6];  // nbr[s][pi]: slot holding axis permutation pi of slot s's tile
};

// Thread 0 builds the distinct permuted tiles of (t0,t1,t2) and the
// neighbour table; everybody waits.
__device__ void build_orbit_set(OrbitSet &os, int t0, int t1, int t2) {
    if (threadIdx.x == 0) {
        int T[3] = {t0, t1, t2};
        int n = 0;
        for (int s = 0; s < 6; s++) {
            int c[3] = {T[perm3(s, 0)], T[perm3(s, 1)], T[perm3(s, 2)]};
            bool dup = false;
            for (int q = 0; q < n; q++)
                if (os.tile[q][0] == c[0] && os.tile[q][1] == c[1] && os.tile[q][2] == c[2]) dup = true;
            if (!dup) {
                os.tile[n][0] = c[0];
                os.tile[n][1] = c[1];
                os.tile[n][2] = c[2];
                n++;
            }
        }
        os.nslot = n;
        for (int s = 0; s < n; s++)
            for (int p = 0; p < 6; p++) {
                int c[3] = {os.tile[s][perm3(p, 0)], os.tile[s][perm3(p, 1)], os.tile[s][perm3(p, 2)]};
                int q = 0;
                while (!(os.tile[q][0] == c[0] && os.tile[q][1] == c[1] && os.tile[q][2] == c[2])) q++;
                os.nbr[s][p] = q;
            }
    }
    __syncthreads();
}

// Value at axis permutation p of local position (x,y,z) in slot s; the six
// maps are 0:(x,y,z) 1:(x,z,y) 2:(y,x,z) 3:(y,z,x) 4:(z,x,y) 5:(z,y,x).
template <int P>
__device__ __forceinline__ double pv(const double *sm, const int *nbr, int x, int y, int z) {
    int o = nbr[P] * SLOT;
    if (P == 0) return sm[o + sidx(x, y, z)];
    if (P == 1) return sm[o + sidx(x, z, y)];
    if (P == 2) return sm[o + sidx(y, x, z)];
    if (P == 3) return sm[o + sidx(y, z, x)];
    if (P == 4) return sm[o + sidx(z, x, y)];
    return sm[o + sidx(z, y, x)];
}

__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async4(float *smem, const float *gmem) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}
// one element, by its size
__device__ __forceinline__ void cp_async_el(double *smem, const double *gmem) { cp_async8(smem, gmem); }
__device__ __forceinline__ void cp_async_el(float *smem, const float *gmem) { cp_async4(smem, gmem); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Issue asynchronous copies of every slot of the orbit set of block `blk`
// into `sm` (no wait): each thread has all of its loads in flight at once.
__device__ __forceinline__ void load_orbit_tiles_async(double *sm, const OrbitSet &os, const double *blk, int nv) {
    for (int s = 0; s < os.nslot; s++) {
        const int X0 = os.tile[s][0] * TE, Y0 = os.tile[s][1] * TE, Z0 = os.tile[s][2] * TE;
        for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
            int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
            int gx = X0 + x, gy = Y0 + y, gz = Z0 + z;
            if (gx < nv && gy < nv && gz < nv) cp_async8(sm + s * SLOT + sidx(x, y, z), blk + ((int64_t)gx * nv + gy) * nv + gz);
        }
    }
}

struct P3Coef {
    double p0, p1, p2, p3, p4, alpha, beta, p012, ap34;
};

// comp6(X, s): the axis map equal to "s, then X" (X(s(u)) = comp6(X, s)(u)),
// i.e. the table {0,1,2,3,4,5}, {1,0,3,2,5,4}, {2,4,0,5,1,3}, {3,5,1,4,0,2},
// {4,2,5,0,3,1}, {5,3,4,1,2,0}.  constexpr, so that with unrolled s the
// register-array indices it yields are compile-time constants.
__host__ __device__ constexpr int comp6(int X, int s) {
    return X == 0 ? (s == 0 ? 0 : (s == 1 ? 1 : (s == 2 ? 2 : (s == 3 ? 3 : (s == 4 ? 4 : (5)))))) : (X == 1 ? (s == 0 ? 1 : (s == 1 ? 0 : (s == 2 ? 3 : (s == 3 ? 2 : (s == 4 ? 5 : (4)))))) : (X == 2 ? (s == 0 ? 2 : (s == 1 ? 4 : (s == 2 ? 0 : (s == 3 ? 5 : (s == 4 ? 1 : (3)))))) : (X == 3 ? (s == 0 ? 3 : (s == 1 ? 5 : (s == 2 ? 1 : (s == 3 ? 4 : (s == 4 ? 0 : (2)))))) : (X == 4 ? (s == 0 ? 4 : (s == 1 ? 2 : (s == 2 ? 5 : (s == 3 ? 0 : (s == 4 ? 3 : (1)))))) : (s == 0 ? 5 : (s == 1 ? 3 : (s == 2 ? 4 : (s == 3 ? 1 : (s == 4 ? 2 : (0))))))))));
}

// P3 spin summation of a whole orbit set in shared memory, in place.  Each
// thread takes canonical positions u (global u0 <= u1 <= u2, all inside slot
// 0), reads the six values v[s] = A(s(u)) once and writes the six results
//   R(w) = beta A(w) + alpha (p3 T(w) + p4 T(w0,w2,w1)),
//   T(w) = p0 A(w) + p1 A(w2,w1,w0) + p2 A(w1,w0,w2),     w = s(u),
// which read only values of the same orbit; positions that coincide (equal
// indices) get identical values from the same thread.
__device__ __forceinline__ void p3_orbits_inplace(double *buf, const OrbitSet &os, int t0, int t1, int t2, int nv,
                                                  const P3Coef &k) {
    const int *nbr = os.nbr[0];
    for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
        const int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        const int gx = t0 * TE + x, gy = t1 * TE + y, gz = t2 * TE + z;
        if (gx >= nv || gy >= nv || gz >= nv) continue;
        if ((t0 == t1 && x > y) || (t1 == t2 && y > z)) continue;  // not canonical
        int a[6];
        a[0] = nbr[0] * SLOT + sidx(x, y, z);
        a[1] = nbr[1] * SLOT + sidx(x, z, y);
        a[2] = nbr[2] * SLOT + sidx(y, x, z);
        a[3] = nbr[3] * SLOT + sidx(y, z, x);
        a[4] = nbr[4] * SLOT + sidx(z, x, y);
        a[5] = nbr[5] * SLOT + sidx(z, y, x);
        double v[6];
#pragma unroll
        for (int q = 0; q < 6; q++) v[q] = buf[a[q]];
        if (gx == gy && gy == gz) {
            buf[a[0]] = dadd(dmul(k.beta, v[0]), dmul(k.ap34, dmul(k.p012, v[0])));
            continue;
        }
        double r[6];
#pragma unroll
        for (int q = 0; q < 6; q++) {
            double tu = dadd(dadd(dmul(k.p0, v[q]), dmul(k.p1, v[comp6(5, q)])), dmul(k.p2, v[comp6(2, q)]));
            double tw = dadd(dadd(dmul(k.p0, v[comp6(1, q)]), dmul(k.p1, v[comp6(3, q)])), dmul(k.p2, v[comp6(4, q)]));
            r[q] = dadd(dmul(k.beta, v[q]), dmul(k.alpha, dadd(dmul(k.p3, tu), dmul(k.p4, tw))));
        }
#pragma unroll
        for (int q = 0; q < 6; q++) buf[a[q]] = r[q];
    }
}

// Coalesced store of every slot of an orbit set from shared memory.
__device__ __forceinline__ void store_orbit_tiles(double *blk, const double *buf, const OrbitSet &os, int nv) {
    for (int s = 0; s < os.nslot; s++) {
        const int X0 = os.tile[s][0] * TE, Y0 = os.tile[s][1] * TE, Z0 = os.tile[s][2] * TE;
        for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
            int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
            int gx = X0 + x, gy = Y0 + y, gz = Z0 + z;
            if (gx < nv && gy < nv && gz < nv) blk[((int64_t)gx * nv + gy) * nv + gz] = buf[s * SLOT + sidx(x, y, z)];
        }
    }
}

// Orbit-tile kernel.  MODE 0: P3 spin summation in place (out0 == in).
// MODE 1: triple-sym (out0..out2).  MODE 2: transpose-add (out0).
// Each CTA owns one canonical tile triple and walks the blocks
// b = blockIdx.y, blockIdx.y + gridDim.y, ...; the copies of block b+gridDim.y
// are in flight (double buffer) while block b is evaluated and stored.
template <int MODE>
__global__ void __launch_bounds__(OT_THREADS) k_orbit3(const double *in, double *out0, double *out1, double *out2,
                                                       int64_t nblocks, int nv, int ntile, P3Coef k) {
    extern __shared__ double sm[];  // 2 x 6 x SLOT doubles
    __shared__ OrbitSet os;
    int t0, t1, t2;
    decode_tri3(blockIdx.x, ntile, t0, t1, t2);
    build_orbit_set(os, t0, t1, t2);
    const int64_t n3 = (int64_t)nv * nv * nv;
    int64_t b = blockIdx.y;
    if (b >= nblocks) return;
    load_orbit_tiles_async(sm, os, in + b * n3, nv);
    cp_async_commit();
    for (int stage = 0; b < nblocks; b += gridDim.y, stage ^= 1) {
        const int64_t nb = b + gridDim.y;
        if (nb < nblocks) {
            load_orbit_tiles_async(sm + (stage ^ 1) * 6 * SLOT, os, in + nb * n3, nv);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        if (MODE == 0) {
            p3_orbits_inplace(sm + stage * 6 * SLOT, os, t0, t1, t2, nv, k);
            __syncthreads();
            store_orbit_tiles(out0 + b * n3, sm + stage * 6 * SLOT, os, nv);
            __syncthreads();  // buf is refilled two iterations later
            continue;
        }
        const double *buf = sm + stage * 6 * SLOT;
        for (int s = 0; s < os.nslot; s++) {
            const int X0 = os.tile[s][0] * TE, Y0 = os.tile[s][1] * TE, Z0 = os.tile[s][2] * TE;
            const int *nbr = os.nbr[s];
            for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
                int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
                int gx = X0 + x, gy = Y0 + y, gz = Z0 + z;
                if (gx >= nv || gy >= nv || gz >= nv) continue;
                int64_t g = b * n3 + ((int64_t)gx * nv + gy) * nv + gz;
                double a0 = pv<0>(buf, nbr, x, y, z);
                if (MODE == 0) {
                    double r;
                    if (gx == gy && gy == gz) {
                        r = dadd(dmul(k.beta, a0), dmul(k.ap34, dmul(k.p012, a0)));
                    } else {
                        // T(u) = p0 A(u) + p1 A(u2,u1,u0) + p2 A(u1,u0,u2); T at (u0,u2,u1)
                        double tu = dadd(dadd(dmul(k.p0, a0), dmul(k.p1, pv<5>(buf, nbr, x, y, z))),
                                         dmul(k.p2, pv<2>(buf, nbr, x, y, z)));
                        double tw = dadd(dadd(dmul(k.p0, pv<1>(buf, nbr, x, y, z)), dmul(k.p1, pv<3>(buf, nbr, x, y, z))),
                                         dmul(k.p2, pv<4>(buf, nbr, x, y, z)));
                        r = dadd(dmul(k.beta, a0), dmul(k.alpha, dadd(dmul(k.p3, tu), dmul(k.p4, tw))));
                    }
                    out0[g] = r;
                } else if (MODE == 1) {
                    double bac = pv<2>(buf, nbr, x, y, z), acb = pv<1>(buf, nbr, x, y, z),
                           cba = pv<5>(buf, nbr, x, y, z);
                    double two = dmul(2.0, a0);
                    double d0 = dsub(dsub(two, acb), cba);
                    out0[g] = d0;
                    out1[g] = dsub(dsub(two, bac), acb);
                    out2[g] = dsub(dadd(d0, acb), bac);
                } else {
                    out0[g] = dadd(a0, pv<4>(buf, nbr, x, y, z));
                }
            }
        }
        __syncthreads();  // buf is refilled two iterations later
    }
}

// P3 spin summation, in place (out == A) or out of place.  The tile geometry of a CTA is the same for
// every block, so each thread computes its shared/global offsets once: up to
// 12 (slot, element) copies and up to 2 canonical orbits (6 shared addresses
// each).  Per block the CTA then issues its cp.async copies, sums its orbits
// in shared memory and stores, while the copies of the next block are in
// flight; thread 0 also stages its share of the block after next into L2
// (cp.async.bulk.prefetch.L2) so the 64-byte tile rows are read from L2.
__global__ void __launch_bounds__(OT_THREADS, 3) k_p3_inplace(const double *A, double *out, int64_t nblocks, int nv,
                                                              int ntile, P3Coef k) {
    extern __shared__ double sm[];  // 2 x 6 x SLOT doubles
    __shared__ OrbitSet os;
    int t0, t1, t2;
    decode_tri3(blockIdx.x, ntile, t0, t1, t2);
    build_orbit_set(os, t0, t1, t2);
    const int64_t n3 = (int64_t)nv * nv * nv;
    // copies: pair j -> slot j / 2, element threadIdx.x + 256 * (j % 2)
    int goff[12];
    unsigned short soff[12];
    unsigned nload = 0;
    for (int j = 0; j < 12; j++) {
        const int sl = j >> 1, e = threadIdx.x + OT_THREADS * (j & 1);
        goff[j] = -1;
        soff[j] = 0;
        if (sl >= os.nslot) continue;
        const int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        const int gx = os.tile[sl][0] * TE + x, gy = os.tile[sl][1] * TE + y, gz = os.tile[sl][2] * TE + z;
        if (gx >= nv || gy >= nv || gz >= nv) continue;
        goff[j] = (gx * nv + gy) * nv + gz;
        soff[j] = (unsigned short)(sl * SLOT + sidx(x, y, z));
        nload |= 1u << j;
    }
    // canonical orbit positions of this thread (inside slot 0)
    unsigned short oa[2][6];
    int ocls[2];  // 0: none, 1: generic, 2: all indices equal
    for (int h = 0; h < 2; h++) {
        const int e = threadIdx.x + OT_THREADS * h;
        const int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        const int gx = t0 * TE + x, gy = t1 * TE + y, gz = t2 * TE + z;
        ocls[h] = 0;
        if (gx >= nv || gy >= nv || gz >= nv || (t0 == t1 && x > y) || (t1 == t2 && y > z)) continue;
        const int *nb = os.nbr[0];
        oa[h][0] = (unsigned short)(nb[0] * SLOT + sidx(x, y, z));
        oa[h][1] = (unsigned short)(nb[1] * SLOT + sidx(x, z, y));
        oa[h][2] = (unsigned short)(nb[2] * SLOT + sidx(y, x, z));
        oa[h][3] = (unsigned short)(nb[3] * SLOT + sidx(y, z, x));
        oa[h][4] = (unsigned short)(nb[4] * SLOT + sidx(z, x, y));
        oa[h][5] = (unsigned short)(nb[5] * SLOT + sidx(z, y, x));
        ocls[h] = (gx == gy && gy == gz) ? 2 : 1;
    }
    // this CTA's share of a block for the L2 staging prefetch
    const int64_t ntri = gridDim.x;
    const int64_t share = ((n3 * 8 + ntri - 1) / ntri + 15) / 16 * 16;
    const int64_t pf_off = share * blockIdx.x;
    const int64_t pf_len = pf_off >= n3 * 8 ? 0 : (pf_off + share > n3 * 8 ? ((n3 * 8 - pf_off) / 16) * 16 : share);

    int64_t b = blockIdx.y;
    if (b >= nblocks) return;
    auto issue = [&](double *buf, const double *blk) {
#pragma unroll
        for (int j = 0; j < 12; j++)
            if (nload & (1u << j)) cp_async8(buf + soff[j], blk + goff[j]);
    };
    auto stage_l2 = [&](int64_t bb) {
        const char *src = (const char *)(A + bb * n3) + pf_off;
        // the bulk prefetch needs a 16-byte aligned source (blocks of odd nvir^3 are only 8-aligned)
        if (threadIdx.x == 0 && bb < nblocks && pf_len > 0 && (((uintptr_t)src) & 15) == 0) {
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"((unsigned)pf_len) : "memory");
        }
    };
    stage_l2(b + gridDim.y);
    issue(sm, A + b * n3);
    cp_async_commit();
    for (int stage = 0; b < nblocks; b += gridDim.y, stage ^= 1) {
        const int64_t nb_ = b + gridDim.y;
        stage_l2(nb_ + gridDim.y);
        if (nb_ < nblocks) {
            issue(sm + (stage ^ 1) * 6 * SLOT, A + nb_ * n3);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        double *buf = sm + stage * 6 * SLOT;
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
            if (ocls[h] == 0) continue;
            double v[6];
#pragma unroll
            for (int q = 0; q < 6; q++) v[q] = buf[oa[h][q]];
            if (ocls[h] == 2) {
                buf[oa[h][0]] = dadd(dmul(k.beta, v[0]), dmul(k.ap34, dmul(k.p012, v[0])));
                continue;
            }
            double r[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                double tu = dadd(dadd(dmul(k.p0, v[q]), dmul(k.p1, v[comp6(5, q)])), dmul(k.p2, v[comp6(2, q)]));
                double tw =
                    dadd(dadd(dmul(k.p0, v[comp6(1, q)]), dmul(k.p1, v[comp6(3, q)])), dmul(k.p2, v[comp6(4, q)]));
                r[q] = dadd(dmul(k.beta, v[q]), dmul(k.alpha, dadd(dmul(k.p3, tu), dmul(k.p4, tw))));
            }
#pragma unroll
            for (int q = 0; q < 6; q++) buf[oa[h][q]] = r[q];
        }
        __syncthreads();
        double *blk = out + b * n3;
#pragma unroll
        for (int j = 0; j < 12; j++)
            if (nload & (1u << j)) blk[goff[j]] = buf[soff[j]];
        __syncthreads();  // buf is refilled two iterations later
    }
}

// Element of an 8^3 tile for lane l (0..31) and step j (0..15): a linear
// map over GF(2) of the lane and step bits, chosen so that for every
// simultaneous permutation p the 16 lanes of each half-warp reading position
// p(u) of a dense [a][b][c] tile hit 16 different 8-byte bank pairs (a 64-bit
// shared access is served per half-warp), i.e. all six permuted read patterns
// are conflict-free; over (l, j) it is a bijection onto the 512 positions.
__device__ __forceinline__ void tile_element(int l, int j, int u[3]) {
    const int l0 = l & 1, l1 = (l >> 1) & 1, l2 = (l >> 2) & 1, l3 = (l >> 3) & 1, l4 = (l >> 4) & 1;
    const int j0 = j & 1, j1 = (j >> 1) & 1, j2 = (j >> 2) & 1, j3 = (j >> 3) & 1;
    u[0] = l0 | (l1 << 1) | (l2 << 2);
    u[1] = l3 | ((l1 ^ l4) << 1) | ((l2 ^ j0) << 2);
    u[2] = (l0 ^ l3 ^ j3) | ((l1 ^ j1) << 1) | ((l2 ^ j2) << 2);
}

// Element owned by thread t (0..255) of a CTA, half h: the step is (warp, h).
__device__ __forceinline__ void tg_element(int t, int h, int u[3]) { tile_element(t & 31, (t >> 5) | (h << 3), u); }

// In-place P3 spin summation with TMA-moved orbit tiles.  A CTA of eight warps
// owns one orbit set at a time: one thread loads the distinct permuted 8^3
// tiles of its canonical tile triple (cp.async.bulk.tensor, box 8 x 8 x 8 of
// the [nblocks][nv][nv][nv] array; the ragged edge is zero-filled on load and
// clipped on store) into a dense 6 x 8^3 buffer, the warps evaluate every
// canonical position of the set in shared memory (lanes/steps follow
// tile_element, so the six permuted reads and writes are conflict-free), and
// the same thread stores the tiles back with TMA.  Two buffers per CTA: the
// tiles of the CTA's next set are in flight while the current set is summed
// and stored.  Two CTAs of eight warps per SM: with about 600 sets (1.6
// blocks) in flight, a tile row is still in L2 when its neighbours in the
// same 128-byte line are written, which measured 1.4x faster than four CTAs
// of two warps (rows of nvir doubles are not line-aligned).  Same arithmetic
// as k_p3_inplace; P3_full drops the unit coefficients (x * 1.0 == x
// exactly).
//
// Each wait on a load is bounded: thread 0 waits (WAIT_NS of %globaltimer),
// and on a timeout records DCC_ERR_TIMEOUT in *status, waits (bounded) for
// its copies in flight and the CTA returns.
constexpr int P3T_WARPS = 8;
constexpr int P3T_CTAS_PER_SM = 2;

__device__ __forceinline__ bool p3_wait_bounded(uint32_t bar, uint32_t parity, int *status) {
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (globaltimer() - t0 > WAIT_NS) {
            atomicExch(status, DCC_ERR_TIMEOUT);
            return false;
        }
    }
}

// MODE 0: P3, general pattern; 1: P3_full; 2: no arithmetic (the tiles go back unchanged:
// the traffic of the kernel alone, for measuring the layout's ceiling); 3: triple-sym into
// out[0..2]; 4: transpose-add into out[0]; 5, 6, 7: output B0, B1 or B2 of triple-sym alone
// into out[0].  Modes 0-2 work in place (out[0] is the input's map).
// Modes 3 and 4 write out[0] through the input buffer (each element is read and written by
// the one thread owning its canonical position) and mode 3 out[1], out[2] through two more
// 6 x 8^3 buffers.
struct OrbitMaps {
    CUtensorMap in, out[3];
};

template <int MODE>
__global__ void __launch_bounds__(32 * P3T_WARPS, P3T_CTAS_PER_SM)
    k_orbit_tma(const __grid_constant__ OrbitMaps maps, int64_t nblocks, int nv, int ntile, P3Coef k, int *status) {
    extern __shared__ __align__(128) double smbuf[];  // 2 x 6 x TE3 doubles (+ 2 x 6 x TE3 for mode 3)
    double *xbuf = smbuf + 12 * TE3;                  // mode 3: out[1], out[2]
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_ok;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t ntri = (int64_t)ntile * (ntile + 1) * (ntile + 2) / 6;
    const int64_t nwork = nblocks * ntri;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar[0]), 1);
        mbar_init(smem_u32(&bar[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // work item = (block, tile triple), triples fastest
    struct Item {
        int64_t b;
        int t[3];
        unsigned slot_of;  // slot s holds tile perm_s(T); slot_of = first slot with the same tile (3 bits per slot)
    };
    auto make = [&](int64_t wi) {
        Item it;
        it.b = wi / ntri;
        decode_tri3(wi % ntri, ntile, it.t[0], it.t[1], it.t[2]);
        unsigned so = 0;
#pragma unroll
        for (int sl = 0; sl < 6; sl++) {
            int first = sl;
#pragma unroll
            for (int q = sl - 1; q >= 0; q--)
                if (it.t[perm3(q, 0)] == it.t[perm3(sl, 0)] && it.t[perm3(q, 1)] == it.t[perm3(sl, 1)] &&
                    it.t[perm3(q, 2)] == it.t[perm3(sl, 2)])
                    first = q;
            so |= (unsigned)first << (3 * sl);
        }
        it.slot_of = so;
        return it;
    };
    auto distinct = [](const Item &it, int sl) { return ((it.slot_of >> (3 * sl)) & 7u) == (unsigned)sl; };
    auto issue = [&](const Item &it, int bi) {  // thread 0
        int nd = 0;
        for (int sl = 0; sl < 6; sl++) nd += distinct(it, sl);
        const uint32_t b = smem_u32(&bar[bi]);
        mbar_expect_tx(b, (uint32_t)nd * TE3 * 8);
        for (int sl = 0; sl < 6; sl++)
            if (distinct(it, sl))
                tma_load_5d(smem_u32(smbuf + (bi * 6 + sl) * TE3), &maps.in, b, it.t[perm3(sl, 2)] * TE,
                            it.t[perm3(sl, 1)] * TE, it.t[perm3(sl, 0)] * TE, (int)it.b, 0);
    };
    int64_t wi = blockIdx.x;
    if (wi >= nwork) return;
    Item cur = make(wi);
    if (threadIdx.x == 0) issue(cur, 0);
    uint32_t phase = 0;  // bit i: parity of buffer i
    for (int bi = 0; wi < nwork; wi += gridDim.x, bi ^= 1) {
        const int64_t wn = wi + gridDim.x;
        Item nxt = cur;
        if (wn < nwork) nxt = make(wn);
        if (threadIdx.x == 0) {
            // the stores of the buffer about to be refilled (and, mode 3, of the extra buffers) have read it
            if (wn < nwork || MODE == 3) bulk_wait_read<0>();
            if (wn < nwork) issue(nxt, bi ^ 1);
            s_ok = p3_wait_bounded(smem_u32(&bar[bi]), (phase >> bi) & 1u, status);
            if (!s_ok) {  // drain this CTA's copies in flight, then leave
                mbar_wait_quiet(smem_u32(&bar[bi ^ 1]), (phase >> (bi ^ 1)) & 1u);
                bulk_wait<0>();
            }
        }
        __syncthreads();
        if (!s_ok) return;
        mbar_wait_quiet(smem_u32(&bar[bi]), (phase >> bi) & 1u);  // complete already: acquires the tiles
        phase ^= 1u << bi;
        double *buf = smbuf + bi * 6 * TE3;
        const int t0 = cur.t[0], t1 = cur.t[1], t2 = cur.t[2];
        auto sof = [&](int sl) { return (int)((cur.slot_of >> (3 * sl)) & 7u); };
#pragma unroll
        for (int jj = 0; jj < 16 / P3T_WARPS; jj++) {
            if (MODE == 2) break;
            const int j = w * (16 / P3T_WARPS) + jj;
            int u[3];
            tile_element(lane, j, u);
            const int x = u[0], y = u[1], z = u[2];
            if (t0 * TE + x >= nv || t1 * TE + y >= nv || t2 * TE + z >= nv || (t0 == t1 && x > y) ||
                (t1 == t2 && y > z))
                continue;
            int a[6];
            a[0] = sof(0) * TE3 + x * 64 + y * 8 + z;
            a[1] = sof(1) * TE3 + x * 64 + z * 8 + y;
            a[2] = sof(2) * TE3 + y * 64 + x * 8 + z;
            a[3] = sof(3) * TE3 + y * 64 + z * 8 + x;
            a[4] = sof(4) * TE3 + z * 64 + x * 8 + y;
            a[5] = sof(5) * TE3 + z * 64 + y * 8 + x;
            double v[6];
#pragma unroll
            for (int q = 0; q < 6; q++) v[q] = buf[a[q]];
            if (MODE == 3) {  // B0 = 2T - T_acb - T_cba, B1 = 2T - T_bac - T_acb, B2 = B0 + T_acb - T_bac
                double o0[6], o1[6], o2[6];
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const double acb = v[comp6(1, q)], cba = v[comp6(5, q)], bac = v[comp6(2, q)];
                    const double two = dmul(2.0, v[q]);
                    o0[q] = dsub(dsub(two, acb), cba);
                    o1[q] = dsub(dsub(two, bac), acb);
                    o2[q] = dsub(dadd(o0[q], acb), bac);
                }
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    buf[a[q]] = o0[q];
                    xbuf[a[q]] = o1[q];
                    xbuf[6 * TE3 + a[q]] = o2[q];
                }
                continue;
            }
            if (MODE >= 5) {  // one output of triple-sym: B0 (5), B1 (6) or B2 (7), same operations
                double o[6];
#pragma unroll
                for (int q = 0; q < 6; q++) {
                    const double acb = v[comp6(1, q)], cba = v[comp6(5, q)], bac = v[comp6(2, q)];
                    const double two = dmul(2.0, v[q]);
                    const double b0 = dsub(dsub(two, acb), cba);
                    o[q] = MODE == 5 ? b0 : (MODE == 6 ? dsub(dsub(two, bac), acb) : dsub(dadd(b0, acb), bac));
                }
#pragma unroll
                for (int q = 0; q < 6; q++) buf[a[q]] = o[q];
                continue;
            }
            if (MODE == 4) {  // B = T + T_cab
                double o[6];
#pragma unroll
                for (int q = 0; q < 6; q++) o[q] = dadd(v[q], v[comp6(4, q)]);
#pragma unroll
                for (int q = 0; q < 6; q++) buf[a[q]] = o[q];
                continue;
            }
            if (t0 == t1 && t1 == t2 && x == y && y == z) {
                buf[a[0]] = dadd(dmul(k.beta, v[0]), dmul(k.ap34, dmul(k.p012, v[0])));
                continue;
            }
            double r[6];
#pragma unroll
            for (int q = 0; q < 6; q++) {
                if (MODE == 1) {
                    const double tu = dadd(dadd(v[q], v[comp6(5, q)]), v[comp6(2, q)]);
                    const double tw = dadd(dadd(v[comp6(1, q)], v[comp6(3, q)]), v[comp6(4, q)]);
                    r[q] = dadd(dmul(k.beta, v[q]), dmul(k.alpha, dadd(tu, tw)));
                } else {
                    const double tu =
                        dadd(dadd(dmul(k.p0, v[q]), dmul(k.p1, v[comp6(5, q)])), dmul(k.p2, v[comp6(2, q)]));
                    const double tw = dadd(dadd(dmul(k.p0, v[comp6(1, q)]), dmul(k.p1, v[comp6(3, q)])),
                                           dmul(k.p2, v[comp6(4, q)]));
                    r[q] = dadd(dmul(k.beta, v[q]), dmul(k.alpha, dadd(dmul(k.p3, tu), dmul(k.p4, tw))));
                }
            }
#pragma unroll
            for (int q = 0; q < 6; q++) buf[a[q]] = r[q];
        }
        fence_proxy_async_smem();  // the sums become visible to the TMA stores
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int sl = 0; sl < 6; sl++)
                if (distinct(cur, sl)) {
                    const int c0 = cur.t[perm3(sl, 2)] * TE, c1 = cur.t[perm3(sl, 1)] * TE, c2 = cur.t[perm3(sl, 0)] * TE;
                    tma_store_5d(&maps.out[0], smem_u32(buf + sl * TE3), c0, c1, c2, (int)cur.b, 0);
                    if (MODE == 3) {
                        tma_store_5d(&maps.out[1], smem_u32(xbuf + sl * TE3), c0, c1, c2, (int)cur.b, 0);
                        tma_store_5d(&maps.out[2], smem_u32(xbuf + (6 + sl) * TE3), c0, c1, c2, (int)cur.b, 0);
                    }
                }
            bulk_commit();
        }
        cur = nxt;
    }
    if (threadIdx.x == 0) bulk_wait<0>();
}

int p3_pattern(const char *name, double p[5]) {
    static const struct {
        const char *n;
        double c[5];
    } tab[] = {{"P3_full", {1.0, 1.0, 1.0, 1.0, 1.0}},
               {"P3_422", {2.0, -1.0, -1.0, 2.0, -1.0}},
               {"P3_201", {2.0, -1.0, -1.0, 1.0, 0.0}}};
    if (!name) return -1;
    for (auto &t : tab)
        if (strcmp(name, t.n) == 0) {
            memcpy(p, t.c, sizeof(t.c));
            return 0;
        }
    return -1;
}

// Status word of the bounded waits in the TMA symmetrizer (0, or DCC_ERR_TIMEOUT once a
// wait gave up); one per device, read and cleared by dcc_t3_symmetrize_status.
static __device__ int g_sym_status;

static int *sym_status_word() {
    static std::mutex mu;
    static struct {
        unsigned long long ctx;
        int *addr;
    } cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    unsigned long long ctx = current_context_id();
    if (!cache[dev].addr || !ctx || cache[dev].ctx != ctx) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sym_status) != cudaSuccess) return nullptr;
        cache[dev].addr = (int *)p;
        cache[dev].ctx = current_context_id();
    }
    return cache[dev].addr;
}

// The TMA orbit-tile kernel on nblocks nvir^3 blocks (even nvir, 16-byte aligned buffers);
// DCC_ERR_UNSUPPORTED when the layout does not allow it (the caller then uses another kernel).
static int orbit_tma_launch(int mode, const double *in, double *const out[3], int64_t nblocks, int64_t nvir,
                            const P3Coef &k, cudaStream_t st) {
    const int nout = mode == 3 ? 3 : 1;
    if (nvir % 2 != 0 || ((uintptr_t)in & 15) != 0 || nblocks >= (1ll << 31) || nvir > 65536) return DCC_ERR_UNSUPPORTED;
    for (int o = 0; o < nout; o++)
        if (((uintptr_t)out[o] & 15) != 0) return DCC_ERR_UNSUPPORTED;
    EncodeTiledFn fn = encode_fn();
    int *status = sym_status_word();
    if (!fn || !status) return DCC_ERR_UNSUPPORTED;
    OrbitMaps maps;
    memset(&maps, 0, sizeof(maps));
    const cuuint64_t nv = (cuuint64_t)nvir;
    const cuuint64_t dims[5] = {nv, nv, nv, (cuuint64_t)nblocks, 1};
    const cuuint64_t strides[4] = {nv * 8, nv * nv * 8, nv * nv * nv * 8, nv * nv * nv * 8 * (cuuint64_t)nblocks};
    const cuuint32_t box[5] = {TE, TE, TE, 1, 1}, es[5] = {1, 1, 1, 1, 1};
    for (int o = -1; o < nout; o++) {
        CUtensorMap *m = o < 0 ? &maps.in : &maps.out[o];
        void *base = o < 0 ? const_cast<double *>(in) : out[o];
        if (fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return DCC_ERR_UNSUPPORTED;
    }
    const int ntile = (int)ceil_div(nvir, TE);
    const int64_t ntri = (int64_t)ntile * (ntile + 1) * (ntile + 2) / 6;
    const size_t tsm = (size_t)(mode == 3 ? 4 : 2) * 6 * TE3 * sizeof(double);
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // triple-sym writes three outputs per tile: half the sets in flight keeps its lines in L2
    const int64_t nwork = nblocks * ntri, cap = (int64_t)nsm * (mode == 3 ? 1 : P3T_CTAS_PER_SM);
    const unsigned grid = (unsigned)(nwork < cap ? nwork : cap);
#define DCC_ORBIT_TMA(M)                                                                                  \
    case M:                                                                                               \
        cudaFuncSetAttribute(k_orbit_tma<M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsm);      \
        k_orbit_tma<M><<<grid, 32 * P3T_WARPS, tsm, st>>>(maps, nblocks, (int)nvir, ntile, k, status);   \
        break;
    switch (mode) {
        DCC_ORBIT_TMA(0)
        DCC_ORBIT_TMA(1)
        DCC_ORBIT_TMA(2)
        DCC_ORBIT_TMA(3)
        DCC_ORBIT_TMA(4)
        DCC_ORBIT_TMA(5)
        DCC_ORBIT_TMA(6)
        DCC_ORBIT_TMA(7)
        default:
            return DCC_ERR_UNSUPPORTED;
    }
#undef DCC_ORBIT_TMA
    return DCC_OK;
}

static int orbit3_launch(int mode, const double *in, double *o0, double *o1, double *o2, int64_t nblocks,
                         int64_t nvir, const P3Coef &k, void *stream) {
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    int ntile = (int)ceil_div(nvir, TE);
    int64_t ntri = (int64_t)ntile * (ntile + 1) * (ntile + 2) / 6;
    // about 8 CTA waves of 148 SMs x 4 resident CTAs, each CTA walking several blocks
    int64_t gy = (148 * 4 * 8 + ntri - 1) / ntri;
    gy = gy < 1 ? 1 : (gy > nblocks ? nblocks : gy);
    gy = gy > 65535 ? 65535 : gy;
    dim3 grid((unsigned)ntri, (unsigned)gy);
    size_t smem = 2 * 6 * SLOT * sizeof(double);
    cudaStream_t st = as_stream(stream);
    {
        const bool full = k.p0 == 1.0 && k.p1 == 1.0 && k.p2 == 1.0 && k.p3 == 1.0 && k.p4 == 1.0;
        const int tm = mode == 0 ? (full ? 1 : 0) : (mode == 1 ? 3 : 4);
        double *const outs[3] = {o0, o1, o2};
        if (mode == 1 && nvir % 8 != 0) {
            // rows not 64-byte aligned: three single-output passes (each output's partial lines
            // merge in L2 one stream at a time), measured 2x faster than one pass with three
            // output streams at nvir = 90
            int rc = DCC_OK;
            for (int o = 0; o < 3 && rc == DCC_OK; o++) {
                double *const one[3] = {outs[o], nullptr, nullptr};
                rc = orbit_tma_launch(5 + o, in, one, nblocks, nvir, k, st);
            }
            if (rc == DCC_OK) return launch_status("orbit-tile T3 kernel");
        } else if (orbit_tma_launch(tm, in, outs, nblocks, nvir, k, st) == DCC_OK) {
            return launch_status(mode == 0 ? "P3 spin summation" : "orbit-tile T3 kernel");
        }
    }
    if (mode == 0 && nvir <= 1290) {  // 32-bit element offsets inside a block
        cudaFuncSetAttribute(k_p3_inplace, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_p3_inplace<<<grid, OT_THREADS, smem, st>>>(in, o0, nblocks, (int)nvir, ntile, k);
        return launch_status("P3 spin summation");
    }
    if (mode == 0) cudaFuncSetAttribute(k_orbit3<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (mode == 1) cudaFuncSetAttribute(k_orbit3<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (mode == 2) cudaFuncSetAttribute(k_orbit3<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (mode == 0)
        k_orbit3<0><<<grid, OT_THREADS, smem, st>>>(in, o0, o1, o2, nblocks, (int)nvir, ntile, k);
    else if (mode == 1)
        k_orbit3<1><<<grid, OT_THREADS, smem, st>>>(in, o0, o1, o2, nblocks, (int)nvir, ntile, k);
    else
        k_orbit3<2><<<grid, OT_THREADS, smem, st>>>(in, o0, o1, o2, nblocks, (int)nvir, ntile, k);
    return launch_status("orbit-tile T3 kernel");
}

// ---------------------------------------------------------------- unpack

// out[n] = T3[ijk[n]] for any ordering.  A CTA owns one 8^3 output tile
// position and walks n = blockIdx.y, blockIdx.y + gridDim.y, ...; the source
// tile of the next n is copied asynchronously while the current one is
// written out through the shared-memory transpose.
struct TakeSrc {
    int cs;
    int64_t l;
    int V[3];
};

__device__ __forceinline__ TakeSrc take_src(const int32_t *ijk, const int64_t *loc, int64_t n, int nocc,
                                            const int T[3]) {
    TakeSrc r;
    int64_t s[3];
    int i = ijk[3 * n], j = ijk[3 * n + 1], k = ijk[3 * n + 2];
    bool ok = i >= 0 && j >= 0 && k >= 0 && i < nocc && j < nocc && k < nocc;
    r.cs = order_case3(ok ? i : 0, ok ? j : 0, ok ? k : 0, s);
    r.l = ok ? loc[ijk_linear(s[0], s[1], s[2], nocc)] : -1;
    // output tile T comes from source tile V with V[perm3(cs,m)] = T[m]
    for (int m = 0; m < 3; m++) r.V[perm3(r.cs, m)] = T[m];
    return r;
}

__device__ __forceinline__ void take_load_async(double *sm, const double *t3, const TakeSrc &src, int nv) {
    if (src.l < 0) return;
    const double *blk = t3 + src.l * (int64_t)nv * nv * nv;
    for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
        int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        int gx = src.V[0] * TE + x, gy = src.V[1] * TE + y, gz = src.V[2] * TE + z;
        if (gx < nv && gy < nv && gz < nv) cp_async8(sm + sidx(x, y, z), blk + ((int64_t)gx * nv + gy) * nv + gz);
    }
}

__global__ void __launch_bounds__(OT_THREADS) k_take_t3(const double *t3, double *out, const int32_t *ijk,
                                                        const int64_t *loc, int64_t count, int nocc, int nv,
                                                        int ntile) {
    __shared__ double sm[2 * SLOT];
    const int64_t n3 = (int64_t)nv * nv * nv;
    const int T[3] = {(int)(blockIdx.x / (ntile * ntile)), (int)((blockIdx.x / ntile) % ntile),
                      (int)(blockIdx.x % ntile)};
    int64_t n = blockIdx.y;
    if (n >= count) return;
    TakeSrc cur = take_src(ijk, loc, n, nocc, T);
    take_load_async(sm, t3, cur, nv);
    cp_async_commit();
    for (int stage = 0; n < count; n += gridDim.y, stage ^= 1) {
        const int64_t nn = n + gridDim.y;
        TakeSrc nxt;
        if (nn < count) {
            nxt = take_src(ijk, loc, nn, nocc, T);
            take_load_async(sm + (stage ^ 1) * SLOT, t3, nxt, nv);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double *buf = sm + stage * SLOT;
        double *dst = out + n * n3;
        for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
            int u[3] = {e >> 6, (e >> 3) & 7, e & 7};
            int gx = T[0] * TE + u[0], gy = T[1] * TE + u[1], gz = T[2] * TE + u[2];
            if (gx >= nv || gy >= nv || gz >= nv) continue;
            int v[3];
            for (int m = 0; m < 3; m++) v[perm3(cur.cs, m)] = u[m];
            dst[((int64_t)gx * nv + gy) * nv + gz] = (cur.l >= 0) ? buf[sidx(v[0], v[1], v[2])] : 0.0;
        }
        __syncthreads();
        if (nn < count) cur = nxt;
    }
}

// Whole-block copies: out[r] = in[map[req[r]]] (map/req optional).
__global__ void k_copy_blocks(const double *in, double *out, const int32_t *req, const int64_t *map, int64_t nreq,
                              int64_t blk) {
    for (int64_t r = blockIdx.y; r < nreq; r += gridDim.y) {
        int64_t l = map ? map[req ? req[r] : r] : (req ? req[r] : r);
        if (l < 0) continue;
        const double *s = in + l * blk;
        double *d = out + r * blk;
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < blk; e += (int64_t)gridDim.x * blockDim.x)
            d[e] = s[e];
    }
}

// ---------------------------------------------------------------- divide / update

// One warp per row (q, a, b) of nvir contiguous elements; D_ab is formed once
// per row, lanes stride over c.  D = (eia[i,a] + eia[j,b]) + eia[k,c].
__global__ void k_r3_divide(double *r3, const double *eia, const int32_t *ijk, int64_t nblocks, int nv) {
    const int lane = threadIdx.x & 31;
    const int64_t nrow = nblocks * nv * nv;
    for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrow;
         row += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int64_t q = row / (nv * nv);
        int ab = (int)(row - q * nv * nv), a = ab / nv, b = ab - a * nv;
        double dab = dadd(eia[(int64_t)ijk[3 * q] * nv + a], eia[(int64_t)ijk[3 * q + 1] * nv + b]);
        const double *ek = eia + (int64_t)ijk[3 * q + 2] * nv;
        double *r = r3 + row * nv;
        for (int c = lane; c < nv; c += 32) r[c] = __ddiv_rn(r[c], dadd(dab, ek[c]));
    }
}

constexpr int UPD_THREADS = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Fused divide + t3 update + squared norms, one warp per row (q, a, b);
// per-CTA partials go to ws[2*cta].
__global__ void __launch_bounds__(UPD_THREADS) k_t3_divide_update(double *t3, double *r3, const double *eia,
                                                                  const int32_t *ijk, int64_t nblocks, int nv,
                                                                  int nact, int write_r3, double *ws) {
    const int lane = threadIdx.x & 31;
    const int64_t nrow = nblocks * nv * nv;
    double s_all = 0.0, s_act = 0.0;
    for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < nrow;
         row += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int64_t q = row / (nv * nv);
        int ab = (int)(row - q * nv * nv), a = ab / nv, b = ab - a * nv;
        double dab = dadd(eia[(int64_t)ijk[3 * q] * nv + a], eia[(int64_t)ijk[3 * q + 1] * nv + b]);
        const double *ek = eia + (int64_t)ijk[3 * q + 2] * nv;
        double *rr = r3 + row * nv, *tt = t3 + row * nv;
        const bool act_ab = a < nact && b < nact;
        for (int c0 = 0; c0 < nv; c0 += 96) {
            // issue every load of this chunk before the first use
            double rv[3], tv[3], ev[3];
#pragma unroll
            for (int u = 0; u < 3; u++) {
                const int c = c0 + lane + 32 * u;
                rv[u] = c < nv ? rr[c] : 0.0;
                tv[u] = c < nv ? tt[c] : 0.0;
                ev[u] = c < nv ? ek[c] : 1.0;
            }
#pragma unroll
            for (int u = 0; u < 3; u++) {
                const int c = c0 + lane + 32 * u;
                if (c >= nv) continue;
                double r = __ddiv_rn(rv[u], dadd(dab, ev[u]));
                if (write_r3) rr[c] = r;
                tt[c] = dadd(tv[u], r);
                double r2 = r * r;
                s_all += r2;
                if (act_ab && c < nact) s_act += r2;
            }
        }
    }
    __shared__ double red[2][UPD_THREADS / 32];
    s_all = warp_sum(s_all);
    s_act = warp_sum(s_act);
    int w = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][w] = s_all;
        red[1][w] = s_act;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int i = 0; i < UPD_THREADS / 32; i++) {
            x += red[0][i];
            y += red[1][i];
        }
        ws[2 * blockIdx.x] = x;
        ws[2 * blockIdx.x + 1] = y;
    }
}

// Deterministic final sum of n partial pairs into out[0..1].
__global__ void k_sum_pairs(const double *ws, int64_t n, double *out) {
    __shared__ double red[2][32];
    double a = 0.0, b = 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        a += ws[2 * i];
        b += ws[2 * i + 1];
    }
    a = warp_sum(a);
    b = warp_sum(b);
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = a;
        red[1][threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) {
            x += red[0][i];
            y += red[1][i];
        }
        out[0] = x;
        out[1] = y;
    }
}

// 1-D grid of row-walking CTAs: 148 SMs x 8 resident CTAs x 4 waves at most.
static unsigned row_grid(int64_t nrow, int threads) {
    int64_t g = (nrow * 32 + threads - 1) / threads;
    return (unsigned)(g < 148 * 32 ? (g ? g : 1) : 148 * 32);
}

// ---------------------------------------------------------------- IJK -> ABC

// t3_abc[g][x][y][z]: the canonical block of sorted(x,y,z) read at
// sigma_p^{-1}(A,B,C) for the largest axis map p with sigma_p^{-1}(x,y,z)
// sorted (the last record the reference's pack order writes there).
__global__ void k_ijk_to_abc(const double *t3_ijk, double *t3_abc, int no, int nv, int64_t nabc) {
    const int64_t o3 = (int64_t)no * no * no;
    for (int64_t g = blockIdx.y; g < nabc; g += gridDim.y) {
        // decode g -> A<=B<=C
        int64_t r = g;
        int A = 0;
        for (;; A++) {
            int64_t m = (int64_t)(nv - A) * (nv - A + 1) / 2;
            if (r < m) break;
            r -= m;
        }
        int B = A;
        for (;; B++) {
            if (r < nv - B) break;
            r -= nv - B;
        }
        int C = B + (int)r;
        int tgt[3] = {A, B, C};
        for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < o3; e += (int64_t)gridDim.x * blockDim.x) {
            int xyz[3] = {(int)(e / (no * no)), (int)((e / no) % no), (int)(e % no)};
            int best = 0, w0 = 0, w1 = 0, w2 = 0;
            for (int p = 0; p < 6; p++) {
                int w[3];
                for (int m = 0; m < 3; m++) w[perm3(p, m)] = xyz[m];
                if (w[0] <= w[1] && w[1] <= w[2]) {
                    best = p;
                    w0 = w[0];
                    w1 = w[1];
                    w2 = w[2];
                }
            }
            int abc[3];
            for (int m = 0; m < 3; m++) abc[perm3(best, m)] = tgt[m];
            const double *blk = t3_ijk + ijk_linear(w0, w1, w2, no) * (int64_t)nv * nv * nv;
            t3_abc[g * o3 + e] = blk[((int64_t)abc[0] * nv + abc[1]) * nv + abc[2]];
        }
    }
}

// Ordering case of (a,b,c) chosen by the reference's three c-regions
// (src/rccsdt_q.c:690-743).
__device__ __forceinline__ int abc_case(int a, int b, int c, int s[3]) {
    int lo = a < b ? a : b, hi = a < b ? b : a, cs;
    if (c > hi) cs = (a <= b) ? 0 : 2;
    else if (c > lo) cs = (a <= b) ? ((b <= c) ? 0 : 1) : ((a <= c) ? 2 : 4);
    else cs = (a <= b) ? ((a <= c) ? 1 : 3) : ((b <= c) ? 4 : 5);
    int v[3] = {a, b, c};
    // sorted triple = (v[perm3(cs,0)], ...) read through the case's axis map
    int srt[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {2, 0, 1}, {1, 2, 0}, {2, 1, 0}};
    s[0] = v[srt[cs][0]];
    s[1] = v[srt[cs][1]];
    s[2] = v[srt[cs][2]];
    return cs;
}

// One CTA per (ia, ib, c) block of nocc^3: load the ABC block, write it with
// the occupied axes permuted.
__global__ void k_fill_t3_abc(double *target, int a0, int a1, int b0, int b1, int nv, int no,
                              const double *t3_abc, int64_t ld_b) {
    extern __shared__ double blk[];
    const int o3 = no * no * no;
    const int ba = a1 - a0, bb = b1 - b0;
    const int64_t nwork = (int64_t)ba * bb * nv;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        int c = (int)(w % nv), ib = (int)((w / nv) % bb), ia = (int)(w / ((int64_t)nv * bb));
        int s[3];
        int cs = abc_case(a0 + ia, b0 + ib, c, s);
        const double *src = t3_abc + abc_linear(s[0], s[1], s[2], nv) * o3;
        for (int e = threadIdx.x; e < o3; e += blockDim.x) blk[e] = src[e];
        __syncthreads();
        double *dst = target + (((int64_t)ia * ld_b + ib) * nv + c) * o3;
        for (int e = threadIdx.x; e < o3; e += blockDim.x) {
            int u[3] = {e / (no * no), (e / no) % no, e % no};
            // dst[v[P0],v[P1],v[P2]] = src[v]  =>  src index v with v[P[m]] = u[m]
            int v[3];
            for (int m = 0; m < 3; m++) v[perm3(cs, m)] = u[m];
            dst[e] = blk[(v[0] * no + v[1]) * no + v[2]];
        }
        __syncthreads();
    }
}

// Single-block unpack with the case and source block resolved on the host.
__global__ void __launch_bounds__(OT_THREADS) k_take_t3_one(const double *t3, double *out, int i, int j, int k,
                                                            int64_t l, int nv, int ntile) {
    __shared__ double sm[SLOT];
    const int64_t n3 = (int64_t)nv * nv * nv;
    int T[3] = {(int)(blockIdx.x / (ntile * ntile)), (int)((blockIdx.x / ntile) % ntile), (int)(blockIdx.x % ntile)};
    int64_t s[3];
    int cs = order_case3(i, j, k, s);
    int V[3];
    for (int m = 0; m < 3; m++) V[perm3(cs, m)] = T[m];
    const double *src = t3 + l * n3;
    for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
        int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        int gx = V[0] * TE + x, gy = V[1] * TE + y, gz = V[2] * TE + z;
        if (gx < nv && gy < nv && gz < nv) sm[sidx(x, y, z)] = src[((int64_t)gx * nv + gy) * nv + gz];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
        int u[3] = {e >> 6, (e >> 3) & 7, e & 7};
        int gx = T[0] * TE + u[0], gy = T[1] * TE + u[1], gz = T[2] * TE + u[2];
        if (gx >= nv || gy >= nv || gz >= nv) continue;
        int v[3];
        for (int m = 0; m < 3; m++) v[perm3(cs, m)] = u[m];
        out[((int64_t)gx * nv + gy) * nv + gz] = sm[sidx(v[0], v[1], v[2])];
    }
}

}  // namespace dcc

using namespace dcc;

// ---------------------------------------------------------------- C ABI

static int p3_coef(const char *pattern, double alpha, double beta, P3Coef &k) {
    double p[5];
    if (p3_pattern(pattern, p)) {
        set_error("unrecognized pattern \"%s\"", pattern ? pattern : "(null)");
        return DCC_ERR_PATTERN;
    }
    k = P3Coef{p[0], p[1], p[2], p[3], p[4], alpha, beta, (p[0] + p[1]) + p[2], alpha * (p[3] + p[4])};
    return DCC_OK;
}

extern "C" int dcc_t3_spin_summation_inplace(double *A, int64_t nblocks, int64_t nvir, const char *pattern,
                                             double alpha, double beta, void *stream) {
    clear_error();
    P3Coef k;
    int rc = p3_coef(pattern, alpha, beta, k);
    if (rc) return rc;
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE(A || nblocks * nvir == 0, DCC_ERR_NULL, "A is NULL");
    return orbit3_launch(0, A, A, nullptr, nullptr, nblocks, nvir, k, stream);
}

namespace dcc {

// Out-of-place P3 for the patterns whose p4 is 0 (P3_201: B = beta A + alpha p3 (p0 A + p1 A^cba
// + p2 A^bac)) by strips, for nvir <= 104 at any row pitch: a work item is a block, a middle
// index b and a tile of 32 first indices a.  The CTA stages the column strip A[:, b, a0..a0+31]
// (every c; 256-byte segments, row pitch 33 doubles so the transposed reads are conflict-free)
// in shared memory, then each warp writes whole output rows B[a, b, :]: it issues the loads of
// both rows A[a,b,:] and A[b,a,:] (every c of the row at once, up to 8 in flight per lane) before
// the arithmetic, which takes A[c,b,a] from the strip.  Every element is read three times (strip,
// and the two rows), the repeats L2 hits: the items of one block run side by side.  The
// arithmetic is the orbit kernel's with its p4 term (0 x the second half) left out: equal results
// up to the sign of a zero.
constexpr int SP3_W = 32, SP3_PITCH = 33, SP3_MAXNV = 104;
// T: the storage type of A and B (double; float for the FP32 copies of the split precisions,
// whose values the arithmetic takes exactly as doubles, rounding the result once)
template <typename T>
__global__ void __launch_bounds__(256, 4) k_p3_strips(const T *__restrict__ A, T *__restrict__ B,
                                                      int64_t nblocks, int nv, int ntile, P3Coef k) {
    __shared__ T S[SP3_MAXNV * SP3_PITCH];  // S[c][s] = A[c][b][a0 + s]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t n3 = (int64_t)nv * nv * nv, nv2 = (int64_t)nv * nv;
    const int64_t per_blk = (int64_t)nv * ntile, nwork = nblocks * per_blk;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t blk = w / per_blk;
        const int r = (int)(w - blk * per_blk), b = r / ntile, a0 = (r - b * ntile) * SP3_W;
        const int h = nv - a0 < SP3_W ? nv - a0 : SP3_W;
        const T *Ab = A + blk * n3;
        T *Bb = B + blk * n3;
        for (int c = warp; c < nv; c += 8)
            if (lane < h) cp_async_el(S + c * SP3_PITCH + lane, Ab + (int64_t)c * nv2 + (int64_t)b * nv + a0 + lane);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (int s = warp; s < h; s += 8) {
            const int a = a0 + s;
            const T *rab = Ab + (int64_t)a * nv2 + (int64_t)b * nv, *rba = Ab + (int64_t)b * nv2 + (int64_t)a * nv;
            T *out = Bb + (int64_t)a * nv2 + (int64_t)b * nv;
            double vab[4], vba[4];  // c = lane + 32 j covers nv <= 128
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = lane + 32 * j;
                vab[j] = c < nv ? (double)__ldg(rab + c) : 0.0;
                vba[j] = c < nv ? (double)__ldg(rba + c) : 0.0;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int c = lane + 32 * j;
                if (c < nv) {
                    const double cba = (double)S[c * SP3_PITCH + s];
                    const double tu = dadd(dadd(dmul(k.p0, vab[j]), dmul(k.p1, cba)), dmul(k.p2, vba[j]));
                    out[c] = (T)dadd(dmul(k.beta, vab[j]), dmul(k.alpha, dmul(k.p3, tu)));
                }
            }
        }
        __syncthreads();  // the strip is refilled by the next item
    }
}

}  // namespace dcc

// The strip kernel for out-of-place P3 with p4 == 0, nvir <= 104; returns DCC_ERR_UNSUPPORTED
// (nothing launched) where it does not apply.
template <typename T>
static int p3_strips_launch(const T *A, T *B, int64_t nblocks, int64_t nvir, const P3Coef &k, void *stream) {
    if (k.p4 != 0.0 || A == B || nvir < 1 || nvir > SP3_MAXNV) return DCC_ERR_UNSUPPORTED;
    const int ntile = (int)ceil_div(nvir, SP3_W);
    int dev = 0, nsm = 148, per_sm = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_p3_strips<T>, 256, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t nwork = nblocks * nvir * ntile, cap = (int64_t)nsm * per_sm;
    const unsigned grid = (unsigned)(nwork < cap ? nwork : cap);
    k_p3_strips<T><<<grid, 256, 0, as_stream(stream)>>>(A, B, nblocks, (int)nvir, ntile, k);
    return DCC_OK;
}

extern "C" int dcc_t3_spin_summation(const double *A, double *B, int64_t nblocks, int64_t nvir, const char *pattern,
                                     double alpha, double beta, void *stream) {
    clear_error();
    P3Coef k;
    int rc = p3_coef(pattern, alpha, beta, k);
    if (rc) return rc;
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE((A && B) || nblocks * nvir == 0, DCC_ERR_NULL, "NULL buffer");
    const int64_t bytes = nblocks * nvir * nvir * nvir * (int64_t)sizeof(double);
    DCC_REQUIRE(A == B || (const char *)B + bytes <= (const char *)A || (const char *)A + bytes <= (const char *)B,
                DCC_ERR_SHAPE, "A and B overlap");
    if (nblocks > 0 && p3_strips_launch(A, B, nblocks, nvir, k, stream) == DCC_OK) return launch_status("P3 by strips");
    return orbit3_launch(0, A, B, nullptr, nullptr, nblocks, nvir, k, stream);
}

extern "C" int dcc_t3_spin_summation_kernel(const double *A, double *B, int64_t nblocks, int64_t nvir,
                                            const char *pattern, double alpha, double beta, int kernel, void *stream) {
    clear_error();
    DCC_REQUIRE(kernel >= 0 && kernel <= 2, DCC_ERR_UNSUPPORTED, "kernel must be 0..2");
    if (kernel == 0) return dcc_t3_spin_summation(A, B, nblocks, nvir, pattern, alpha, beta, stream);
    P3Coef k;
    int rc = p3_coef(pattern, alpha, beta, k);
    if (rc) return rc;
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE((A && B) || nblocks * nvir == 0, DCC_ERR_NULL, "NULL buffer");
    const int64_t bytes = nblocks * nvir * nvir * nvir * (int64_t)sizeof(double);
    DCC_REQUIRE(A == B || (const char *)B + bytes <= (const char *)A || (const char *)A + bytes <= (const char *)B,
                DCC_ERR_SHAPE, "A and B overlap");
    if (nblocks == 0) return DCC_OK;
    if (kernel == 2) return orbit3_launch(0, A, B, nullptr, nullptr, nblocks, nvir, k, stream);
    DCC_REQUIRE(p3_strips_launch(A, B, nblocks, nvir, k, stream) == DCC_OK, DCC_ERR_UNSUPPORTED,
                "this kernel does not apply to the pattern or shape");
    return launch_status("P3 by strips");
}

extern "C" int dcc_t3_spin_summation_f32(const float *A, float *B, int64_t nblocks, int64_t nvir, const char *pattern,
                                         double alpha, double beta, void *stream) {
    clear_error();
    P3Coef k;
    int rc = p3_coef(pattern, alpha, beta, k);
    if (rc) return rc;
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE((A && B) || nblocks * nvir == 0, DCC_ERR_NULL, "NULL buffer");
    const int64_t bytes = nblocks * nvir * nvir * nvir * (int64_t)sizeof(float);
    DCC_REQUIRE((const char *)B + bytes <= (const char *)A || (const char *)A + bytes <= (const char *)B,
                DCC_ERR_SHAPE, "A and B overlap");
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(p3_strips_launch(A, B, nblocks, nvir, k, stream) == DCC_OK, DCC_ERR_UNSUPPORTED,
                "the FP32 P3 serves the patterns without a p4 term (P3_201) at nvir <= %d", SP3_MAXNV);
    return launch_status("P3 by strips (FP32)");
}

namespace dcc {

// Stage ordering PI's values at the orbit positions P_q(E) of a canonical element E (shared
// addresses oa[q] in the staging buffer st and in the canonical block's orbit tiles `in`), from
// the values v[q] = C[P_q(E)] = in[oa[q]]: U[P_q(E)] =
// C[P_comp6(PI, q)(E)] = v[comp6(PI, q)] (xpass false), or the P3 spin summation of U there (xpass
// true: the per-position formula of k_p3_inplace over U's values, so the result equals a P3 pass
// over U bit for bit).  diag: all of E's indices equal (one position).
struct OrbitAddr {
    unsigned short a[6];
};

template <int PI>
__device__ __forceinline__ void stage_orbit(double *st, const OrbitAddr oa, const double *in, const P3Coef &k,
                                            bool diag, bool xpass) {
    double v[6];
#pragma unroll
    for (int q = 0; q < 6; q++) v[q] = in[oa.a[q]];
    if (diag) {
        const double u = v[comp6(PI, 0)];
        st[oa.a[0]] = xpass ? dadd(dmul(k.beta, u), dmul(k.ap34, dmul(k.p012, u))) : u;
        return;
    }
    if (!xpass) {
#pragma unroll
        for (int q = 0; q < 6; q++) st[oa.a[q]] = v[comp6(PI, q)];
        return;
    }
#pragma unroll
    for (int q = 0; q < 6; q++) {
        const double tu = dadd(dadd(dmul(k.p0, v[comp6(PI, q)]), dmul(k.p1, v[comp6(PI, comp6(5, q))])),
                               dmul(k.p2, v[comp6(PI, comp6(2, q))]));
        const double tw = dadd(dadd(dmul(k.p0, v[comp6(PI, comp6(1, q))]), dmul(k.p1, v[comp6(PI, comp6(3, q))])),
                               dmul(k.p2, v[comp6(PI, comp6(4, q))]));
        st[oa.a[q]] = dadd(dmul(k.beta, v[comp6(PI, q)]), dmul(k.alpha, dadd(dmul(k.p3, tu), dmul(k.p4, tw))));
    }
}

// Unpack and P3 of every ordering in one pass: for every canonical block C = t3[q] and every
// distinct ordering o of its occupied indices, U[o] = C with its virtual axes permuted (the
// unpack of k_unpack_band / k_unpack_all) and X[o] = beta U[o] + alpha P(U[o]) (the pass
// k_p3_inplace makes over U), both from the orbit tiles of C in shared memory.  A CTA owns one
// tile triple (as k_p3_inplace) and walks the canonical blocks; per block it loads the (up to
// six) orbit tiles once and writes 2 x 6 tiles per ordering through one staging buffer, so X
// costs no read of U: at an odd nvir the two passes read U with 8-byte copies whose 64-byte tile
// rows straddle sectors (1.9x the algorithmic DRAM reads under ncu).
__global__ void __launch_bounds__(OT_THREADS, 2) k_unpack_p3(const double *t3, double *U, double *X, int64_t nblocks,
                                                             int nocc, int nv, int ntile, P3Coef k) {
    extern __shared__ double sm[];  // orbit tiles of C (6 x SLOT), staging of one output (6 x SLOT)
    double *in = sm, *st = sm + 6 * SLOT;
    __shared__ OrbitSet os;
    int t0, t1, t2;
    decode_tri3(blockIdx.x, ntile, t0, t1, t2);
    build_orbit_set(os, t0, t1, t2);
    const int64_t n3 = (int64_t)nv * nv * nv;
    int goff[12];
    unsigned short soff[12];
    unsigned nload = 0;
    for (int j = 0; j < 12; j++) {
        const int sl = j >> 1, e = threadIdx.x + OT_THREADS * (j & 1);
        goff[j] = -1;
        soff[j] = 0;
        if (sl >= os.nslot) continue;
        const int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        const int gx = os.tile[sl][0] * TE + x, gy = os.tile[sl][1] * TE + y, gz = os.tile[sl][2] * TE + z;
        if (gx >= nv || gy >= nv || gz >= nv) continue;
        goff[j] = (gx * nv + gy) * nv + gz;
        soff[j] = (unsigned short)(sl * SLOT + sidx(x, y, z));
        nload |= 1u << j;
    }
    OrbitAddr oa[2];
    int ocls[2];  // 0: none, 1: generic, 2: all indices equal
    for (int h = 0; h < 2; h++) {
        const int e = threadIdx.x + OT_THREADS * h;
        const int x = e >> 6, y = (e >> 3) & 7, z = e & 7;
        const int gx = t0 * TE + x, gy = t1 * TE + y, gz = t2 * TE + z;
        ocls[h] = 0;
        if (gx >= nv || gy >= nv || gz >= nv || (t0 == t1 && x > y) || (t1 == t2 && y > z)) continue;
        const int *nb = os.nbr[0];
        oa[h].a[0] = (unsigned short)(nb[0] * SLOT + sidx(x, y, z));
        oa[h].a[1] = (unsigned short)(nb[1] * SLOT + sidx(x, z, y));
        oa[h].a[2] = (unsigned short)(nb[2] * SLOT + sidx(y, x, z));
        oa[h].a[3] = (unsigned short)(nb[3] * SLOT + sidx(y, z, x));
        oa[h].a[4] = (unsigned short)(nb[4] * SLOT + sidx(z, x, y));
        oa[h].a[5] = (unsigned short)(nb[5] * SLOT + sidx(z, y, x));
        ocls[h] = (gx == gy && gy == gz) ? 2 : 1;
    }
    for (int64_t q = blockIdx.y; q < nblocks; q += gridDim.y) {
        const double *blk = t3 + q * n3;
#pragma unroll
        for (int j = 0; j < 12; j++)
            if (nload & (1u << j)) cp_async8(in + soff[j], blk + goff[j]);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();  // the orbit tiles of C have landed
        int o[3];
        decode_tri3(q, nocc, o[0], o[1], o[2]);
        for (int g = 0; g < 6; g++) {
            const int xyz[3] = {o[perm3(g, 0)], o[perm3(g, 1)], o[perm3(g, 2)]};
            bool dup = false;
            for (int sp = 0; sp < g; sp++)
                if (o[perm3(sp, 0)] == xyz[0] && o[perm3(sp, 1)] == xyz[1] && o[perm3(sp, 2)] == xyz[2]) dup = true;
            if (dup) continue;  // uniform over the CTA
            int64_t srt[3];
            const int c = order_case3(xyz[0], xyz[1], xyz[2], srt);
            const int pi = c == 3 ? 4 : (c == 4 ? 3 : c);  // the inverse permutation of case c
            const int64_t out = ((int64_t)xyz[0] * nocc + xyz[1]) * nocc + xyz[2];
            for (int pass = 0; pass < 2; pass++) {
                double *dst = pass == 0 ? U : X;
                if (dst == nullptr) continue;
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    if (!ocls[h]) continue;
                    const bool diag = ocls[h] == 2, xp = pass == 1;
                    switch (pi) {
                    case 0: stage_orbit<0>(st, oa[h], in, k, diag, xp); break;
                    case 1: stage_orbit<1>(st, oa[h], in, k, diag, xp); break;
                    case 2: stage_orbit<2>(st, oa[h], in, k, diag, xp); break;
                    case 3: stage_orbit<3>(st, oa[h], in, k, diag, xp); break;
                    case 4: stage_orbit<4>(st, oa[h], in, k, diag, xp); break;
                    default: stage_orbit<5>(st, oa[h], in, k, diag, xp); break;
                    }
                }
                __syncthreads();  // the staged tiles are complete
                double *ob = dst + out * n3;
#pragma unroll
                for (int j = 0; j < 12; j++)
                    if (nload & (1u << j)) ob[goff[j]] = st[soff[j]];
                __syncthreads();  // the staging buffer is free again
            }
        }
    }
}

}  // namespace dcc

extern "C" int dcc_t3_unpack_p3(const double *t3, double *U, double *X, int64_t nocc, int64_t nvir,
                                const char *pattern, double alpha, double beta, void *stream) {
    clear_error();
    P3Coef k;
    int rc = p3_coef(pattern, alpha, beta, k);
    if (rc) return rc;
    DCC_REQUIRE(nocc >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nocc == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t3 && X, DCC_ERR_NULL, "NULL buffer");
    DCC_REQUIRE(nvir <= 1290 && nocc < 1290, DCC_ERR_UNSUPPORTED, "nvir > 1290 exceeds 32-bit block offsets");
    const int64_t n3 = nvir * nvir * nvir * (int64_t)sizeof(double);
    const int64_t nblocks = nocc * (nocc + 1) * (nocc + 2) / 6, nu = nocc * nocc * nocc;
    auto apart = [](const void *a, int64_t na, const void *b, int64_t nb) {
        return (const char *)a + na <= (const char *)b || (const char *)b + nb <= (const char *)a;
    };
    DCC_REQUIRE(apart(t3, nblocks * n3, X, nu * n3) && (!U || (apart(t3, nblocks * n3, U, nu * n3) &&
                                                            apart(U, nu * n3, X, nu * n3))),
                DCC_ERR_SHAPE, "t3, U and X overlap");
    const int ntile = (int)ceil_div(nvir, TE);
    const int64_t ntri = (int64_t)ntile * (ntile + 1) * (ntile + 2) / 6;
    int64_t gy = (148 * 4 * 8 + ntri - 1) / ntri;
    gy = gy < 1 ? 1 : (gy > nblocks ? nblocks : gy);
    gy = gy > 65535 ? 65535 : gy;
    const size_t smem = 2 * 6 * SLOT * sizeof(double);
    cudaFuncSetAttribute(k_unpack_p3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_unpack_p3<<<dim3((unsigned)ntri, (unsigned)gy), OT_THREADS, smem, as_stream(stream)>>>(
        t3, U, X, nblocks, (int)nocc, (int)nvir, ntile, k);
    return launch_status("t3_unpack_p3");
}

extern "C" int dcc_t3_single_spin_summation_inplace(double *A, int64_t nvir, const char *pattern, double alpha,
                                                    double beta, void *stream) {
    return dcc_t3_spin_summation_inplace(A, 1, nvir, pattern, alpha, beta, stream);
}

extern "C" int dcc_t3_spin_summation_triple_sym(const double *A, double *B0, double *B1, double *B2,
                                                int64_t nblocks, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE((A && B0 && B1 && B2) || nblocks * nvir == 0, DCC_ERR_NULL, "NULL buffer");
    DCC_REQUIRE(A != B0 && A != B1 && A != B2, DCC_ERR_SHAPE, "triple_sym is out of place");
    P3Coef k{};
    return orbit3_launch(1, A, B0, B1, B2, nblocks, nvir, k, stream);
}

extern "C" int dcc_t3_transpose_add(const double *A, double *B, int64_t nblocks, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE((A && B) || nblocks * nvir == 0, DCC_ERR_NULL, "NULL buffer");
    DCC_REQUIRE(A != B, DCC_ERR_SHAPE, "transpose_add is out of place");
    P3Coef k{};
    return orbit3_launch(2, A, B, nullptr, nullptr, nblocks, nvir, k, stream);
}

extern "C" int dcc_t3_orbit_roundtrip(double *A, int64_t nblocks, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(A, DCC_ERR_NULL, "A is NULL");
    P3Coef k{};
    double *const outs[3] = {A, nullptr, nullptr};
    DCC_REQUIRE(orbit_tma_launch(2, A, outs, nblocks, nvir, k, as_stream(stream)) == DCC_OK, DCC_ERR_UNSUPPORTED,
                "needs even nvir and a 16-byte aligned buffer");
    return launch_status("orbit tile round trip");
}

extern "C" int dcc_t3_symmetrize_status(int *out, void *stream) {
    clear_error();
    DCC_REQUIRE(out, DCC_ERR_NULL, "out is NULL");
    int *word = sym_status_word();
    DCC_REQUIRE(word, DCC_ERR_CUDA, "status word unavailable");
    cudaStream_t st = as_stream(stream);
    if (cudaMemcpyAsync(out, word, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess || cudaMemsetAsync(word, 0, sizeof(int), st) != cudaSuccess)
        return launch_status("symmetrize status");
    return DCC_OK;
}

extern "C" int dcc_take_t3_batched(const double *t3_local, double *out, const int32_t *ijk,
                                   const int64_t *ijk_to_local_idx, int64_t count, int64_t nocc, int64_t nvir,
                                   void *stream) {
    clear_error();
    DCC_REQUIRE(count >= 0 && nocc >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (count == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t3_local && out && ijk && ijk_to_local_idx, DCC_ERR_NULL, "NULL buffer");
    int ntile = (int)ceil_div(nvir, TE);
    int64_t nt3 = (int64_t)ntile * ntile * ntile;
    int64_t gy = (148 * 8 * 8 + nt3 - 1) / nt3;
    gy = gy < 1 ? 1 : (gy > count ? count : gy);
    gy = gy > 65535 ? 65535 : gy;
    dim3 grid((unsigned)nt3, (unsigned)gy);
    k_take_t3<<<grid, OT_THREADS, 0, as_stream(stream)>>>(t3_local, out, ijk, ijk_to_local_idx, count, (int)nocc,
                                                          (int)nvir, ntile);
    return launch_status("take_t3");
}

extern "C" int dcc_take_t3_ijk_single(const double *t3_local, double *t3_blk, const int64_t *ijk_to_local_idx,
                                      int64_t i, int64_t j, int64_t k, int64_t nocc, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(i >= 0 && j >= 0 && k >= 0 && i < nocc && j < nocc && k < nocc, DCC_ERR_SHAPE,
                "occupied index out of range");
    DCC_REQUIRE(ijk_to_local_idx && t3_local && t3_blk, DCC_ERR_NULL, "NULL buffer");
    int64_t s[3];
    int cs = order_case3(i, j, k, s);
    int64_t loc = ijk_to_local_idx[ijk_linear(s[0], s[1], s[2], nocc)];
    if (loc < 0) {
        set_error("block (%lld,%lld,%lld) is not stored", (long long)s[0], (long long)s[1], (long long)s[2]);
        return DCC_ERR_NOT_LOCAL;
    }
    (void)cs;
    int ntile = (int)ceil_div(nvir, TE);
    k_take_t3_one<<<dim3((unsigned)(ntile * ntile * ntile)), OT_THREADS, 0, as_stream(stream)>>>(
        t3_local, t3_blk, (int)i, (int)j, (int)k, loc, (int)nvir, ntile);
    return launch_status("take_t3_ijk_single");
}

extern "C" int dcc_fill_local_data_ijk(const double *t3_local, double *send_data, const int32_t *requests,
                                       const int64_t *ijk_to_local_idx, int64_t n_requests, int64_t nvir,
                                       void *stream) {
    clear_error();
    DCC_REQUIRE(n_requests >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (n_requests == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t3_local && send_data && requests && ijk_to_local_idx, DCC_ERR_NULL, "NULL buffer");
    int64_t blk = nvir * nvir * nvir;
    dim3 grid(ceil_div(blk, 256 * 4) < 64 ? ceil_div(blk, 256 * 4) : 64,
              (unsigned)(n_requests < 65535 ? n_requests : 65535));
    k_copy_blocks<<<grid, 256, 0, as_stream(stream)>>>(t3_local, send_data, requests, ijk_to_local_idx, n_requests,
                                                       blk);
    return launch_status("fill_local_data_ijk");
}

extern "C" int dcc_r3_tri_divide_e(double *r3, const double *eia, const int32_t *ijk, int64_t nblocks, int64_t nvir,
                                   void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(r3 && eia && ijk, DCC_ERR_NULL, "NULL buffer");
    k_r3_divide<<<row_grid(nblocks * nvir * nvir, 256), 256, 0, as_stream(stream)>>>(r3, eia, ijk, nblocks, (int)nvir);
    return launch_status("r3_tri_divide_e");
}

extern "C" size_t dcc_t3_update_workspace_bytes(int64_t nblocks, int64_t nvir) {
    if (nblocks <= 0 || nvir <= 0) return 16;
    return (size_t)row_grid(nblocks * nvir * nvir, UPD_THREADS) * 2 * sizeof(double);
}

extern "C" int dcc_t3_divide_update(double *t3, double *r3, const double *eia, const int32_t *ijk, int64_t nblocks,
                                    int64_t nvir, int64_t nvir_active, int write_r3, double *norms, void *workspace,
                                    size_t workspace_bytes, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE(norms, DCC_ERR_NULL, "norms is NULL");
    cudaStream_t st = as_stream(stream);
    if (nblocks == 0 || nvir == 0) {
        if (cudaMemsetAsync(norms, 0, 2 * sizeof(double), st) != cudaSuccess) return launch_status("memset");
        return DCC_OK;
    }
    DCC_REQUIRE(t3 && r3 && eia && ijk && workspace, DCC_ERR_NULL, "NULL buffer");
    size_t need = dcc_t3_update_workspace_bytes(nblocks, nvir);
    DCC_REQUIRE(workspace_bytes >= need, DCC_ERR_WORKSPACE, "workspace needs %zu bytes, got %zu", need,
                workspace_bytes);
    if (nvir_active < 0 || nvir_active > nvir) nvir_active = nvir;
    unsigned grid = row_grid(nblocks * nvir * nvir, UPD_THREADS);
    k_t3_divide_update<<<grid, UPD_THREADS, 0, st>>>(t3, r3, eia, ijk, nblocks, (int)nvir, (int)nvir_active,
                                                      write_r3, (double *)workspace);
    int rc = launch_status("t3_divide_update");
    if (rc) return rc;
    k_sum_pairs<<<1, 256, 0, st>>>((const double *)workspace, (int64_t)grid, norms);
    return launch_status("t3_divide_update reduce");
}

extern "C" int dcc_redistribute_ijk_to_abc(const double *t3_ijk, double *t3_abc, int64_t nocc, int64_t nvir,
                                           void *stream) {
    clear_error();
    DCC_REQUIRE(nocc >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nocc == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t3_ijk && t3_abc, DCC_ERR_NULL, "NULL buffer");
    int64_t nabc = nvir * (nvir + 1) * (nvir + 2) / 6;
    int64_t o3 = nocc * nocc * nocc;
    dim3 grid(ceil_div(o3, 256) < 16 ? ceil_div(o3, 256) : 16, (unsigned)(nabc < 65535 ? nabc : 65535));
    k_ijk_to_abc<<<grid, 256, 0, as_stream(stream)>>>(t3_ijk, t3_abc, (int)nocc, (int)nvir, nabc);
    return launch_status("redistribute_ijk_to_abc");
}

extern "C" int dcc_fill_t3_from_abc(double *target, int64_t a0, int64_t a1, int64_t b0, int64_t b1, int64_t nvir,
                                    int64_t nocc, const double *t3_abc, int64_t ld_b, void *stream) {
    clear_error();
    DCC_REQUIRE(0 <= a0 && a0 <= a1 && a1 <= nvir && 0 <= b0 && b0 <= b1 && b1 <= nvir, DCC_ERR_SHAPE,
                "virtual range out of bounds");
    DCC_REQUIRE(ld_b >= b1 - b0, DCC_ERR_SHAPE, "ld_b smaller than the b range");
    if (a1 == a0 || b1 == b0 || nocc == 0) return DCC_OK;
    DCC_REQUIRE(target && t3_abc, DCC_ERR_NULL, "NULL buffer");
    int64_t o3 = nocc * nocc * nocc;
    DCC_REQUIRE(o3 * 8 <= 200 * 1024, DCC_ERR_UNSUPPORTED, "nocc^3 block exceeds shared memory");
    int64_t nwork = (a1 - a0) * (b1 - b0) * nvir;
    unsigned grid = (unsigned)(nwork < 148 * 16 ? nwork : 148 * 16);
    size_t smem = (size_t)o3 * sizeof(double);
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_fill_t3_abc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_fill_t3_abc<<<grid, 256, smem, as_stream(stream)>>>(target, (int)a0, (int)a1, (int)b0, (int)b1, (int)nvir,
                                                          (int)nocc, t3_abc, ld_b);
    return launch_status("fill_t3_from_abc");
}

// ---------------------------------------------------------------- unpack every ordering

namespace dcc {

// U[(x*nocc + y)*nocc + z] = T3[x,y,z] for every ordered (x,y,z), from the
// canonical blocks.  A CTA owns one canonical tile triple: it loads the
// orbit set of block q once and writes it to each distinct ordering of q's
// triple (up to 6 output blocks x up to 6 tiles), every output tile being a
// permuted tile of the same set.
__global__ void __launch_bounds__(OT_THREADS) k_unpack_all(const double *t3, double *U, int64_t nblocks, int nocc,
                                                           int nv, int ntile) {
    extern __shared__ double sm[];  // 2 x 6 x SLOT
    __shared__ OrbitSet os;
    __shared__ int qtrip[3];
    int t0, t1, t2;
    decode_tri3(blockIdx.x, ntile, t0, t1, t2);
    build_orbit_set(os, t0, t1, t2);
    const int64_t n3 = (int64_t)nv * nv * nv;
    const int pinv[6] = {0, 1, 2, 4, 3, 5};  // inverse of each axis map
    // even nvir: every row starts on 16 bytes (U 16-byte aligned), so threads write (z, z+1) pairs
    const bool vec = (nv & 1) == 0 && ((uintptr_t)U & 15) == 0 && blockDim.x == TE3 / 2;
    const int px = threadIdx.x >> 5, py = (threadIdx.x >> 2) & 7, pz = (threadIdx.x & 3) * 2;
    const int64_t prel = ((int64_t)px * nv + py) * nv + pz;
    int64_t q = blockIdx.y;
    if (q >= nblocks) return;
    load_orbit_tiles_async(sm, os, t3 + q * n3, nv);
    cp_async_commit();
    for (int stage = 0; q < nblocks; q += gridDim.y, stage ^= 1) {
        const int64_t nq = q + gridDim.y;
        if (nq < nblocks) {
            load_orbit_tiles_async(sm + (stage ^ 1) * 6 * SLOT, os, t3 + nq * n3, nv);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        if (threadIdx.x == 0) {
            // canonical triple of block q (lexicographic rank -> i<=j<=k)
            int a, b, c;
            decode_tri3(q, nocc, a, b, c);
            qtrip[0] = a;
            qtrip[1] = b;
            qtrip[2] = c;
        }
        __syncthreads();
        const double *buf = sm + stage * 6 * SLOT;
        const int o[3] = {qtrip[0], qtrip[1], qtrip[2]};
        for (int sg = 0; sg < 6; sg++) {
            const int xyz[3] = {o[perm3(sg, 0)], o[perm3(sg, 1)], o[perm3(sg, 2)]};
            bool dup = false;  // the same ordered triple from an earlier map (repeated indices)
            for (int sp = 0; sp < sg; sp++)
                if (o[perm3(sp, 0)] == xyz[0] && o[perm3(sp, 1)] == xyz[1] && o[perm3(sp, 2)] == xyz[2]) dup = true;
            if (dup) continue;
            int64_t srt[3];
            const int cs = order_case3(xyz[0], xyz[1], xyz[2], srt);
            const int pi = pinv[cs];
            double *dst = U + (((int64_t)xyz[0] * nocc + xyz[1]) * nocc + xyz[2]) * n3;
            if (vec) {
                // one 16-byte pair (z, z+1) per thread: its two shared-memory sources for this
                // axis map, then one store per tile of the set
                auto c0 = [&](int m) { return m == 0 ? px : (m == 1 ? py : pz); };
                auto c1 = [&](int m) { return m == 0 ? px : (m == 1 ? py : pz + 1); };
                const int off0 = sidx(c0(perm3(pi, 0)), c0(perm3(pi, 1)), c0(perm3(pi, 2)));
                const int off1 = sidx(c1(perm3(pi, 0)), c1(perm3(pi, 1)), c1(perm3(pi, 2)));
                for (int s = 0; s < os.nslot; s++) {
                    const int X0 = os.tile[s][0] * TE, Y0 = os.tile[s][1] * TE, Z0 = os.tile[s][2] * TE;
                    if (X0 + px >= nv || Y0 + py >= nv || Z0 + pz >= nv) continue;
                    const double *b = buf + os.nbr[s][pi] * SLOT;
                    *(double2 *)(dst + ((int64_t)X0 * nv + Y0) * nv + Z0 + prel) = make_double2(b[off0], b[off1]);
                }
                continue;
            }
            for (int s = 0; s < os.nslot; s++) {
                const int src_slot = os.nbr[s][pi];
                const int X0 = os.tile[s][0] * TE, Y0 = os.tile[s][1] * TE, Z0 = os.tile[s][2] * TE;
                for (int e = threadIdx.x; e < TE3; e += blockDim.x) {
                    const int u[3] = {e >> 6, (e >> 3) & 7, e & 7};
                    const int gx = X0 + u[0], gy = Y0 + u[1], gz = Z0 + u[2];
                    if (gx >= nv || gy >= nv || gz >= nv) continue;
                    dst[((int64_t)gx * nv + gy) * nv + gz] =
                        buf[src_slot * SLOT + sidx(u[perm3(pi, 0)], u[perm3(pi, 1)], u[perm3(pi, 2)])];
                }
            }
        }
        __syncthreads();
    }
}

// Unpack of every ordering by output row bands (even nvir, 16-byte aligned buffers).  A work
// item is one ordered output block U[x,y,z] and one band of 8 x 8 of its rows (all of c): one
// thread loads the band's source tiles (one 8^3 TMA box per output tile, from the canonical
// block with its axes permuted), the CTA transposes them into a dense [8][8][nvir] band in
// shared memory (lanes/steps follow tile_element, so the permuted tile reads are free of bank
// conflicts), and the band goes out as one TMA store of whole rows.  Whole rows reach DRAM as
// whole lines, where the orbit-tile kernel's 64-byte row pieces did not.  Items run
// block-major, so the orderings of one canonical block read it from L2.
// NB source buffers and NB band buffers per CTA of NT threads (with NB = 2 the tiles of the
// next item load while the current band is transposed).  The launcher runs NB = 1 with two
// CTAs per SM: one CTA of 16 warps with NB = 2 measured 1.9x slower.
template <int NB, int NT>
__global__ void __launch_bounds__(NT, NB == 2 ? 1 : 2)
    k_unpack_band(const __grid_constant__ CUtensorMap src, const __grid_constant__ CUtensorMap dst, int64_t nblocks,
                  int nocc, int nv, int ntile, int *status) {
    extern __shared__ __align__(128) double sm[];  // NB x ntile x TE3 source tiles, then NB x 8 x 8 x nv bands
    const size_t tile_dbl = (size_t)ntile * TE3, band_dbl = (size_t)TE * TE * nv;
    __shared__ __align__(8) uint64_t bar[NB];
    __shared__ int s_ok;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int STEPS = 16 / (NT / 32);  // tile_element steps per warp and tile
    const int pinv[6] = {0, 1, 2, 4, 3, 5};  // inverse of each axis map
    const int64_t per_q = 6 * (int64_t)ntile * ntile, nwork = nblocks * per_q;
    struct Item {
        int64_t w;
        int64_t out;  // output block (x * nocc + y) * nocc + z
        int q, pi, X, Y;
    };
    // the first item at or after wi (stepping by the grid) whose ordering is new for its block
    auto next_item = [&](int64_t wi) {
        Item it{};
        for (; wi < nwork; wi += gridDim.x) {
            const int64_t q = wi / per_q;
            const int g = (int)((wi / ((int64_t)ntile * ntile)) % 6);
            int o[3];
            decode_tri3(q, nocc, o[0], o[1], o[2]);
            const int xyz[3] = {o[perm3(g, 0)], o[perm3(g, 1)], o[perm3(g, 2)]};
            bool dup = false;
            for (int sp = 0; sp < g; sp++)
                if (o[perm3(sp, 0)] == xyz[0] && o[perm3(sp, 1)] == xyz[1] && o[perm3(sp, 2)] == xyz[2]) dup = true;
            if (dup) continue;
            int64_t srt[3];
            it.pi = pinv[order_case3(xyz[0], xyz[1], xyz[2], srt)];
            it.out = ((int64_t)xyz[0] * nocc + xyz[1]) * nocc + xyz[2];
            it.q = (int)q;
            const int xy = (int)(wi % ((int64_t)ntile * ntile));
            it.X = xy / ntile;
            it.Y = xy % ntile;
            break;
        }
        it.w = wi;
        return it;
    };
    auto issue = [&](const Item &it, int bi) {  // thread 0: the band's source tiles into buffer bi
        const uint32_t b = smem_u32(&bar[bi]);
        mbar_expect_tx(b, (uint32_t)ntile * TE3 * 8);
        for (int zt = 0; zt < ntile; zt++) {
            const int T[3] = {it.X, it.Y, zt};
            tma_load_5d(smem_u32(sm + bi * tile_dbl + zt * TE3), &src, b, T[perm3(it.pi, 2)] * TE,
                        T[perm3(it.pi, 1)] * TE, T[perm3(it.pi, 0)] * TE, it.q, 0);
        }
    };
    if (threadIdx.x == 0) {
        for (int i = 0; i < NB; i++) mbar_init(smem_u32(&bar[i]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    Item cur = next_item(blockIdx.x);
    if (cur.w >= nwork) return;
    Item ahead = cur;  // the last item whose loads were issued
    if (threadIdx.x == 0) issue(cur, 0);
    for (int i = 1; i < NB; i++) {
        ahead = next_item(ahead.w + gridDim.x);
        if (threadIdx.x == 0 && ahead.w < nwork) issue(ahead, i);
    }
    for (int n = 0; cur.w < nwork; n++) {
        const int bi = n % NB;
        const uint32_t par = (uint32_t)(n / NB) & 1u;
        if (threadIdx.x == 0) {
            bulk_wait_read<NB - 1>();  // the store that last used band buffer bi has read it
            s_ok = p3_wait_bounded(smem_u32(&bar[bi]), par, status);
            if (!s_ok) {  // drain this CTA's copies in flight, then leave
                for (int i = 0; i < NB; i++) mbar_wait_quiet(smem_u32(&bar[(n + i) % NB]), (uint32_t)((n + i) / NB) & 1u);
                bulk_wait<0>();
            }
        }
        __syncthreads();
        if (!s_ok) return;
        mbar_wait_quiet(smem_u32(&bar[bi]), par);  // complete already: acquires the tiles
        const double *tiles = sm + bi * tile_dbl;
        double *band = sm + NB * tile_dbl + bi * band_dbl;
        const int p0 = perm3(cur.pi, 0), p1 = perm3(cur.pi, 1), p2 = perm3(cur.pi, 2);
        // this thread's elements of every output tile: source offset in the tile, band offset, z
        int soff[STEPS], boff[STEPS], zl[STEPS];
#pragma unroll
        for (int jj = 0; jj < STEPS; jj++) {
            int u[3];
            tile_element(lane, w * STEPS + jj, u);
            auto sel = [&](int m) { return m == 0 ? u[0] : (m == 1 ? u[1] : u[2]); };
            soff[jj] = (sel(p0) * TE + sel(p1)) * TE + sel(p2);
            boff[jj] = (u[0] * TE + u[1]) * nv + u[2];
            zl[jj] = u[2];
        }
        for (int zt = 0; zt < ntile; zt++) {
            const double *tl = tiles + zt * TE3;
            const int zrem = nv - zt * TE;  // elements of this tile inside the row
#pragma unroll
            for (int jj = 0; jj < STEPS; jj++)
                if (zl[jj] < zrem) band[boff[jj] + zt * TE] = tl[soff[jj]];
        }
        fence_proxy_async_smem();  // the band becomes visible to the TMA store
        __syncthreads();           // every thread is done with the source tiles
        ahead = next_item(ahead.w + gridDim.x);
        if (threadIdx.x == 0) {
            if (ahead.w < nwork) issue(ahead, bi);  // buffer bi is free again
            tma_store_5d(&dst, smem_u32(band), 0, cur.Y * TE, cur.X * TE, (int)cur.out, 0);
            bulk_commit();
        }
        cur = next_item(cur.w + gridDim.x);
    }
    if (threadIdx.x == 0) bulk_wait<0>();
}

}  // namespace dcc

namespace dcc {

// The unpack of every ordering for nvir <= 104 by strips.  A work item is a canonical block C, an
// ordering, one fixed index x and a tile of 32 values y0.. of another; it writes the 32 output rows
// U[o][x][y][:] (or U[o][y][x][:]).  When the ordering keeps c the fastest axis of C (two of the
// six) those rows are whole rows of C, loaded two output rows at a time with every load issued
// before the stores; otherwise each output row is a column of C (c as C's middle or first axis),
// and the item stages the strip C[..c..][x][y0..y0+31] for every c in shared memory (8-byte copies
// of 256-byte segments; row pitch 33 doubles) before its warps write the rows.  Items run
// canonical block by canonical block, so the orderings of a block reuse it from L2.
constexpr int US_W = 32, US_PITCH = 33, US_MAXNV = 104;

// UT: the type of U (double; float for the FP32 copy of the split precisions, each value rounded
// once)
template <typename UT>
__global__ void __launch_bounds__(256, 4) k_unpack_strips(const double *__restrict__ t3, UT *__restrict__ U,
                                                          int64_t nblocks, int nocc, int nv, int ntile) {
    __shared__ double T[US_MAXNV * US_PITCH];  // T[c][j]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t n3 = (int64_t)nv * nv * nv, nv2 = (int64_t)nv * nv;
    const int64_t per_g = (int64_t)nv * ntile, per_q = 6 * per_g, nwork = nblocks * per_q;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t q = w / per_q;
        const int rem = (int)(w - q * per_q), g = rem / (int)per_g, r2 = rem - g * (int)per_g;
        const int x = r2 / ntile, y0 = (r2 - x * ntile) * US_W, h = nv - y0 < US_W ? nv - y0 : US_W;
        int o[3];
        decode_tri3(q, nocc, o[0], o[1], o[2]);
        const int xyz[3] = {o[perm3(g, 0)], o[perm3(g, 1)], o[perm3(g, 2)]};
        bool dup = false;
        for (int sp = 0; sp < g; sp++)
            if (o[perm3(sp, 0)] == xyz[0] && o[perm3(sp, 1)] == xyz[1] && o[perm3(sp, 2)] == xyz[2]) dup = true;
        if (dup) continue;  // uniform over the CTA
        int64_t srt[3];
        const int cs = order_case3(xyz[0], xyz[1], xyz[2], srt);
        const int pi = cs == 3 ? 4 : (cs == 4 ? 3 : cs);  // U[o][u] = C[u[perm3(pi, 0)], u[perm3(pi, 1)], u[perm3(pi, 2)]]
        const double *C = t3 + q * n3;
        UT *Uo = U + (((int64_t)xyz[0] * nocc + xyz[1]) * nocc + xyz[2]) * n3;
        // x is a for pi = 0, 1, 4 (rows U[x][y][:]) and b for 2, 3, 5 (rows U[y][x][:])
        const bool xa = pi == 0 || pi == 1 || pi == 4;
        const int64_t ostep = xa ? nv : nv2;  // output row y0 + j at Uo + obase + j * ostep
        const int64_t obase = xa ? x * nv2 + (int64_t)y0 * nv : (int64_t)y0 * nv2 + x * nv;
        if (pi == 0 || pi == 2) {  // whole rows: C[x][y][:] (pi 0: U[x][y] = C[x][y]; pi 2: U[y][x] = C[x][y])
            const double *src = C + x * nv2 + (int64_t)y0 * nv;
            for (int j = warp; j < h; j += 16) {
                double v[2][4];
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const bool ok = j + 8 * e < h;
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        const int c = lane + 32 * m;
                        v[e][m] = ok && c < nv ? __ldg(src + (int64_t)(j + 8 * e) * nv + c) : 0.0;
                    }
                }
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    if (j + 8 * e >= h) continue;
                    UT *dst = Uo + obase + (int64_t)(j + 8 * e) * ostep;
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        const int c = lane + 32 * m;
                        if (c < nv) dst[c] = (UT)v[e][m];
                    }
                }
            }
            continue;
        }
        // columns: U[x][y][c] = C[x][c][y] (pi 1), C[c][x][y] (pi 4); U[y][x][c] = C[x][c][y] (pi 3),
        // C[c][x][y] (pi 5)
        const int64_t sc = (pi == 1 || pi == 3) ? nv : nv2, sx = (pi == 1 || pi == 3) ? nv2 : nv;
        const double *src = C + x * sx + y0;
        for (int c = warp; c < nv; c += 8)
            if (lane < h) cp_async8(T + c * US_PITCH + lane, src + c * sc + lane);
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        for (int j = warp; j < h; j += 8) {
            UT *dst = Uo + obase + (int64_t)j * ostep;
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int c = lane + 32 * m;
                if (c < nv) dst[c] = (UT)T[c * US_PITCH + j];
            }
        }
        __syncthreads();  // the strip is refilled by the next item
    }
}

}  // namespace dcc

// The strip unpack for nvir <= 104; DCC_ERR_UNSUPPORTED (nothing launched) where it does not apply.
template <typename UT>
static int unpack_strips_launch(const double *t3, UT *U, int64_t nocc, int64_t nvir, void *stream) {
    const int64_t nblocks = nocc * (nocc + 1) * (nocc + 2) / 6;
    if (nvir > US_MAXNV || nocc * nocc * nocc >= (1ll << 31) || nblocks >= (1ll << 31) || nocc > 1290)
        return DCC_ERR_UNSUPPORTED;
    const int nst = (int)ceil_div(nvir, US_W);
    int dev = 0, nsm = 148, per_sm = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unpack_strips<UT>, 256, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t nwork = nblocks * 6 * nvir * (int64_t)nst, cap = (int64_t)nsm * per_sm;
    const unsigned grid = (unsigned)(nwork < cap ? nwork : cap);
    k_unpack_strips<UT><<<grid, 256, 0, as_stream(stream)>>>(t3, U, nblocks, (int)nocc, (int)nvir, nst);
    return DCC_OK;
}

extern "C" int dcc_t3_unpack_all_f32(const double *t3, float *U, int64_t nocc, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nocc >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nocc == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t3 && U && (const void *)t3 != (const void *)U, DCC_ERR_NULL, "NULL or aliased buffer");
    DCC_REQUIRE(unpack_strips_launch(t3, U, nocc, nvir, stream) == DCC_OK, DCC_ERR_UNSUPPORTED,
                "the FP32 unpack needs nvir <= %d", US_MAXNV);
    return launch_status("t3_unpack_all_f32");
}

extern "C" int dcc_t3_unpack_all(const double *t3, double *U, int64_t nocc, int64_t nvir, void *stream) {
    clear_error();
    DCC_REQUIRE(nocc >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    if (nocc == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(t3 && U && t3 != U, DCC_ERR_NULL, "NULL or aliased buffer");
    const int64_t nblocks = nocc * (nocc + 1) * (nocc + 2) / 6;
    int ntile = (int)ceil_div(nvir, TE);
    {
        // whole rows, columns through staged strips (k_unpack_strips); the kernel for odd nvir
        if (unpack_strips_launch(t3, U, nocc, nvir, stream) == DCC_OK) return launch_status("t3_unpack_all");
    }
    {
        // band kernel: even nvir (16-byte rows), aligned buffers, box sides <= 256, shared memory
        const size_t bsm = ((size_t)ntile * TE3 + (size_t)TE * TE * nvir) * sizeof(double);
        EncodeTiledFn fn = encode_fn();
        int *status = sym_status_word();
        if (nvir % 2 == 0 && nvir <= 256 && bsm <= 200 * 1024 && ((uintptr_t)t3 & 15) == 0 &&
            ((uintptr_t)U & 15) == 0 && nocc * nocc * nocc < (1ll << 31) && fn && status) {
            const cuuint64_t nv = (cuuint64_t)nvir, n3 = nv * nv * nv;
            const cuuint64_t sdims[5] = {nv, nv, nv, (cuuint64_t)nblocks, 1};
            const cuuint64_t ddims[5] = {nv, nv, nv, (cuuint64_t)(nocc * nocc * nocc), 1};
            const cuuint64_t sstr[4] = {nv * 8, nv * nv * 8, n3 * 8, n3 * 8 * (cuuint64_t)nblocks};
            const cuuint64_t dstr[4] = {nv * 8, nv * nv * 8, n3 * 8, n3 * 8 * (cuuint64_t)(nocc * nocc * nocc)};
            const cuuint32_t sbox[5] = {TE, TE, TE, 1, 1}, dbox[5] = {(cuuint32_t)nvir, TE, TE, 1, 1};
            const cuuint32_t es[5] = {1, 1, 1, 1, 1};
            CUtensorMap ms, md;
            if (fn(&ms, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double *>(t3), sdims, sstr, sbox, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
                fn(&md, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, U, ddims, dstr, dbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS) {
                int dev = 0, nsm = 148;
                if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
                const int64_t nwork = nblocks * 6 * (int64_t)ntile * ntile;
                // one buffer and two CTAs of 8 warps per SM (two buffers in one CTA of 16 warps measured
                // 1.9x slower at nocc = 10, nvir = 90)
                const int64_t cap = (int64_t)nsm * (bsm <= 100 * 1024 ? 2 : 1);
                const unsigned grid = (unsigned)(nwork < cap ? nwork : cap);
                cudaFuncSetAttribute(k_unpack_band<1, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm);
                k_unpack_band<1, 256><<<grid, 256, bsm, as_stream(stream)>>>(ms, md, nblocks, (int)nocc, (int)nvir, ntile,
                                                                             status);
                return launch_status("t3_unpack_all");
            }
        }
    }
    int64_t ntri = (int64_t)ntile * (ntile + 1) * (ntile + 2) / 6;
    int64_t gy = (148 * 4 * 8 + ntri - 1) / ntri;
    gy = gy < 1 ? 1 : (gy > nblocks ? nblocks : gy);
    size_t smem = 2 * 6 * SLOT * sizeof(double);
    cudaFuncSetAttribute(k_unpack_all, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_unpack_all<<<dim3((unsigned)ntri, (unsigned)gy), OT_THREADS, smem, as_stream(stream)>>>(t3, U, nblocks, (int)nocc,
                                                                                            (int)nvir, ntile);
    return launch_status("t3_unpack_all");
}

// ---------------------------------------------------------------- permutation gather

namespace dcc {

constexpr int PG_MAX_SRC = 4;
constexpr int PG_MAX_SLOTS = 12;

struct PermSrc {
    const double *base;
    double scale;
    int64_t st[6];  // strides of (x, y, z, a, b, c)
    int mask;       // bit p set: include the simultaneous permutation p
};

struct PermGatherArgs {
    PermSrc src[PG_MAX_SRC];
    int nsrc, nslot;
    int slot_src[PG_MAX_SLOTS], slot_perm[PG_MAX_SLOTS];
    double slot_scale[PG_MAX_SLOTS];
};

// r3[q][a][b][c] = beta*r3 + sum_s scale_s sum_{p in mask_s} U_s(p(ijk), p(abc)).
// A CTA owns one 8^3 output tile and walks the blocks q; the source tiles of
// the next block are copied while the current block is summed.  The virtual
// part of every source offset and every shared address depend only on the
// tile, so each thread computes them once (2 elements x up to 12 slots).
__global__ void __launch_bounds__(256) k_perm_gather(double *r3, const int32_t *ijk, int64_t nblocks, int nv,
                                                     int ntile, double beta, PermGatherArgs g) {
    extern __shared__ double pg_sm[];  // 2 x nslot x SLOT
    const int T[3] = {(int)(blockIdx.x / (ntile * ntile)), (int)((blockIdx.x / ntile) % ntile),
                      (int)(blockIdx.x % ntile)};
    const int64_t n3 = (int64_t)nv * nv * nv;
    int voff[PG_MAX_SLOTS][2];            // virtual offset of the copied source element, -1: none
    unsigned short rd[PG_MAX_SLOTS][2];   // shared address read for output element h
    unsigned short wr[2];                 // shared address the copy of element h lands at (per slot base added)
    int ooff[2];                          // output element offset in the block, -1: outside
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int e = threadIdx.x + 256 * h;
        const int u[3] = {e >> 6, (e >> 3) & 7, e & 7};
        wr[h] = (unsigned short)sidx(u[0], u[1], u[2]);
        const int ga = T[0] * TE + u[0], gb = T[1] * TE + u[1], gc = T[2] * TE + u[2];
        ooff[h] = (ga < nv && gb < nv && gc < nv) ? (ga * nv + gb) * nv + gc : -1;
#pragma unroll
        for (int sl = 0; sl < PG_MAX_SLOTS; sl++) {
            voff[sl][h] = -1;
            rd[sl][h] = 0;
            if (sl >= g.nslot) continue;
            const PermSrc &S = g.src[g.slot_src[sl]];
            const int p = g.slot_perm[sl];
            // copy: slot tile = p(T), element u in the source's own order
            const int TT[3] = {T[perm3(p, 0)], T[perm3(p, 1)], T[perm3(p, 2)]};
            const int sa = TT[0] * TE + u[0], sb = TT[1] * TE + u[1], sc = TT[2] * TE + u[2];
            if (sa < nv && sb < nv && sc < nv) voff[sl][h] = (int)(sa * S.st[3] + sb * S.st[4] + sc * S.st[5]);
            // read: output element u needs the source element p(u) of the slot
            rd[sl][h] = (unsigned short)(sl * SLOT + sidx(u[perm3(p, 0)], u[perm3(p, 1)], u[perm3(p, 2)]));
        }
    }
    auto issue = [&](double *buf, int64_t q) {
        const int o[3] = {ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]};
#pragma unroll
        for (int sl = 0; sl < PG_MAX_SLOTS; sl++) {
            if (sl >= g.nslot) continue;
            const PermSrc &S = g.src[g.slot_src[sl]];
            const int p = g.slot_perm[sl];
            const double *base = S.base + o[perm3(p, 0)] * S.st[0] + o[perm3(p, 1)] * S.st[1] + o[perm3(p, 2)] * S.st[2];
#pragma unroll
            for (int h = 0; h < 2; h++)
                if (voff[sl][h] >= 0) cp_async8(buf + sl * SLOT + wr[h], base + voff[sl][h]);
        }
    };
    int64_t q = blockIdx.y;
    if (q >= nblocks) return;
    issue(pg_sm, q);
    cp_async_commit();
    for (int stage = 0; q < nblocks; q += gridDim.y, stage ^= 1) {
        const int64_t nq = q + gridDim.y;
        if (nq < nblocks) {
            issue(pg_sm + (stage ^ 1) * g.nslot * SLOT, nq);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double *buf = pg_sm + stage * g.nslot * SLOT;
        double *dst = r3 + q * n3;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            if (ooff[h] < 0) continue;
            double acc = 0.0;
#pragma unroll
            for (int sl = 0; sl < PG_MAX_SLOTS; sl++)
                if (sl < g.nslot) acc = fma(g.slot_scale[sl], buf[rd[sl][h]], acc);
            double *out = dst + ooff[h];
            *out = (beta == 0.0) ? acc : fma(beta, *out, acc);
        }
        __syncthreads();
    }
}

}  // namespace dcc

extern "C" int dcc_t3_perm_gather(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nvir, double beta,
                                  int nsrc, const double *const *bases, const double *scales, const int64_t *strides,
                                  const int *masks, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE(nsrc >= 1 && nsrc <= PG_MAX_SRC, DCC_ERR_SHAPE, "1..%d sources", PG_MAX_SRC);
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(r3 && ijk && bases && scales && strides && masks, DCC_ERR_NULL, "NULL argument");
    PermGatherArgs g{};
    g.nsrc = nsrc;
    int nslot = 0;
    for (int s = 0; s < nsrc; s++) {
        DCC_REQUIRE(bases[s], DCC_ERR_NULL, "source %d is NULL", s);
        DCC_REQUIRE(masks[s] > 0 && masks[s] < 64, DCC_ERR_SHAPE, "source %d: permutation mask must be in 1..63", s);
        g.src[s].base = bases[s];
        g.src[s].scale = scales[s];
        for (int m = 0; m < 6; m++) g.src[s].st[m] = strides[6 * s + m];
        g.src[s].mask = masks[s];
        for (int p = 0; p < 6; p++)
            if (masks[s] & (1 << p)) {
                DCC_REQUIRE(nslot < PG_MAX_SLOTS, DCC_ERR_UNSUPPORTED, "more than %d source tiles", PG_MAX_SLOTS);
                g.slot_src[nslot] = s;
                g.slot_perm[nslot] = p;
                g.slot_scale[nslot] = scales[s];
                nslot++;
            }
    }
    g.nslot = nslot;
    for (int s = 0; s < nsrc; s++) {
        const int64_t vmax = (nvir + 7) / 8 * 8 * (g.src[s].st[3] + g.src[s].st[4] + g.src[s].st[5]);
        DCC_REQUIRE(g.src[s].st[3] >= 0 && g.src[s].st[4] >= 0 && g.src[s].st[5] >= 0 && vmax < (1ll << 31),
                    DCC_ERR_UNSUPPORTED, "source %d: virtual strides must be non-negative and span < 2^31", s);
    }
    DCC_REQUIRE(nvir <= 1290, DCC_ERR_UNSUPPORTED, "nvir > 1290 exceeds 32-bit block offsets");
    int ntile = (int)ceil_div(nvir, TE);
    int64_t nt3 = (int64_t)ntile * ntile * ntile;
    int64_t gy = (148 * 4 * 8 + nt3 - 1) / nt3;
    gy = gy < 1 ? 1 : (gy > nblocks ? nblocks : gy);
    gy = gy > 65535 ? 65535 : gy;
    size_t smem = (size_t)2 * nslot * SLOT * sizeof(double);
    cudaFuncSetAttribute(k_perm_gather, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_perm_gather<<<dim3((unsigned)nt3, (unsigned)gy), 256, smem, as_stream(stream)>>>(r3, ijk, nblocks, (int)nvir,
                                                                                       ntile, beta, g);
    return launch_status("t3_perm_gather");
}

extern "C" int dcc_t3_s3_gather(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nvir, double beta,
                                const double *u0, double scale0, const int64_t *strides0, const double *u1,
                                double scale1, const int64_t *strides1, void *stream) {
    clear_error();
    DCC_REQUIRE(u0 && strides0, DCC_ERR_NULL, "first source is NULL");
    const double *bases[2] = {u0, u1};
    double scales[2] = {scale0, scale1};
    int64_t st[12];
    for (int m = 0; m < 6; m++) {
        st[m] = strides0[m];
        st[6 + m] = u1 ? strides1[m] : 0;
    }
    int masks[2] = {63, 63};
    if (u1) DCC_REQUIRE(strides1, DCC_ERR_NULL, "strides1 is NULL");
    return dcc_t3_perm_gather(r3, ijk, nblocks, nvir, beta, u1 ? 2 : 1, bases, scales, st, masks, stream);
}

// ---------------------------------------------------------------- permutation gather, TMA pipeline

namespace dcc {

constexpr int TG_WARPS = 8;                   // compute warps
constexpr int TG_THREADS = 32 * (TG_WARPS + 1);  // + one producer warp
constexpr uint32_t TG_TILE_BYTES = TE3 * 8;   // one dense 8x8x8 FP64 tile
constexpr int TG_SMEM_BUDGET = 200 * 1024;

struct TmaMaps {
    CUtensorMap m[PG_MAX_SRC + 1];  // sources, then r3
};

struct TmaGatherArgs {
    int nslot;  // (source, permutation) pairs
    double slot_scale[PG_MAX_SLOTS];
    int slot_perm[PG_MAX_SLOTS];
    // per load (slots, then the r3 tile): map, output-tile axis feeding c / b / a,
    // block-coordinate coefficients of (o_x, o_y, o_z) for the two block dims,
    // and the logical coordinate (c, b, a, block 0, block 1) of each TMA dim
    int map[PG_MAX_SLOTS + 1];
    int tax[PG_MAX_SLOTS + 1][3];
    int cb0[PG_MAX_SLOTS + 1][3], cb1[PG_MAX_SLOTS + 1][3];
    int sel[PG_MAX_SLOTS + 1][5];
};

__device__ __forceinline__ int pick5(int k, int v0, int v1, int v2, int v3, int v4) {
    return k == 0 ? v0 : (k == 1 ? v1 : (k == 2 ? v2 : (k == 3 ? v3 : v4)));
}

__device__ __forceinline__ void named_sync_compute() { asm volatile("bar.sync 1, %0;" ::"n"(32 * TG_WARPS) : "memory"); }

// Persistent gather: work item w = (block q, output tile T).  Warp 8 issues
// one TMA box load per (source, permutation) slot (plus the r3 tile when
// beta != 0) into a ring of stages; warps 0..7 sum the slots from shared
// memory, write the output tile densely and one thread stores it with TMA
// (out-of-range elements of edge tiles are clipped by the copy engine).
// Every mbarrier wait is bounded; after a timeout the CTA finishes its
// iterations without waiting or storing so the named barriers stay matched.
__global__ void __launch_bounds__(TG_THREADS, 1)
    k_perm_gather_tma(const __grid_constant__ TmaMaps maps, const int32_t *ijk, int64_t nwork, int ntile, double beta,
                      TmaGatherArgs g, int stages, int *status) {
    extern __shared__ __align__(1024) uint8_t tg_smem[];
    uint8_t *base = (uint8_t *)(((uintptr_t)tg_smem + 1023) & ~(uintptr_t)1023);
    const int nload = g.nslot + (beta != 0.0 ? 1 : 0);
    const uint32_t stage_bytes = (uint32_t)nload * TG_TILE_BYTES;
    double *outb = (double *)(base + (size_t)stages * stage_bytes);  // 2 output tiles
    uint64_t *full = (uint64_t *)(base + (size_t)stages * stage_bytes + 2 * TG_TILE_BYTES);
    uint64_t *empty = full + stages;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int nt3 = ntile * ntile * ntile;
    if (t == 0) {
        for (int s = 0; s < stages; s++) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), TG_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == TG_WARPS) {
        // ---------------- producer warp: lane l issues load l of each work item
        if (lane <= PG_MAX_SRC) tma_prefetch_desc(&maps.m[lane]);
        int64_t it = 0;
        for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x, it++) {
            const int s = (int)(it % stages);
            const uint32_t ph = (uint32_t)(it / stages) & 1u;
            bool ok = lane == 0 ? mbar_wait(smem_u32(&empty[s]), ph ^ 1u, status) : true;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
            const uint32_t fb = smem_u32(&full[s]);
            if (lane == 0) mbar_expect_tx(fb, (uint32_t)nload * TG_TILE_BYTES);
            __syncwarp();
            if (lane < nload) {
                const int64_t q = w / nt3;
                const int T = (int)(w % nt3);
                const int TT[3] = {T / (ntile * ntile), (T / ntile) % ntile, T % ntile};
                const int o0 = ijk[3 * q], o1 = ijk[3 * q + 1], o2 = ijk[3 * q + 2];
                const int l = lane;
                const int vc = TT[g.tax[l][0]] * TE, vb = TT[g.tax[l][1]] * TE, va = TT[g.tax[l][2]] * TE;
                int v3 = o0 * g.cb0[l][0] + o1 * g.cb0[l][1] + o2 * g.cb0[l][2];
                const int v4 = o0 * g.cb1[l][0] + o1 * g.cb1[l][1] + o2 * g.cb1[l][2];
                if (l == g.nslot) v3 = (int)q;  // the r3 tile
                tma_load_5d(smem_u32(base + (size_t)s * stage_bytes + (size_t)l * TG_TILE_BYTES), &maps.m[g.map[l]], fb,
                            pick5(g.sel[l][0], vc, vb, va, v3, v4), pick5(g.sel[l][1], vc, vb, va, v3, v4),
                            pick5(g.sel[l][2], vc, vb, va, v3, v4), pick5(g.sel[l][3], vc, vb, va, v3, v4),
                            pick5(g.sel[l][4], vc, vb, va, v3, v4));
            }
        }
        // no copy may still be landing in this CTA's shared memory when it exits (the compute
        // warps stop waiting for them after a timeout): wait, bounded, for the last ones issued
        if (lane == 0) {
            const int64_t first = it > stages ? it - stages : 0;
            for (int64_t k = first; k < it; k++)
                mbar_wait_quiet(smem_u32(&full[k % stages]), (uint32_t)(k / stages) & 1u);
        }
        return;
    }

    // ---------------- compute warps
    int rd[PG_MAX_SLOTS][2];
    int oidx[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        int u[3];
        tg_element(t, h, u);
        oidx[h] = u[0] * 64 + u[1] * 8 + u[2];
#pragma unroll
        for (int sl = 0; sl < PG_MAX_SLOTS; sl++) {
            const int p = sl < g.nslot ? g.slot_perm[sl] : 0;
            rd[sl][h] = sl * TE3 + u[perm3(p, 0)] * 64 + u[perm3(p, 1)] * 8 + u[perm3(p, 2)];
        }
    }
    bool dry = false;
    int64_t it = 0;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x, it++) {
        const int s = (int)(it % stages);
        const uint32_t ph = (uint32_t)(it / stages) & 1u;
        if (!dry && !mbar_wait(smem_u32(&full[s]), ph, status)) dry = true;
        const double *st = (const double *)(base + (size_t)s * stage_bytes);
        double acc[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double a = 0.0;
#pragma unroll
            for (int sl = 0; sl < PG_MAX_SLOTS; sl++)
                if (sl < g.nslot) a = fma(g.slot_scale[sl], st[rd[sl][h]], a);
            acc[h] = beta != 0.0 ? fma(beta, st[g.nslot * TE3 + oidx[h]], a) : a;
        }
        __syncwarp();
        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&empty[s])) : "memory");
        double *ob = outb + (it & 1) * TE3;
        if (t == 0) bulk_wait_read<1>();  // the store of two items ago has read this buffer
        named_sync_compute();
        ob[oidx[0]] = acc[0];
        ob[oidx[1]] = acc[1];
        fence_proxy_async_smem();
        named_sync_compute();
        if (t == 0 && !dry) {
            const int64_t q = w / nt3;
            const int T = (int)(w % nt3);
            const int vc = (T % ntile) * TE, vb = ((T / ntile) % ntile) * TE, va = (T / (ntile * ntile)) * TE;
            const int v3 = (int)q;
            const int *sl = g.sel[PG_MAX_SLOTS];
            tma_store_5d(&maps.m[PG_MAX_SRC], smem_u32(ob), pick5(sl[0], vc, vb, va, v3, 0),
                         pick5(sl[1], vc, vb, va, v3, 0), pick5(sl[2], vc, vb, va, v3, 0),
                         pick5(sl[3], vc, vb, va, v3, 0), pick5(sl[4], vc, vb, va, v3, 0));
            bulk_commit();
        }
    }
    if (t == 0) bulk_wait<0>();
}

// Tensor map over a strided FP64 array given as (extent, stride in elements)
// pairs with the unit-stride dimension first; the other dimensions are
// ordered by stride, and pos[k] records where input dimension k went.
static int encode_strided(CUtensorMap *map, const double *base, const int64_t ext[5], const int64_t str[5],
                          const uint32_t box[5], int pos[5]) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is unavailable");
        return DCC_ERR_CUDA;
    }
    int order[5] = {0, 1, 2, 3, 4};
    for (int i = 1; i < 5; i++)  // insertion sort of dims 1..4 by stride
        for (int j = i; j > 1 && str[order[j]] < str[order[j - 1]]; j--) {
            int tmp = order[j];
            order[j] = order[j - 1];
            order[j - 1] = tmp;
        }
    cuuint64_t dims[5], strides[4];
    cuuint32_t bx[5], es[5] = {1, 1, 1, 1, 1};
    for (int i = 0; i < 5; i++) {
        dims[i] = (cuuint64_t)ext[order[i]];
        bx[i] = box[order[i]];
        pos[order[i]] = i;
        if (i > 0) strides[i - 1] = (cuuint64_t)(str[order[i]] * 8);
    }
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<double *>(base), dims, strides, bx, es,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return DCC_ERR_CUDA;
    }
    return DCC_OK;
}

// Block dimensions of a source as one or two TMA dims: the three block strides
// (x, y, z) collapse when one is nocc times another.  Returns false when they
// do not.
static bool block_dims(const int64_t st[3], int64_t no, int64_t ext[2], int64_t str[2], int c1[3], int c2[3]) {
    for (int i = 0; i < 3; i++) c1[i] = c2[i] = 0;
    // all three merge: st[p] = no^2 st[r], st[q] = no st[r]
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
            const int r = 3 - p - q;
            if (p == q || r < 0 || r > 2 || r == p || r == q) continue;
            if (st[p] == no * st[q] && st[q] == no * st[r]) {
                ext[0] = no * no * no, str[0] = st[r], ext[1] = 1, str[1] = st[p] * no;
                c1[p] = (int)(no * no), c1[q] = (int)no, c1[r] = 1;
                return true;
            }
        }
    for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
            if (p == q) continue;
            const int r = 3 - p - q;
            if (st[p] == no * st[q]) {
                ext[0] = no * no, str[0] = st[q], ext[1] = no, str[1] = st[r];
                c1[p] = (int)no, c1[q] = 1, c2[r] = 1;
                return true;
            }
        }
    return false;
}

}  // namespace dcc

namespace dcc {

// The S3 gather of one full-layout source (every permutation, the residual's S) for rows that are
// not 16-byte aligned, by rows: r3[q][a,b,c] = beta r3 + scale sum_p S[p(ijk)][p(abc)].  Of the six
// terms of an output row (a,b,:), S[ijk][a,b,:] and S[jik][b,a,:] are whole rows; the other four
// are columns (c in the middle or first position of the source) and come from four tiles staged
// in shared memory for a pair of 8-wide index tiles (a in I, b in J) and a chunk of c.  Each warp
// then streams output rows with coalesced loads and stores.  The slots are summed in the order of
// the orbit-tile kernels (p = 0..5, one fma each), so the result is theirs bit for bit.
// ST: the storage type of S (double; float for the FP32 accumulator of the split precisions, whose
// values enter the same FP64 sums exactly).
constexpr int GB_PITCH = 65;  // elements per (c) row of a staged tile: 8 x 8 + 1 (conflict-free transposed reads)
template <typename ST>
__global__ void __launch_bounds__(256, 2) k_gather_band(const ST *__restrict__ S, double *__restrict__ r3,
                                                        const int32_t *__restrict__ ijk, int64_t nblocks, int nocc,
                                                        int nv, int ntile, int cchunk, double scale, double beta) {
    extern __shared__ double gb_sm[];  // tiles of the slots p = 1, 3, 4, 5: [cc][a_local * 8 + b_local]
    ST *T1 = reinterpret_cast<ST *>(gb_sm), *T3 = T1 + (size_t)cchunk * GB_PITCH, *T4 = T3 + (size_t)cchunk * GB_PITCH,
       *T5 = T4 + (size_t)cchunk * GB_PITCH;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t n3 = (int64_t)nv * nv * nv, nv2 = (int64_t)nv * nv;
    const int nch = (nv + cchunk - 1) / cchunk;
    const int64_t per_q = (int64_t)ntile * ntile * nch, nwork = nblocks * per_q;
    for (int64_t w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t q = w / per_q;
        const int rem = (int)(w % per_q);
        const int I = rem / (ntile * nch), J = (rem / nch) % ntile, ch = rem % nch;
        const int c0 = ch * cchunk, cn = min(cchunk, nv - c0);
        const int o[3] = {ijk[3 * q], ijk[3 * q + 1], ijk[3 * q + 2]};
        const ST *src[6];
#pragma unroll
        for (int p = 0; p < 6; p++)
            src[p] = S + (((int64_t)o[perm3(p, 0)] * nocc + o[perm3(p, 1)]) * nocc + o[perm3(p, 2)]) * n3;
        const int a0 = I * TE, b0 = J * TE;
        for (int e = threadIdx.x; e < cn * 64; e += blockDim.x) {
            const int cc = e >> 6, r = (e >> 3) & 7, t = e & 7, c = c0 + cc, off = cc * GB_PITCH;
            if (a0 + r < nv && b0 + t < nv) {  // a = a0 + r, b = b0 + t: b contiguous
                const int a = a0 + r, b = b0 + t;
                cp_async_el(T1 + off + r * 8 + t, src[1] + a * nv2 + (int64_t)c * nv + b);  // S1[a][c][b]
                cp_async_el(T4 + off + r * 8 + t, src[4] + c * nv2 + (int64_t)a * nv + b);  // S4[c][a][b]
            }
            if (b0 + r < nv && a0 + t < nv) {  // b = b0 + r, a = a0 + t: a contiguous
                const int a = a0 + t, b = b0 + r;
                cp_async_el(T3 + off + t * 8 + r, src[3] + b * nv2 + (int64_t)c * nv + a);  // S3[b][c][a]
                cp_async_el(T5 + off + t * 8 + r, src[5] + c * nv2 + (int64_t)b * nv + a);  // S5[c][b][a]
            }
        }
        cp_async_commit();
        cp_async_wait<0>();
        __syncthreads();
        // two output rows per pass (al and al + 1), every global load of both (the two source
        // rows, and the output when beta != 0; cc = lane + 32 j covers cchunk <= 64) issued
        // before the arithmetic: up to 12 loads in flight per lane
        for (int rw = warp; rw < 64; rw += 16) {
            double v0[2][2], v2[2][2], vo[2][2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int al = (rw >> 3) + h, bl = rw & 7, a = a0 + al, b = b0 + bl;
                const bool ok = a < nv && b < nv;
                const ST *r0 = src[0] + a * nv2 + (int64_t)b * nv, *r2 = src[2] + b * nv2 + (int64_t)a * nv;
                const double *out = r3 + q * n3 + a * nv2 + (int64_t)b * nv;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int cc = lane + 32 * j, c = c0 + cc;
                    const bool in = ok && cc < cn;
                    v0[h][j] = in ? (double)__ldg(r0 + c) : 0.0;
                    v2[h][j] = in ? (double)__ldg(r2 + c) : 0.0;
                    vo[h][j] = in && beta != 0.0 ? out[c] : 0.0;
                }
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int al = (rw >> 3) + h, bl = rw & 7, a = a0 + al, b = b0 + bl;
                if (a >= nv || b >= nv) continue;
                double *out = r3 + q * n3 + a * nv2 + (int64_t)b * nv;
                const int ti = al * 8 + bl;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const int cc = lane + 32 * j, c = c0 + cc;
                    if (cc >= cn) continue;
                    const int off = cc * GB_PITCH + ti;
                    double acc = fma(scale, v0[h][j], 0.0);
                    acc = fma(scale, (double)T1[off], acc);
                    acc = fma(scale, v2[h][j], acc);
                    acc = fma(scale, (double)T3[off], acc);
                    acc = fma(scale, (double)T4[off], acc);
                    acc = fma(scale, (double)T5[off], acc);
                    out[c] = beta == 0.0 ? acc : fma(beta, vo[h][j], acc);
                }
            }
        }
        __syncthreads();  // the tiles are refilled by the next item
    }
}

}  // namespace dcc

// The row gather for one full-layout source with every permutation at an odd nvir; returns
// DCC_ERR_UNSUPPORTED (nothing launched) where it does not apply.
template <typename ST>
static int gather_band_launch(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nocc, int64_t nvir, double beta,
                              int nsrc, const ST *const *bases, const double *scales, const int64_t *strides,
                              const int *masks, void *stream) {
    if (nsrc != 1 || masks[0] != 63 || nvir > 104 || nocc < 1 || nocc > 1290 || !bases[0]) return DCC_ERR_UNSUPPORTED;
    const int64_t n3 = nvir * nvir * nvir;
    const int64_t full[6] = {nocc * nocc * n3, nocc * n3, n3, nvir * nvir, nvir, 1};
    for (int m = 0; m < 6; m++)
        if (strides[m] != full[m]) return DCC_ERR_UNSUPPORTED;
    const int64_t sbytes = nocc * nocc * nocc * n3 * (int64_t)sizeof(ST), rbytes = nblocks * n3 * (int64_t)sizeof(double);
    if (!((const char *)bases[0] + sbytes <= (const char *)r3 || (const char *)r3 + rbytes <= (const char *)bases[0]))
        return DCC_ERR_UNSUPPORTED;
    const int ntile = (int)ceil_div(nvir, TE);
    const int cchunk = (int)((nvir + 1) / 2);  // two chunks of c: four tiles fit twice in an SM
    const size_t smem = 4 * (size_t)cchunk * GB_PITCH * sizeof(ST);
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t nwork = nblocks * (int64_t)ntile * ntile * 2, cap = (int64_t)nsm * 2;
    const unsigned grid = (unsigned)(nwork < cap ? nwork : cap);
    cudaFuncSetAttribute(k_gather_band<ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_gather_band<ST><<<grid, 256, smem, as_stream(stream)>>>(bases[0], r3, ijk, nblocks, (int)nocc, (int)nvir, ntile,
                                                              cchunk, scales[0], beta);
    return DCC_OK;
}

// r3 = beta r3 + scale sum_p S[p(ijk)][p(abc)] over every simultaneous permutation p, from a
// full-layout FP32 S [nocc^3][nvir^3] (the split precisions' accumulator), nvir <= 104.
extern "C" int dcc_t3_s3_gather_f32(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nocc, int64_t nvir,
                                    double beta, const float *S, double scale, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0 && nocc >= 0, DCC_ERR_SHAPE, "negative size");
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(r3 && ijk && S, DCC_ERR_NULL, "NULL argument");
    DCC_REQUIRE(nvir <= 104 && nocc >= 1 && nocc <= 1290, DCC_ERR_UNSUPPORTED,
                "the FP32 gather serves nvir <= 104 (nvir = %lld)", (long long)nvir);
    const int64_t n3 = nvir * nvir * nvir;
    const int64_t full[6] = {nocc * nocc * n3, nocc * n3, n3, nvir * nvir, nvir, 1};
    const int mask = 63;
    const float *bases[1] = {S};
    const int rc = gather_band_launch(r3, ijk, nblocks, nocc, nvir, beta, 1, bases, &scale, full, &mask, stream);
    DCC_REQUIRE(rc == DCC_OK, DCC_ERR_SHAPE, "S and r3 overlap");
    return launch_status("t3_gather_band (FP32 S)");
}

extern "C" int dcc_t3_perm_gather_tma(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nocc, int64_t nvir,
                                      double beta, int nsrc, const double *const *bases, const double *scales,
                                      const int64_t *strides, const int *masks, int *status, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0 && nocc >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE(nsrc >= 1 && nsrc <= PG_MAX_SRC, DCC_ERR_SHAPE, "1..%d sources", PG_MAX_SRC);
    if (nblocks == 0 || nvir == 0) return DCC_OK;
    DCC_REQUIRE(r3 && ijk && bases && scales && strides && masks && status, DCC_ERR_NULL, "NULL argument");
    // the residual's gather (one full-layout source, every permutation) runs by rows: at nocc=10 /
    // nvir=90 2.90 ms against 3.39 ms for the TMA pipeline below, and at odd nvir, where TMA
    // cannot describe the rows, 13.5 ms against 22.0 ms for the cp.async kernel at nocc=15
    if (gather_band_launch(r3, ijk, nblocks, nocc, nvir, beta, nsrc, bases, scales, strides, masks, stream) == DCC_OK)
        return launch_status("t3_gather_band");
    // the copy engine needs 16-byte strides, a unit-stride c and b faster than a; otherwise the
    // cp.async kernel serves the call
    bool tma = nvir % 2 == 0 && nocc >= 1 && nocc <= 1290 && nvir <= 65536;
    TmaGatherArgs g{};
    TmaMaps maps;
    memset(&maps, 0, sizeof(maps));
    int nslot = 0;
    for (int s = 0; s < nsrc && tma; s++) {
        const int64_t *st = strides + 6 * s;
        DCC_REQUIRE(bases[s], DCC_ERR_NULL, "source %d is NULL", s);
        DCC_REQUIRE(masks[s] > 0 && masks[s] < 64, DCC_ERR_SHAPE, "source %d: permutation mask must be in 1..63", s);
        bool even = true;
        for (int m = 0; m < 5; m++) even = even && st[m] > 0 && st[m] % 2 == 0;
        if (!even || st[5] != 1 || st[4] >= st[3] || ((uintptr_t)bases[s] & 15)) {
            tma = false;
            break;
        }
        int64_t bext[2], bstr[2];
        int c1[3], c2[3];
        if (!block_dims(st, nocc, bext, bstr, c1, c2)) {
            tma = false;
            break;
        }
        const int64_t ext[5] = {nvir, nvir, nvir, bext[0], bext[1]};
        const int64_t str[5] = {1, st[4], st[3], bstr[0], bstr[1]};
        const uint32_t box[5] = {TE, TE, TE, 1, 1};
        int pos[5];
        int rc = encode_strided(&maps.m[s], bases[s], ext, str, box, pos);
        if (rc) return rc;
        for (int p = 0; p < 6; p++)
            if (masks[s] & (1 << p)) {
                DCC_REQUIRE(nslot < PG_MAX_SLOTS, DCC_ERR_UNSUPPORTED, "more than %d source tiles", PG_MAX_SLOTS);
                const int P[3] = {perm3(p, 0), perm3(p, 1), perm3(p, 2)};
                g.slot_perm[nslot] = p;
                g.slot_scale[nslot] = scales[s];
                g.map[nslot] = s;
                // slot tile = p(T): its c / b / a tiles are T[P2] / T[P1] / T[P0]; its block is
                // (o[P0], o[P1], o[P2]) as the source's (x, y, z)
                g.tax[nslot][0] = P[2], g.tax[nslot][1] = P[1], g.tax[nslot][2] = P[0];
                for (int m = 0; m < 3; m++) {
                    g.cb0[nslot][P[m]] = c1[m];
                    g.cb1[nslot][P[m]] = c2[m];
                }
                for (int k = 0; k < 5; k++) g.sel[nslot][pos[k]] = k;
                nslot++;
            }
    }
    if (!tma || ((uintptr_t)r3 & 15))
        return dcc_t3_perm_gather(r3, ijk, nblocks, nvir, beta, nsrc, bases, scales, strides, masks, stream);
    g.nslot = nslot;
    {
        const int64_t ext[5] = {nvir, nvir, nvir, nblocks, 1};
        const int64_t str[5] = {1, nvir, nvir * nvir, nvir * nvir * nvir, nvir * nvir * nvir * nblocks};
        const uint32_t box[5] = {TE, TE, TE, 1, 1};
        int pos[5];
        int rc = encode_strided(&maps.m[PG_MAX_SRC], r3, ext, str, box, pos);
        if (rc) return rc;
        // the r3 tile (load slot nslot when beta != 0, and the store): tile (a, b, c) = T, block q
        for (int k = 0; k < 5; k++) g.sel[PG_MAX_SLOTS][pos[k]] = k;
        g.map[nslot] = PG_MAX_SRC;
        g.tax[nslot][0] = 2, g.tax[nslot][1] = 1, g.tax[nslot][2] = 0;
        for (int k = 0; k < 5; k++) g.sel[nslot][k] = g.sel[PG_MAX_SLOTS][k];
    }
    const int ntile = (int)ceil_div(nvir, TE);
    const int64_t nwork = nblocks * ntile * ntile * ntile;
    const int nload = nslot + (beta != 0.0 ? 1 : 0);
    int stages = (int)((TG_SMEM_BUDGET - 2 * TG_TILE_BYTES) / (nload * TG_TILE_BYTES));
    stages = stages > 8 ? 8 : stages;
    DCC_REQUIRE(stages >= 2, DCC_ERR_UNSUPPORTED, "too many source tiles for the pipeline");
    const size_t smem = 1024 + (size_t)stages * nload * TG_TILE_BYTES + 2 * TG_TILE_BYTES + 2 * stages * 8;
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = nwork < nsm ? nwork : nsm;
    cudaFuncSetAttribute(k_perm_gather_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_perm_gather_tma<<<(unsigned)grid, TG_THREADS, smem, as_stream(stream)>>>(maps, ijk, nwork, ntile, beta, g, stages,
                                                                               status);
    return launch_status("t3_perm_gather_tma");
}

// ---------------------------------------------------------------- no-allocation update


namespace dcc {

// Rows (q, a, b) per CTA of the no-allocation update, and the most CTAs the
// static scratch can serve: 8192 pairs of partial sums = 128 KiB, which
// covers nblocks * nvir^2 <= 8 388 608 rows (e.g. 680 blocks of nvir = 93).
constexpr int64_t NOALLOC_ROWS_PER_CTA = 1024;
constexpr int64_t NOALLOC_MAX_CTAS = 8192;

// Partial squared norms of dcc_t3_divide_update_noalloc, two doubles per CTA.
// Every GPU that loads the library holds this array until the process exits;
// all calls on a device share it.
static __device__ __align__(256) double g_update_scratch[2 * NOALLOC_MAX_CTAS];

// Device address of g_update_scratch for the current device, looked up once per device
// (again only if the device's context was replaced, e.g. after cudaDeviceReset).  In host
// code the symbol names a host-side stand-in, so kernels must be given this address instead.
static int update_scratch_address(double **out) {
    static std::mutex mu;
    static struct {
        unsigned long long ctx;
        double *addr;
    } cache[128] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("cudaGetDevice: %s", cudaGetErrorString(e));
        return DCC_ERR_CUDA;
    }
    if (dev < 0 || dev >= 128) {
        set_error("device ordinal %d out of range", dev);
        return DCC_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(mu);
    unsigned long long ctx = current_context_id();
    if (!cache[dev].addr || !ctx || cache[dev].ctx != ctx) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_update_scratch);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(update scratch): %s", cudaGetErrorString(e));
            return DCC_ERR_CUDA;
        }
        cache[dev].addr = (double *)p;
        cache[dev].ctx = current_context_id();
    }
    *out = cache[dev].addr;
    return DCC_OK;
}

}  // namespace dcc

extern "C" int dcc_t3_divide_update_noalloc(double *t3, double *r3, const double *eia, const int32_t *ijk,
                                            int64_t nblocks, int64_t nvir, int64_t nvir_active, int write_r3,
                                            double *norms, void *stream) {
    clear_error();
    DCC_REQUIRE(nblocks >= 0 && nvir >= 0, DCC_ERR_SHAPE, "negative size");
    DCC_REQUIRE(norms, DCC_ERR_NULL, "norms is NULL");
    cudaStream_t st = as_stream(stream);
    if (nblocks == 0 || nvir == 0) {
        if (cudaMemsetAsync(norms, 0, 2 * sizeof(double), st) != cudaSuccess) return launch_status("memset");
        return DCC_OK;
    }
    DCC_REQUIRE(t3 && r3 && eia && ijk, DCC_ERR_NULL, "NULL buffer");
    const int64_t rows = nblocks * nvir * nvir;
    const int64_t ctas = (rows + NOALLOC_ROWS_PER_CTA - 1) / NOALLOC_ROWS_PER_CTA;
    DCC_REQUIRE(ctas <= NOALLOC_MAX_CTAS, DCC_ERR_SHAPE,
                "nblocks*nvir^2 = %lld rows exceeds the no-allocation limit of %lld rows (static scratch of %lld "
                "partial sums); use dcc_t3_divide_update with a workspace",
                (long long)rows, (long long)(NOALLOC_MAX_CTAS * NOALLOC_ROWS_PER_CTA), (long long)NOALLOC_MAX_CTAS);
    double *scratch = nullptr;
    int rc = update_scratch_address(&scratch);
    if (rc) return rc;
    if (nvir_active < 0 || nvir_active > nvir) nvir_active = nvir;
    // every CTA overwrites its own pair before k_sum_pairs reads exactly `ctas` pairs,
    // so nothing left by an earlier call needs clearing
    k_t3_divide_update<<<(unsigned)ctas, UPD_THREADS, 0, st>>>(t3, r3, eia, ijk, nblocks, (int)nvir, (int)nvir_active,
                                                               write_r3, scratch);
    rc = launch_status("t3_divide_update_noalloc");
    if (rc) return rc;
    k_sum_pairs<<<1, 256, 0, st>>>(scratch, ctas, norms);
    return launch_status("t3_divide_update_noalloc reduce");
}
