// Split-precision tensor-core GEMM for the dense T3 residual contractions
// (tcgen05 + TMEM + TMA, sm_100a).
//
//   C[row_off(m) + col_off(n)] = alpha * sum_k A[m][k] B[n][k] + beta * C[...]
//
// A and B are FP64 operands that have been split into two bf16 (or tf32)
// pieces, x = x_hi + x_lo, stored K-major with K padded to the k-block.  The
// product is accumulated in FP32 in tensor memory as
//   A_hi B_hi + A_hi B_lo + A_lo B_hi
// (the dropped A_lo B_lo term is below the pieces' own rounding), and the
// epilogue adds alpha * acc into an FP64 C with beta scaling.  Row and column
// offsets are three-digit mixed-radix maps,
//   off(m) = (m / (R1*R2)) * S0 + ((m / R2) % R1) * S1 + (m % R2) * S2,
// so permuted contraction outputs (e.g. r3[a,b,c] += X[(q,c),(a,b)]) are
// accumulated in place without a transposed temporary.
//
// CTA = 6 warps: warp 0 issues TMA loads, warp 1 owns TMEM and issues the
// MMAs from one thread, warps 2..5 drain the accumulator (one TMEM lane
// quarter each).  Every mbarrier wait is bounded; on timeout the kernel sets
// *status = DCC_ERR_TIMEOUT, waits (bounded) for its own copies and MMAs,
// frees TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include "async_util.cuh"
#include "dcc_common.cuh"

namespace dcc {

constexpr int GM = 128;       // tile rows (UMMA M)
constexpr int GN = 256;       // tile cols (UMMA N)
// CTA = warp 0 (TMA producer) + warp 1 (MMA issuer) + EPI epilogue warps
template <int EPI>
constexpr int gemm_threads() { return 64 + 32 * EPI; }

// Tunable pipeline shape: bytes of K per operand row and k-block (128, 64 or
// 32 -> 128/64/32-byte swizzle), ring depth, and the number of M-tiles per
// raster group (CTAs that run together share B tiles in L2).
struct GemmConfig {
    int kb_bytes, stages, group_m, tile_n;
};
static GemmConfig g_cfg = {64, 4, 16, 256};

// Four-digit mixed-radix address map:
//   off(m) = (m / (R1 R2 R3)) S0 + ((m / (R2 R3)) % R1) S1 + ((m / R3) % R2) S2 + (m % R3) S3.
// A three-digit map {R1, R2, S0, S1, S2} is {R1, R2, 1, S0, S1, S2, 0}.
struct Map4 {
    int64_t R1, R2, R3, S0, S1, S2, S3;
};

__host__ __device__ __forceinline__ int64_t map4(const Map4 &f, int64_t m) {
    const int64_t r23 = f.R2 * f.R3;
    return (m / (f.R1 * r23)) * f.S0 + ((m / r23) % f.R1) * f.S1 + ((m / f.R3) % f.R2) * f.S2 + (m % f.R3) * f.S3;
}

struct GemmEpi {
    Map4 row, col;
};

// map4 for m < 2^31 and R1 R2 R3 < 2^31 (checked on the host): 32-bit divisions.
__device__ __forceinline__ int64_t map4_32(const Map4 &f, uint32_t m) {
    const uint32_t r3 = (uint32_t)f.R3, r23 = (uint32_t)(f.R2 * f.R3), r123 = (uint32_t)(f.R1 * f.R2 * f.R3);
    const uint32_t d0 = m / r123, m1 = m - d0 * r123;
    const uint32_t d1 = m1 / r23, m2 = m1 - d1 * r23;
    const uint32_t d2 = m2 / r3, d3 = m2 - d2 * r3;
    return (int64_t)d0 * f.S0 + (int64_t)d1 * f.S1 + (int64_t)d2 * f.S2 + (int64_t)d3 * f.S3;
}

// Stride and radix of the fastest digit that varies (R3 == 1: the map has three digits).
__host__ __forceinline__ void fast_digit(const Map4 &f, int64_t &stride, int64_t &radix) {
    stride = f.R3 > 1 ? f.S3 : f.S2;
    radix = f.R3 > 1 ? f.R3 : f.R2;
}

__host__ __forceinline__ Map4 map_from(const int64_t *v, bool four) {
    return four ? Map4{v[0], v[1], v[2], v[3], v[4], v[5], v[6]} : Map4{v[0], v[1], 1, v[2], v[3], v[4], 0};
}

// K-major, swizzled operand tile with rows of KB bytes (KB = 128/64/32 ->
// SWIZZLE_128B/64B/32B): 8-row groups 8*KB bytes apart (stride byte offset),
// Blackwell descriptor version 1.
template <int KB>
__device__ __forceinline__ uint64_t swz_desc(uint32_t saddr) {
    constexpr uint64_t layout = KB == 128 ? 2 : (KB == 64 ? 4 : 6);
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major): 16 B
    d |= (uint64_t)((8 * KB) >> 4) << 32;   // stride byte offset: one 8-row group
    d |= (uint64_t)1 << 46;                 // descriptor version
    d |= layout << 61;
    return d;
}

template <int KIND>  // 0: kind::f16 (bf16 x bf16), 1: kind::tf32
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    if (KIND == 0)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// ----------------------------------------------------------------- kernel

// Fire-and-forget reduction into global memory (red, no value returned; the L2 adds).  The
// pointers may be generic addresses (the grouped GEMM's problem table), for which the compiler
// would emit a returning generic atomic; name the global space here.
__device__ __forceinline__ void red_add(float *p, float v) {
    asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\tred.global.add.f32 [g], %1;\n\t}" ::"l"(p), "f"(v)
                 : "memory");
}
__device__ __forceinline__ void red_add(double *p, double v) {
    asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\tred.global.add.f64 [g], %1;\n\t}" ::"l"(p), "d"(v)
                 : "memory");
}


template <int ST>
struct GemmSmem {
    uint64_t full[ST];
    uint64_t empty[ST];
    uint64_t acc_full[2];   // accumulator b holds a finished tile
    uint64_t acc_empty[2];  // accumulator b has been read out by every epilogue warp
    uint64_t drain;         // all MMAs of this CTA retired (end of kernel)
    uint32_t tmem_base;
};

// per epilogue warp: a 32x33 float transpose buffer, 32 row and 64 column offsets
constexpr uint32_t EPI_WARP_BYTES = 32 * 33 * 4 + 96 * 8;

__device__ __forceinline__ void tile_coords(int t, int num_m, int num_n, int group_m, int &tm, int &tn) {
    const int per_group = group_m * num_n;
    const int first_m = (t / per_group) * group_m;
    const int gsz = (num_m - first_m) < group_m ? (num_m - first_m) : group_m;
    tm = first_m + (t % per_group) % gsz;
    tn = (t % per_group) / gsz;
}

// Persistent: CTA c takes tiles c, c + gridDim.x, ... (linear ids rasterized
// in groups of group_m M-tiles).  Two TMEM accumulators of TN columns let the
// MMAs of tile t+1 run while the epilogue warps drain tile t.
// KIND 0: bf16 pieces; KIND 1: tf32 pieces.  KB: bytes of K per row and
// k-block; ST: ring depth.
// CT: the storage type of C (double; float for the FP32 accumulators of the split precisions,
// whose epilogue reads and writes half the bytes; the arithmetic stays FP64, one rounding per store).
// TN: tile columns (UMMA N), 256 or 128.  A 128-column tile holds half the TMEM (two accumulators
// of 128 columns) and, with two stages of 64-byte k-blocks and four epilogue warps, half the
// shared memory, so two CTAs share an SM.
template <int KIND, int KB, int ST, int EPI, typename CT = double, int TN = GN>
__global__ void __launch_bounds__(gemm_threads<EPI>(), TN == GN ? 1 : 2)
    k_gemm_split3(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                  const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl, int M, int N,
                  int nkb, CT *C, GemmEpi epi, double alpha, double beta, int *status, int group_m,
                  int epi_cols) {
    extern __shared__ __align__(1024) uint8_t g_smem[];
    // operand stages first (1024-byte aligned), then the epilogue buffers and the control block
    uint8_t *base = (uint8_t *)(((uintptr_t)g_smem + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t A_BYTES = GM * KB, B_BYTES = TN * KB;
    constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    uint8_t *epi_base = base + ST * STAGE_BYTES;
    GemmSmem<ST> *cs = (GemmSmem<ST> *)(epi_base + EPI * EPI_WARP_BYTES);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int num_m = (M + GM - 1) / GM, num_n = (N + TN - 1) / TN, ntiles = num_m * num_n;

    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; s++) {
            mbar_init(smem_u32(&cs->full[s]), 1);
            mbar_init(smem_u32(&cs->empty[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&cs->acc_full[b]), 1);
            mbar_init(smem_u32(&cs->acc_empty[b]), EPI);
        }
        mbar_init(smem_u32(&cs->drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        tma_prefetch_desc(&tmAh);
        tma_prefetch_desc(&tmAl);
        tma_prefetch_desc(&tmBh);
        tma_prefetch_desc(&tmBl);
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&cs->tmem_base)),
                     "r"(2 * TN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = cs->tmem_base;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer
        uint32_t g = 0;  // k-blocks issued by this CTA
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            int tm, tn;
            tile_coords(t, num_m, num_n, group_m, tm, tn);
            for (int kb = 0; kb < nkb; kb++) {
                const uint32_t s = g % ST, ph = (g / ST) & 1u;
                if (!mbar_wait(smem_u32(&cs->empty[s]), ph ^ 1u, status)) {
                    ok = false;
                    break;
                }
                uint8_t *st = base + s * STAGE_BYTES;
                const uint32_t fb = smem_u32(&cs->full[s]);
                mbar_expect_tx(fb, STAGE_BYTES);
                const int kc = kb * (KB / (KIND == 0 ? 2 : 4));
                tma_load_2d(smem_u32(st), &tmAh, fb, kc, tm * GM);
                tma_load_2d(smem_u32(st + A_BYTES), &tmAl, fb, kc, tm * GM);
                tma_load_2d(smem_u32(st + 2 * A_BYTES), &tmBh, fb, kc, tn * TN);
                tma_load_2d(smem_u32(st + 2 * A_BYTES + B_BYTES), &tmBl, fb, kc, tn * TN);
                g++;
            }
        }
        // on an early exit, wait (bounded) for the copies still landing in shared memory
        if (!ok) {
            const uint32_t first = g > (uint32_t)ST ? g - ST : 0u;
            for (uint32_t k = first; k < g; k++) mbar_wait_quiet(smem_u32(&cs->full[k % ST]), (k / ST) & 1u);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        constexpr uint32_t idesc = (1u << 4)                          // D: f32
                                   | ((KIND == 0 ? 1u : 2u) << 7)     // A: bf16 | tf32
                                   | ((KIND == 0 ? 1u : 2u) << 10)    // B: bf16 | tf32
                                   | ((uint32_t)(TN >> 3) << 17)      // N
                                   | ((uint32_t)(GM >> 4) << 24);     // M
        constexpr int KSTEPS = KB / 32;  // one UMMA consumes 32 bytes of K
        uint32_t g = 0;
        bool ok = true;
        int it = 0;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, it++) {
            const int b = it & 1;
            if (!mbar_wait(smem_u32(&cs->acc_empty[b]), (((uint32_t)it >> 1) & 1u) ^ 1u, status)) break;
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(b * TN);
            for (int kb = 0; kb < nkb; kb++) {
                const uint32_t s = g % ST, ph = (g / ST) & 1u;
                if (!mbar_wait(smem_u32(&cs->full[s]), ph, status)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t st = smem_u32(base + s * STAGE_BYTES);
                const uint64_t ah = swz_desc<KB>(st), al = swz_desc<KB>(st + A_BYTES),
                               bh = swz_desc<KB>(st + 2 * A_BYTES), bl = swz_desc<KB>(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
                for (int k = 0; k < KSTEPS; k++) {
                    const uint64_t dk = (uint64_t)(k * 32) >> 4;  // advance 32 bytes along K
                    const uint32_t first = (kb | k) != 0;
                    umma<KIND>(d, ah + dk, bh + dk, idesc, first);
                    umma<KIND>(d, ah + dk, bl + dk, idesc, 1u);
                    umma<KIND>(d, al + dk, bh + dk, idesc, 1u);
                }
                umma_commit(smem_u32(&cs->empty[s]));  // stage free once these MMAs retire
                g++;
            }
            if (ok) umma_commit(smem_u32(&cs->acc_full[b]));  // tile complete
        }
        // every MMA issued above retires before TMEM is released
        umma_commit(smem_u32(&cs->drain));
        mbar_wait_quiet(smem_u32(&cs->drain), 0u);
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM -> FP64 C
        const int q = warp & 3;  // TMEM lane quarter of this warp
        // EPI / 4 warps share a lane quarter, each draining TN * 4 / EPI columns
        constexpr int CW = TN * 4 / EPI;
        const int cbeg = ((warp - 2) / 4) * CW, cend = cbeg + CW;
        float *stg = reinterpret_cast<float *>(epi_base + (warp - 2) * EPI_WARP_BYTES);
        int64_t *offs = reinterpret_cast<int64_t *>(epi_base + (warp - 2) * EPI_WARP_BYTES + 32 * 33 * 4);
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
            const int b = it & 1;
            bool ok = mbar_wait(smem_u32(&cs->acc_full[b]), ((uint32_t)it >> 1) & 1u, status);
            ok = __all_sync(0xffffffffu, ok && *(volatile int *)status == 0);  // tcgen05.ld is warp-collective
            if (!ok) break;
            tc_fence_after();
            int tm, tn;
            tile_coords(t, num_m, num_n, group_m, tm, tn);
            const int m0 = tm * GM + q * 32, n0 = tn * TN;  // first row of this warp, first column of the tile
            const int m = m0 + lane;
            const int64_t roff = map4_32(epi.row, (uint32_t)(m < M ? m : 0));
            const int nrow = (M - m0) < 32 ? (M - m0) : 32;
            offs[lane] = roff;  // cols mode: row offsets of the warp's 32 rows
            // an FP32 C with beta = 1 accumulates by L2 reductions (C += fp32(alpha acc)): no load
            // round trip per element, the limit of the short-contraction epilogues
            const bool redc = sizeof(CT) == 4 && beta == 1.0;
            // NCH 32-column chunks per step (two chunks' loads in flight measured no faster for an FP32
            // C: one chunk per step for either type)
            constexpr int NCH = 1;
            for (int c = cbeg; c < cend; c += 32 * NCH) {
                bool cval[NCH];
                int64_t coff[NCH];
#pragma unroll
                for (int h = 0; h < NCH; h++) {
                    const int col = n0 + c + 32 * h + lane;
                    cval[h] = col < N;
                    coff[h] = map4_32(epi.col, (uint32_t)(cval[h] ? col : 0));
                }
                // the chunk's accumulator columns; the warp's last load hands the accumulator back
                auto load_acc = [&](int h, float (&v)[32]) {
                    tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * TN + c + 32 * h), v);
                    if (c + 32 * (h + 1) == cend) {
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                                        smem_u32(&cs->acc_empty[b]))
                                                    : "memory");
                    }
                };
                if (epi_cols) {
                    // lanes walk the 32 columns of one row at a time (columns contiguous in C)
                    bool full[NCH];
#pragma unroll
                    for (int h = 0; h < NCH; h++) full[h] = __all_sync(0xffffffffu, cval[h]) && nrow == 32;
                    CT old[NCH][32];
                    if (beta != 0.0 && !redc) {
#pragma unroll
                        for (int h = 0; h < NCH; h++)
                            if (full[h]) {
#pragma unroll
                                for (int r = 0; r < 32; r++) old[h][r] = __ldcg(C + coff[h] + offs[r]);
                            }
                    }
#pragma unroll
                    for (int h = 0; h < NCH; h++) {
                        float v[32];
                        load_acc(h, v);
#pragma unroll
                        for (int j = 0; j < 32; j++) stg[lane * 33 + j] = v[j];
                        __syncwarp();
                        CT *cp = C + coff[h];
                        if (redc) {
                            const int nr = full[h] ? 32 : (cval[h] ? nrow : 0);
#pragma unroll 8
                            for (int r = 0; r < nr; r++) red_add(cp + offs[r], (CT)(alpha * (double)stg[r * 33 + lane]));
                        } else if (beta == 0.0) {
                            if (full[h]) {
#pragma unroll 8
                                for (int r = 0; r < 32; r++) cp[offs[r]] = (CT)(alpha * (double)stg[r * 33 + lane]);
                            } else {
                                for (int r = 0; r < nrow; r++)
                                    if (cval[h]) cp[offs[r]] = (CT)(alpha * (double)stg[r * 33 + lane]);
                            }
                        } else if (full[h]) {
#pragma unroll
                            for (int r = 0; r < 32; r++)
                                cp[offs[r]] = (CT)fma(beta, (double)old[h][r], alpha * (double)stg[r * 33 + lane]);
                        } else {
                            for (int r = 0; r < nrow; r++)
                                if (cval[h])
                                    cp[offs[r]] = (CT)fma(beta, (double)__ldcg(cp + offs[r]),
                                                          alpha * (double)stg[r * 33 + lane]);
                        }
                        __syncwarp();
                    }
                } else {
                    // lanes are rows (rows contiguous in C): each thread writes its row's columns
                    int64_t *coffs = offs + 32;
#pragma unroll
                    for (int h = 0; h < NCH; h++) coffs[32 * h + lane] = coff[h];
                    __syncwarp();
                    int nvalid[NCH];
#pragma unroll
                    for (int h = 0; h < NCH; h++) nvalid[h] = N - n0 - c - 32 * h;
                    CT *rp = C + roff;
                    CT old[NCH][32];
                    if (beta != 0.0 && !redc && m < M) {
#pragma unroll
                        for (int h = 0; h < NCH; h++)
#pragma unroll
                            for (int j = 0; j < 32; j++)
                                old[h][j] = (j < nvalid[h]) ? __ldcg(rp + coffs[32 * h + j]) : (CT)0;
                    }
#pragma unroll
                    for (int h = 0; h < NCH; h++) {
                        float v[32];
                        load_acc(h, v);
                        if (m < M) {
                            if (redc) {
#pragma unroll
                                for (int j = 0; j < 32; j++)
                                    if (j < nvalid[h]) red_add(rp + coffs[32 * h + j], (CT)(alpha * (double)v[j]));
                            } else if (beta == 0.0) {
#pragma unroll
                                for (int j = 0; j < 32; j++)
                                    if (j < nvalid[h]) rp[coffs[32 * h + j]] = (CT)(alpha * (double)v[j]);
                            } else {
#pragma unroll
                                for (int j = 0; j < 32; j++)
                                    if (j < nvalid[h])
                                        rp[coffs[32 * h + j]] = (CT)fma(beta, (double)old[h][j], alpha * (double)v[j]);
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TN) : "memory");
    }
}

// ----------------------------------------------------------------- split kernels

// x = hi + lo with hi = bf16(x), lo = bf16(x - hi).
__device__ __forceinline__ void split_bf16(double x, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn((float)x);
    lo = __float2bfloat16_rn((float)(x - (double)__bfloat162float(hi)));
}

// x = hi + lo with hi, lo rounded to tf32 (10 explicit mantissa bits).
__device__ __forceinline__ float round_tf32(float f) {
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;
    u += 0x1000u;  // round half away from zero on the 13 dropped bits
    u &= 0xffffe000u;
    return __uint_as_float(u);
}
__device__ __forceinline__ void split_tf32(double x, float &hi, float &lo) {
    hi = round_tf32((float)x);
    lo = round_tf32((float)(x - (double)hi));
}

// Generic split of a strided FP64 operand into K-major pieces:
//   dst[m][k0 + k] for m < M, k < kw (k >= K zero-filled) from src[mmap(m) + kmap(k)]
// with four-digit mixed-radix maps; dst rows are ld elements apart, so a
// K-concatenated operand is filled piece by piece.  Reads run along whichever
// index is contiguous in the source (mode 0: k; mode 1: m; mode 2: the middle
// digit of m, the tile's rows then step that digit), writes are 16-byte packs
// along k.
struct SplitMap {
    Map4 m, k;
};

constexpr int SP_TM = 32, SP_TK = 64;
constexpr int SP_WARPS = 4;          // warps per CTA, each with its own tile
constexpr int SP_PITCH = SP_TK + 1;  // staged elements per row (odd: conflict-free column stores)

// One staged element: the two pieces of one FP64 value.  bf16: hi in the low
// half-word, lo in the high one; tf32: the two floats.
template <int KIND>
struct SplitWord;
template <>
struct SplitWord<0> {
    using T = uint32_t;
    static __device__ __forceinline__ T make(double x) {
        __nv_bfloat16 h, l;
        split_bf16(x, h, l);
        return (uint32_t)__bfloat16_as_ushort(h) | ((uint32_t)__bfloat16_as_ushort(l) << 16);
    }
};
template <>
struct SplitWord<1> {
    using T = uint2;
    static __device__ __forceinline__ T make(double x) {
        float h, l;
        split_tf32(x, h, l);
        return make_uint2(__float_as_uint(h), __float_as_uint(l));
    }
};

// Split parameters of one operand (a row of the grouped split's table).
struct SplitArgs {
    void *hi, *lo;
    int64_t M, K, kw, ld, k0;
    SplitMap mp;
    int64_t nty, rmid, rfast;
    // mode 3: a tile's rows take rA values of digit A (contiguous in the source) times
    // 32 / rA values of digit B; the other digits of m come from the tile index
    // (low part below the lower of the two, mid part between them, the rest above)
    int64_t rA, sA, rB, sB, low, mid, loSpan, hiSpan;
    int32_t mode, src_f32;
};

__device__ __forceinline__ double split_src(const double *p, int o) { return __ldg(p + o); }
__device__ __forceinline__ double split_src(const float *p, int o) { return (double)__ldg(p + o); }

// One warp moves one 32-row x 64-k tile (tile row ty, first column kt) with no
// CTA-wide barrier.  Each lane holds its tile row's source address (64-bit)
// and two contraction offsets (32-bit), broadcast by shuffles; loads are
// issued 16 deep, split at once and staged as pieces (4 bytes per element for
// bf16, so 24 warps fit on an SM), then 8 lanes per row gather 8 staged
// elements each and write one 16-byte pack per piece (two for tf32).
template <int KIND, typename S>
__device__ __forceinline__ void split_tile(const S *__restrict__ src, const SplitArgs &a, int64_t ty, int64_t kt,
                                           typename SplitWord<KIND>::T *tile, int lane) {
    using W = typename SplitWord<KIND>::T;
    int64_t row;
    bool rvalid;
    if (a.mode == 2) {
        // the tiles of one (a0, a2) along the contiguous digit are consecutive, so that the
        // segments of one source run are read side by side
        const int64_t R1 = a.rmid, R2 = a.rfast, nb1 = (R1 + SP_TM - 1) / SP_TM;
        const int64_t a1 = (ty % nb1) * SP_TM + lane, a2 = (ty / nb1) % R2, a0 = ty / (R2 * nb1);
        rvalid = a1 < R1;
        row = (a0 * R1 + a1) * R2 + a2;
    } else if (a.mode == 3) {
        const int64_t n2 = SP_TM / a.rA, nb2 = (a.rB + n2 - 1) / n2;
        const int64_t o = ty / nb2, u1 = lane % a.rA, u2 = (ty % nb2) * n2 + lane / a.rA;
        rvalid = lane < a.rA * n2 && u2 < a.rB;
        const int64_t lo = o % a.low, md = (o / a.low) % a.mid, hi = o / (a.low * a.mid);
        row = hi * a.hiSpan + md * a.loSpan + lo + u1 * a.sA + (rvalid ? u2 : 0) * a.sB;
    } else {
        row = ty * SP_TM + lane;
        rvalid = row < a.M;
    }
    // invalid rows read nothing: their base stays at src and every k offset is masked
    const S *base = src + (rvalid ? map4_32(a.mp.m, (uint32_t)row) : 0);
    const int64_t ka = kt + lane, kb = ka + 32;
    const int koa = ka < a.K ? (int)map4_32(a.mp.k, (uint32_t)ka) : -1;
    const int kob = kb < a.K ? (int)map4_32(a.mp.k, (uint32_t)kb) : -1;
    // loads in flight per lane: 16 (also for an FP32 source: 32 in flight measured 1.8x slower)
    if (a.mode == 0) {
#pragma unroll 8
        for (int r = 0; r < SP_TM; r++) {
            const S *b = (const S *)__shfl_sync(0xffffffffu, (unsigned long long)base, r);
            const bool rv = __shfl_sync(0xffffffffu, rvalid, r);
            const double va = (rv && koa >= 0) ? split_src(b, koa) : 0.0;
            const double vb = (rv && kob >= 0) ? split_src(b, kob) : 0.0;
            tile[r * SP_PITCH + lane] = SplitWord<KIND>::make(va);
            tile[r * SP_PITCH + lane + 32] = SplitWord<KIND>::make(vb);
        }
    } else {
        // only the tile's columns below kw are written: stop there (kw - kt is a multiple of 8)
        const int kn = (int)((a.kw - kt) < SP_TK ? (a.kw - kt) : SP_TK);
#pragma unroll 16
        for (int kk = 0; kk < kn; kk++) {
            const int ko = __shfl_sync(0xffffffffu, kk < 32 ? koa : kob, kk & 31);
            const double v = (rvalid && ko >= 0) ? split_src(base, ko) : 0.0;
            tile[lane * SP_PITCH + kk] = SplitWord<KIND>::make(v);
        }
    }
    __syncwarp();
    // lpr lanes per row write 8 columns each: 8 lanes for a full 64-column tile, fewer
    // (and more rows at a time) for a narrow one
    const int64_t kleft = a.kw - kt;
    const int lsh = kleft > 32 ? 3 : (kleft > 16 ? 2 : (kleft > 8 ? 1 : 0));  // log2(lanes per row)
    const int kc = (lane & ((1 << lsh) - 1)) * 8;
    const int64_t kbeg = kt + kc;
    const int rpi = 32 >> lsh;  // rows per iteration
    for (int rr = 0; rr < SP_TM; rr += rpi) {
        const int r = rr + (lane >> lsh);
        const int64_t rrow = __shfl_sync(0xffffffffu, row, r);
        const bool rv = __shfl_sync(0xffffffffu, rvalid, r);
        if (!rv || kbeg >= a.kw) continue;
        const int64_t dst = rrow * a.ld + a.k0 + kbeg;
        const W *tv = tile + r * SP_PITCH + kc;
        if constexpr (KIND == 0) {
            uint32_t e[8];
#pragma unroll
            for (int j = 0; j < 8; j++) e[j] = tv[j];
            __nv_bfloat16 *H = (__nv_bfloat16 *)a.hi + dst, *Lo = (__nv_bfloat16 *)a.lo + dst;
            if (kbeg + 8 <= a.kw && (dst & 7) == 0) {
                uint4 ph, pl;
                ph.x = __byte_perm(e[0], e[1], 0x5410);
                ph.y = __byte_perm(e[2], e[3], 0x5410);
                ph.z = __byte_perm(e[4], e[5], 0x5410);
                ph.w = __byte_perm(e[6], e[7], 0x5410);
                pl.x = __byte_perm(e[0], e[1], 0x7632);
                pl.y = __byte_perm(e[2], e[3], 0x7632);
                pl.z = __byte_perm(e[4], e[5], 0x7632);
                pl.w = __byte_perm(e[6], e[7], 0x7632);
                *(uint4 *)H = ph;
                *(uint4 *)Lo = pl;
            } else {
                for (int j = 0; j < 8 && kbeg + j < a.kw; j++) {
                    H[j] = __ushort_as_bfloat16((unsigned short)(e[j] & 0xffffu));
                    Lo[j] = __ushort_as_bfloat16((unsigned short)(e[j] >> 16));
                }
            }
        } else {
            uint2 e[8];
#pragma unroll
            for (int j = 0; j < 8; j++) e[j] = tv[j];
            float *H = (float *)a.hi + dst, *Lo = (float *)a.lo + dst;
            if (kbeg + 8 <= a.kw && (dst & 3) == 0) {
                ((uint4 *)H)[0] = make_uint4(e[0].x, e[1].x, e[2].x, e[3].x);
                ((uint4 *)H)[1] = make_uint4(e[4].x, e[5].x, e[6].x, e[7].x);
                ((uint4 *)Lo)[0] = make_uint4(e[0].y, e[1].y, e[2].y, e[3].y);
                ((uint4 *)Lo)[1] = make_uint4(e[4].y, e[5].y, e[6].y, e[7].y);
            } else {
                for (int j = 0; j < 8 && kbeg + j < a.kw; j++) {
                    H[j] = __uint_as_float(e[j].x);
                    Lo[j] = __uint_as_float(e[j].y);
                }
            }
        }
    }
    __syncwarp();  // the tile is rewritten by the warp's next item
}

// Tile t of an operand as (tile row, first column).  Where the rows are contiguous in the
// source (mode 1) the row tiles run fastest, so that neighbouring warps read neighbouring
// segments of each source run (at nocc=15 / nvir=93 the W_oooo operand of U 9.4 -> 8.6 ms);
// elsewhere the column tiles do, so that the 16-byte packs of an output row are written side by
// side (the OO operand's piece with k contiguous in U: 9.6 ms, against 13.5 rows first).
__device__ __forceinline__ void split_tile_coords(const SplitArgs &a, int64_t ntk, int64_t t, int64_t &ty,
                                                  int64_t &kt) {
    if (a.mode == 1) {
        ty = t % a.nty;
        kt = (t / a.nty) * SP_TK;
    } else {
        ty = t / ntk;
        kt = (t % ntk) * SP_TK;
    }
}

// Persistent: warp w of CTA c takes tiles c * SP_WARPS + w, + gridDim.x * SP_WARPS, ...
template <int KIND, typename S>
__global__ void __launch_bounds__(32 * SP_WARPS, KIND == 0 ? 6 : 3)
    k_split(const S *__restrict__ src, SplitArgs a) {
    extern __shared__ __align__(16) unsigned char sp_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    auto *tile = reinterpret_cast<typename SplitWord<KIND>::T *>(sp_raw) + w * SP_TM * SP_PITCH;
    const int64_t ntk = (a.kw + SP_TK - 1) / SP_TK;
    const int64_t ntiles = a.nty * ntk;
    for (int64_t t = (int64_t)blockIdx.x * SP_WARPS + w; t < ntiles; t += (int64_t)gridDim.x * SP_WARPS) {
        int64_t ty, kt;
        split_tile_coords(a, ntk, t, ty, kt);
        split_tile<KIND>(src, a, ty, kt, tile, lane);
    }
}

// Grouped split: one launch for many operands.  probs[p] holds operand p's
// parameters and first global tile (tile_begin[p], ascending, with
// tile_begin[nprob] = total); its source address comes from srcs.p[p], so a
// table built once is reused with new sources.
constexpr int SPLIT_GROUP_MAX = DCC_GROUP_MAX;
struct SplitSrcs {
    const void *p[SPLIT_GROUP_MAX];
};
struct SplitProblem {
    SplitArgs a;
    int64_t tile_begin, ntk;
};

template <int KIND>
__global__ void __launch_bounds__(32 * SP_WARPS, KIND == 0 ? 6 : 3)
    k_split_grouped(const SplitProblem *__restrict__ probs, int nprob, int64_t total,
                    const __grid_constant__ SplitSrcs srcs) {
    extern __shared__ __align__(16) unsigned char sp_raw[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    auto *tile = reinterpret_cast<typename SplitWord<KIND>::T *>(sp_raw) + w * SP_TM * SP_PITCH;
    int p = 0;
    for (int64_t t = (int64_t)blockIdx.x * SP_WARPS + w; t < total; t += (int64_t)gridDim.x * SP_WARPS) {
        while (p + 1 < nprob && probs[p + 1].tile_begin <= t) p++;  // t only grows
        const SplitProblem &pr = probs[p];
        const int64_t lt = t - pr.tile_begin;
        int64_t ty, kt;
        split_tile_coords(pr.a, pr.ntk, lt, ty, kt);
        if (pr.a.src_f32)
            split_tile<KIND>((const float *)srcs.p[p], pr.a, ty, kt, tile, lane);
        else
            split_tile<KIND>((const double *)srcs.p[p], pr.a, ty, kt, tile, lane);
    }
}

// Bound on |offset| over the first n indices of a map (a digit never exceeds
// its radix - 1, nor (n - 1) / the product of the radices inside it).
static int64_t map_span(const Map4 &f, int64_t n) {
    const int64_t m = n - 1, r3 = f.R3, r23 = f.R2 * r3, r123 = f.R1 * r23;
    const int64_t d0 = m / r123, d1 = std::min(f.R1 - 1, m / r23), d2 = std::min(f.R2 - 1, m / r3),
                  d3 = std::min(f.R3 - 1, m);
    return d0 * llabs(f.S0) + d1 * llabs(f.S1) + d2 * llabs(f.S2) + d3 * llabs(f.S3);
}

static bool map_ok(const Map4 &f) {
    return f.R1 >= 1 && f.R2 >= 1 && f.R3 >= 1 && f.R1 * f.R2 < (1ll << 31) && f.R1 * f.R2 * f.R3 < (1ll << 31);
}

// ----------------------------------------------------------------- grouped GEMM

// One problem of a grouped GEMM: C[row(m) + col(n)] += alpha * (A B^T)[m][n]
// through reductions in L2 (red.global.add), so problems that write the same
// C run concurrently in one launch.  C is float (out_f32) or double.
struct alignas(64) GemmProblem {
    CUtensorMap tm[4];  // A hi, A lo, B hi, B lo
    GemmEpi epi;
    void *C;
    double alpha;
    int M, N, nkb, epi_cols;
    int num_m, num_n, out_f32, tile_begin;
};

// Tile t's problem: the last p with tile_begin <= t (tile_begin ascending).
__device__ __forceinline__ int grouped_find(const int *tb, int nprob, int t) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tb[mid] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// One 32-column chunk of a warp's 32 rows: C[row(m) + col(n)] += alpha * v.
// Offsets are 32-bit (checked on the host); reductions go along whichever of
// rows or columns is contiguous in C (epi_cols: lanes walk the columns of one
// row at a time through the warp's transpose buffer).
template <typename T>
__device__ __forceinline__ void grouped_store(T *C, T alpha, int epi_cols, const float (&v)[32], float *stg,
                                              int *offs, int lane, bool rvalid, int nrow, int coff, bool cval,
                                              int nvalid, int roff) {
    if (epi_cols) {
#pragma unroll
        for (int j = 0; j < 32; j++) stg[lane * 33 + j] = v[j];
        __syncwarp();
        if (cval) {
            T *cp = C + coff;
            if (nrow == 32) {
#pragma unroll 8
                for (int r = 0; r < 32; r++) red_add(cp + offs[r], alpha * (T)stg[r * 33 + lane]);
            } else {
                for (int r = 0; r < nrow; r++) red_add(cp + offs[r], alpha * (T)stg[r * 33 + lane]);
            }
        }
        __syncwarp();
    } else {
        int *coffs = offs + 32;
        coffs[lane] = coff;
        __syncwarp();
        if (rvalid) {
            T *rp = C + roff;
            if (nvalid == 32) {
#pragma unroll
                for (int j = 0; j < 32; j++) red_add(rp + coffs[j], alpha * (T)v[j]);
            } else {
#pragma unroll
                for (int j = 0; j < 32; j++)
                    if (j < nvalid) red_add(rp + coffs[j], alpha * (T)v[j]);
            }
        }
        __syncwarp();
    }
}

// Persistent over the tiles of all problems (problem p owns global tiles
// [tile_begin[p], tile_begin[p+1])); the pipeline is k_gemm_split3's.
template <int KIND, int KB, int ST, int EPI, typename OutT>
__global__ void __launch_bounds__(gemm_threads<EPI>(), 1)
    k_gemm_grouped(const GemmProblem *__restrict__ probs, int nprob, int ntiles, int *status, int group_m) {
    extern __shared__ __align__(1024) uint8_t g_smem[];
    uint8_t *base = (uint8_t *)(((uintptr_t)g_smem + 1023) & ~(uintptr_t)1023);
    constexpr uint32_t A_BYTES = GM * KB, B_BYTES = GN * KB;
    constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    uint8_t *epi_base = base + ST * STAGE_BYTES;
    GemmSmem<ST> *cs = (GemmSmem<ST> *)(epi_base + EPI * EPI_WARP_BYTES);
    int *tb = (int *)(cs + 1);  // tile_begin of every problem

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the table's output type must be the one this instance writes
    if (probs[0].out_f32 != (sizeof(OutT) == 4 ? 1 : 0)) {
        if (threadIdx.x == 0) atomicExch(status, DCC_ERR_SHAPE);
        return;
    }
    for (int p = threadIdx.x; p < nprob; p += blockDim.x) tb[p] = probs[p].tile_begin;
    if (threadIdx.x == 0) {
        for (int s = 0; s < ST; s++) {
            mbar_init(smem_u32(&cs->full[s]), 1);
            mbar_init(smem_u32(&cs->empty[s]), 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(smem_u32(&cs->acc_full[b]), 1);
            mbar_init(smem_u32(&cs->acc_empty[b]), EPI);
        }
        mbar_init(smem_u32(&cs->drain), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&cs->tmem_base)),
                     "r"(2 * GN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = cs->tmem_base;

    if (warp == 0 && lane == 0) {
        // ---------------- TMA producer
        uint32_t g = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
            const int p = grouped_find(tb, nprob, t);
            const GemmProblem &pr = probs[p];
            int tm, tn;
            tile_coords(t - tb[p], pr.num_m, pr.num_n, group_m, tm, tn);
            const int nkb = pr.nkb;
            for (int kb = 0; kb < nkb; kb++) {
                const uint32_t s = g % ST, ph = (g / ST) & 1u;
                if (!mbar_wait(smem_u32(&cs->empty[s]), ph ^ 1u, status)) {
                    ok = false;
                    break;
                }
                uint8_t *st = base + s * STAGE_BYTES;
                const uint32_t fb = smem_u32(&cs->full[s]);
                mbar_expect_tx(fb, STAGE_BYTES);
                const int kc = kb * (KB / (KIND == 0 ? 2 : 4));
                tma_load_2d(smem_u32(st), &pr.tm[0], fb, kc, tm * GM);
                tma_load_2d(smem_u32(st + A_BYTES), &pr.tm[1], fb, kc, tm * GM);
                tma_load_2d(smem_u32(st + 2 * A_BYTES), &pr.tm[2], fb, kc, tn * GN);
                tma_load_2d(smem_u32(st + 2 * A_BYTES + B_BYTES), &pr.tm[3], fb, kc, tn * GN);
                g++;
            }
        }
        if (!ok) {
            const uint32_t first = g > (uint32_t)ST ? g - ST : 0u;
            for (uint32_t k = first; k < g; k++) mbar_wait_quiet(smem_u32(&cs->full[k % ST]), (k / ST) & 1u);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer
        constexpr uint32_t idesc = (1u << 4) | ((KIND == 0 ? 1u : 2u) << 7) | ((KIND == 0 ? 1u : 2u) << 10) |
                                   ((uint32_t)(GN >> 3) << 17) | ((uint32_t)(GM >> 4) << 24);
        constexpr int KSTEPS = KB / 32;
        uint32_t g = 0;
        bool ok = true;
        int it = 0;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, it++) {
            const int nkb = probs[grouped_find(tb, nprob, t)].nkb;
            const int b = it & 1;
            if (!mbar_wait(smem_u32(&cs->acc_empty[b]), (((uint32_t)it >> 1) & 1u) ^ 1u, status)) break;
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(b * GN);
            for (int kb = 0; kb < nkb; kb++) {
                const uint32_t s = g % ST, ph = (g / ST) & 1u;
                if (!mbar_wait(smem_u32(&cs->full[s]), ph, status)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t st = smem_u32(base + s * STAGE_BYTES);
                const uint64_t ah = swz_desc<KB>(st), al = swz_desc<KB>(st + A_BYTES),
                               bh = swz_desc<KB>(st + 2 * A_BYTES), bl = swz_desc<KB>(st + 2 * A_BYTES + B_BYTES);
#pragma unroll
                for (int k = 0; k < KSTEPS; k++) {
                    const uint64_t dk = (uint64_t)(k * 32) >> 4;
                    const uint32_t first = (kb | k) != 0;
                    umma<KIND>(d, ah + dk, bh + dk, idesc, first);
                    umma<KIND>(d, ah + dk, bl + dk, idesc, 1u);
                    umma<KIND>(d, al + dk, bh + dk, idesc, 1u);
                }
                umma_commit(smem_u32(&cs->empty[s]));
                g++;
            }
            if (ok) umma_commit(smem_u32(&cs->acc_full[b]));
        }
        umma_commit(smem_u32(&cs->drain));
        mbar_wait_quiet(smem_u32(&cs->drain), 0u);
    } else if (warp >= 2) {
        // ---------------- epilogue: TMEM -> reductions into C
        const int q = warp & 3;
        constexpr int CW = GN * 4 / EPI;
        const int cbeg = ((warp - 2) / 4) * CW, cend = cbeg + CW;
        float *stg = reinterpret_cast<float *>(epi_base + (warp - 2) * EPI_WARP_BYTES);
        int *offs = reinterpret_cast<int *>(epi_base + (warp - 2) * EPI_WARP_BYTES + 32 * 33 * 4);
        int it = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, it++) {
            const int b = it & 1;
            bool ok = mbar_wait(smem_u32(&cs->acc_full[b]), ((uint32_t)it >> 1) & 1u, status);
            ok = __all_sync(0xffffffffu, ok && *(volatile int *)status == 0);
            if (!ok) break;
            tc_fence_after();
            const int p = grouped_find(tb, nprob, t);
            const GemmProblem &pr = probs[p];
            const int M = pr.M, N = pr.N, epi_cols = pr.epi_cols;
            const Map4 rmap = pr.epi.row, cmap = pr.epi.col;
            OutT *C = (OutT *)pr.C;
            const OutT alpha = (OutT)pr.alpha;
            int tm, tn;
            tile_coords(t - tb[p], pr.num_m, pr.num_n, group_m, tm, tn);
            const int m0 = tm * GM + q * 32, n0 = tn * GN;
            const int m = m0 + lane;
            const int roff = (int)map4_32(rmap, (uint32_t)(m < M ? m : 0));
            const int nrow = (M - m0) < 32 ? ((M - m0) > 0 ? (M - m0) : 0) : 32;
            offs[lane] = roff;
            for (int c = cbeg; c < cend; c += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * GN + c), v);
                if (c == cend - 32) {
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                                    smem_u32(&cs->acc_empty[b]))
                                                : "memory");
                }
                const int col = n0 + c + lane;
                if (n0 + c >= N) continue;  // warp-uniform: the chunk is past the last column
                const bool cval = col < N;
                const int coff = (int)map4_32(cmap, (uint32_t)(cval ? col : 0));
                const int nvalid = (N - n0 - c) < 32 ? (N - n0 - c) : 32;
                grouped_store<OutT>(C, alpha, epi_cols, v, stg, offs, lane, m < M, nrow, coff, cval, nvalid, roff);
            }
            __syncwarp();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * GN) : "memory");
    }
}

// ----------------------------------------------------------------- host side

// 2-D K-major piece [rows][Kp] with a (k-block x box_rows) box and the
// swizzle that matches kb_bytes.
static int make_map(CUtensorMap *map, const void *ptr, int kind, int64_t rows, int64_t Kp, int64_t ld,
                    int box_rows, int kb_bytes) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is unavailable");
        return DCC_ERR_CUDA;
    }
    const int esz = kind == 0 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * esz)};
    cuuint32_t box[2] = {(cuuint32_t)(kb_bytes / esz), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMapSwizzle sw = kb_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                                            : (kb_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
    CUresult r = fn(map, kind == 0 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                    const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, sw,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return DCC_ERR_CUDA;
    }
    return DCC_OK;
}

template <int ST, int EPI, int TN = GN>
static size_t gemm_smem_bytes(int kb_bytes) {
    return 1024 + ST * (size_t)(2 * GM * kb_bytes + 2 * TN * kb_bytes) + EPI * EPI_WARP_BYTES +
           sizeof(GemmSmem<ST>);
}

template <int KIND, int KB, int ST, int EPI, typename CT = double, int TN = GN>
static int gemm_launch(const CUtensorMap &a, const CUtensorMap &b, const CUtensorMap &c, const CUtensorMap &d, int M,
                       int N, int nkb, CT *C, const GemmEpi &epi, double alpha, double beta, int *status,
                       int group_m, cudaStream_t st) {
    // write along columns when the column map's fastest digit is contiguous,
    // along rows when only the row map's is
    int64_t cs, cr, rs, rr;
    fast_digit(epi.col, cs, cr);
    fast_digit(epi.row, rs, rr);
    const int epi_cols = (cs == 1 || rs != 1) ? 1 : 0;
    size_t smem = gemm_smem_bytes<ST, EPI, TN>(KB);
    const int64_t tiles = (int64_t)ceil_div(N, TN) * (int64_t)ceil_div(M, GM);
    DCC_REQUIRE(tiles < (1ll << 31), DCC_ERR_SHAPE, "too many output tiles");
    int dev = 0, nsm = 148, per_sm = 1;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    auto kern = k_gemm_split3<KIND, KB, ST, EPI, CT, TN>;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // persistent: as many CTAs as fit at once (one per SM for 256-column tiles, up to two for 128)
    constexpr int max_per_sm = TN == GN ? 1 : 2;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, gemm_threads<EPI>(), smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    per_sm = per_sm > max_per_sm ? max_per_sm : per_sm;
    const int64_t cap = (int64_t)nsm * per_sm;
    const unsigned grid = (unsigned)(tiles < cap ? tiles : cap);
    kern<<<grid, gemm_threads<EPI>(), smem, st>>>(a, b, c, d, M, N, nkb, C, epi, alpha, beta, status, group_m, epi_cols);
    return launch_status("gemm_split3");
}

}  // namespace dcc

using namespace dcc;

// Validated split parameters (mode and tile rows chosen for the maps).
static int split_args(void *hi, void *lo, int64_t M, int64_t K, int64_t kw, int64_t ld, int64_t k0,
                      const int64_t *maps, bool four, int src_f32, SplitArgs &a) {
    DCC_REQUIRE(M >= 0 && K >= 0 && kw >= K && k0 >= 0 && k0 + kw <= ld, DCC_ERR_SHAPE,
                "bad split sizes (M=%lld K=%lld kw=%lld k0=%lld ld=%lld)", (long long)M, (long long)K, (long long)kw,
                (long long)k0, (long long)ld);
    DCC_REQUIRE(hi && lo && maps, DCC_ERR_NULL, "NULL buffer");
    SplitMap mp{map_from(maps, four), map_from(maps + (four ? 7 : 5), four)};
    DCC_REQUIRE(map_ok(mp.m) && map_ok(mp.k), DCC_ERR_SHAPE, "map radices must be >= 1 with products < 2^31");
    DCC_REQUIRE(M < (1ll << 31) && ld < (1ll << 31), DCC_ERR_SHAPE, "split sizes must fit in 31 bits");
    DCC_REQUIRE(K == 0 || map_span(mp.k, K) < (1ll << 31), DCC_ERR_SHAPE, "contraction offsets must fit in 31 bits");
    // read along the contiguous source index: k (mode 0), else m's fastest digit
    // (mode 1), else another digit of m (mode 2: a tile's 32 rows step that digit)
    int64_t ks, kr, ms, mr;
    fast_digit(mp.k, ks, kr);
    fast_digit(mp.m, ms, mr);
    int mode = -1;
    int64_t rrad = 1, rstep = 1;
    int64_t m3[8] = {1, 0, 1, 0, 1, 1, 1, 1};  // rA, sA, rB, sB, low, mid, loSpan, hiSpan
    if (ks == 1 && kr >= 16) {
        mode = 0;
    } else if (ms == 1 || mr == 1) {
        mode = 1;
    } else {
        // digits of m from the fastest: radix, stride, and step (product of the radices below)
        const Map4 &f = mp.m;
        const int64_t inner = f.R1 * f.R2 * f.R3;
        const int64_t rad[4] = {f.R3, f.R2, f.R1, M % inner == 0 ? M / inner : 0};
        const int64_t str[4] = {f.S3, f.S2, f.S1, f.S0};
        const int64_t stp[4] = {1, f.R3, f.R2 * f.R3, inner};
        int q1 = -1;
        for (int q = 1; q < 4; q++)
            if (rad[q] >= 2 && llabs(str[q]) == 1) {
                q1 = q;
                break;
            }
        if (q1 >= 0 && rad[q1] >= SP_TM && M % (rad[q1] * stp[q1]) == 0) {
            mode = 2;  // 32 rows along the contiguous digit
            rrad = rad[q1];
            rstep = stp[q1];
        } else if (q1 >= 0 && rad[3] > 0) {
            // a short contiguous digit: pair it with the digit that continues it in the
            // source (stride = its radix), else with the longest other digit
            int q2 = -1;
            for (int q = 0; q < 4; q++)
                if (q != q1 && rad[q] >= 2 && llabs(str[q]) == rad[q1]) q2 = q;
            if (q2 < 0)
                for (int q = 0; q < 4; q++)
                    if (q != q1 && rad[q] >= 2 && (q2 < 0 || rad[q] > rad[q2])) q2 = q;
            if (q2 >= 0) {
                mode = 3;
                const int ql = q1 < q2 ? q1 : q2, qh = q1 < q2 ? q2 : q1;
                m3[0] = rad[q1];
                m3[1] = stp[q1];
                m3[2] = rad[q2];
                m3[3] = stp[q2];
                m3[4] = stp[ql];
                m3[5] = stp[qh] / (stp[ql] * rad[ql]);
                m3[6] = stp[ql] * rad[ql];
                m3[7] = stp[qh] * rad[qh];
            }
        }
        if (mode < 0) mode = ks == 1 ? 0 : 1;
    }
    int64_t nty;
    if (mode == 2)
        nty = (M / (rrad * rstep)) * ((rrad + SP_TM - 1) / SP_TM) * rstep;
    else if (mode == 3) {
        const int64_t n2 = SP_TM / m3[0];
        nty = (M / (m3[0] * m3[2])) * ((m3[2] + n2 - 1) / n2);
    } else
        nty = (M + SP_TM - 1) / SP_TM;
    a = SplitArgs{hi, lo, M, K, kw, ld, k0, mp, nty, rrad, rstep,
                  m3[0], m3[1], m3[2], m3[3], m3[4], m3[5], m3[6], m3[7], mode, src_f32};
    return DCC_OK;
}

static size_t split_smem(int kind) { return (size_t)SP_WARPS * SP_TM * SP_PITCH * (kind == 0 ? 4 : 8); }

static unsigned split_grid(int64_t ntiles, int kind) {
    const int64_t nwarp_blocks = (ntiles + SP_WARPS - 1) / SP_WARPS;
    const int per_sm = kind == 0 ? 6 : 3;  // resident CTAs per SM (shared memory bound)
    return (unsigned)(nwarp_blocks < 148 * per_sm ? nwarp_blocks : 148 * per_sm);  // persistent
}

// S: the source type (double, or float for the FP32 copies of T3 in the split precisions; a
// float's pieces are those of the same value as a double)
template <typename S>
static int split_operand(const S *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw, int64_t ld,
                         int64_t k0, const int64_t *maps, bool four, int kind, void *stream) {
    clear_error();
    DCC_REQUIRE(kind == 0 || kind == 1, DCC_ERR_UNSUPPORTED, "split kind must be 0 (bf16) or 1 (tf32)");
    if (M == 0 || kw == 0) return DCC_OK;
    DCC_REQUIRE(src, DCC_ERR_NULL, "NULL buffer");
    SplitArgs a;
    int rc = split_args(hi, lo, M, K, kw, ld, k0, maps, four, sizeof(S) == 4 ? 1 : 0, a);
    if (rc) return rc;
    const int64_t ntiles = a.nty * ((kw + SP_TK - 1) / SP_TK);
    const unsigned grid = split_grid(ntiles, kind);
    const size_t smem = split_smem(kind);
    if (kind == 0) {
        cudaFuncSetAttribute(k_split<0, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_split<0, S><<<grid, 32 * SP_WARPS, smem, as_stream(stream)>>>(src, a);
    } else {
        cudaFuncSetAttribute(k_split<1, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_split<1, S><<<grid, 32 * SP_WARPS, smem, as_stream(stream)>>>(src, a);
    }
    return launch_status("split_operand");
}

extern "C" size_t dcc_split_grouped_table_bytes(int nprob) {
    return nprob > 0 ? (size_t)nprob * sizeof(SplitProblem) : 0;
}

extern "C" int dcc_split_grouped_table(const int64_t *spec, int nprob, void *table, size_t table_bytes,
                                       int64_t *total_tiles) {
    clear_error();
    DCC_REQUIRE(nprob >= 1 && nprob <= SPLIT_GROUP_MAX, DCC_ERR_SHAPE, "nprob must be in [1, %d]",
                SPLIT_GROUP_MAX);
    DCC_REQUIRE(spec && table && total_tiles, DCC_ERR_NULL, "NULL argument");
    DCC_REQUIRE(table_bytes >= dcc_split_grouped_table_bytes(nprob), DCC_ERR_WORKSPACE, "table needs %zu bytes",
                dcc_split_grouped_table_bytes(nprob));
    SplitProblem *h = (SplitProblem *)malloc(sizeof(SplitProblem) * nprob);
    DCC_REQUIRE(h, DCC_ERR_CUDA, "host allocation failed");
    int64_t total = 0;
    for (int p = 0; p < nprob; p++) {
        const int64_t *v = spec + (int64_t)p * DCC_SPLIT_SPEC;
        int rc = split_args((void *)v[0], (void *)v[1], v[2], v[3], v[4], v[5], v[6], v + 7, true, (int)v[21], h[p].a);
        if (rc == DCC_OK && !(v[21] == 0 || v[21] == 1)) {
            set_error("source type flag must be 0 (float64) or 1 (float32)");
            rc = DCC_ERR_SHAPE;
        }
        if (rc) {
            free(h);
            return rc;
        }
        h[p].ntk = (h[p].a.kw + SP_TK - 1) / SP_TK;
        h[p].tile_begin = total;
        total += h[p].a.M > 0 ? h[p].a.nty * h[p].ntk : 0;
    }
    cudaError_t e = cudaMemcpy(table, h, sizeof(SplitProblem) * nprob, cudaMemcpyHostToDevice);
    free(h);
    DCC_REQUIRE(e == cudaSuccess, DCC_ERR_CUDA, "table upload failed: %s", cudaGetErrorString(e));
    *total_tiles = total;
    return DCC_OK;
}

extern "C" int dcc_split_grouped(const void *table, int nprob, int64_t total_tiles, const void *const *srcs, int kind,
                                 void *stream) {
    clear_error();
    DCC_REQUIRE(kind == 0 || kind == 1, DCC_ERR_UNSUPPORTED, "split kind must be 0 (bf16) or 1 (tf32)");
    DCC_REQUIRE(nprob >= 1 && nprob <= SPLIT_GROUP_MAX, DCC_ERR_SHAPE, "nprob must be in [1, %d]",
                SPLIT_GROUP_MAX);
    DCC_REQUIRE(table && srcs, DCC_ERR_NULL, "NULL argument");
    DCC_REQUIRE(total_tiles >= 0, DCC_ERR_SHAPE, "negative tile count");
    if (total_tiles == 0) return DCC_OK;
    SplitSrcs s{};
    for (int p = 0; p < nprob; p++) {
        DCC_REQUIRE(srcs[p], DCC_ERR_NULL, "NULL source of operand %d", p);
        s.p[p] = srcs[p];
    }
    const unsigned grid = split_grid(total_tiles, kind);
    const size_t smem = split_smem(kind);
    const SplitProblem *pr = (const SplitProblem *)table;
    if (kind == 0) {
        cudaFuncSetAttribute(k_split_grouped<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_split_grouped<0><<<grid, 32 * SP_WARPS, smem, as_stream(stream)>>>(pr, nprob, total_tiles, s);
    } else {
        cudaFuncSetAttribute(k_split_grouped<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_split_grouped<1><<<grid, 32 * SP_WARPS, smem, as_stream(stream)>>>(pr, nprob, total_tiles, s);
    }
    return launch_status("split_grouped");
}

extern "C" int dcc_split_operand_at(const double *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw,
                                    int64_t ld, int64_t k0, const int64_t *map10, int kind, void *stream) {
    return split_operand(src, hi, lo, M, K, kw, ld, k0, map10, false, kind, stream);
}

extern "C" int dcc_split_operand_at4(const double *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw,
                                     int64_t ld, int64_t k0, const int64_t *map14, int kind, void *stream) {
    return split_operand(src, hi, lo, M, K, kw, ld, k0, map14, true, kind, stream);
}

extern "C" int dcc_split_operand_at4_f32(const float *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw,
                                         int64_t ld, int64_t k0, const int64_t *map14, int kind, void *stream) {
    return split_operand(src, hi, lo, M, K, kw, ld, k0, map14, true, kind, stream);
}

extern "C" int dcc_split_operand(const double *src, void *hi, void *lo, int64_t M, int64_t K, int64_t Kp,
                                 const int64_t *map10, int kind, void *stream) {
    return dcc_split_operand_at(src, hi, lo, M, K, Kp, Kp, 0, map10, kind, stream);
}

static int gemm_split3(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi, const void *B_lo,
                       int64_t ldb, int64_t M, int64_t N, int64_t Kp, void *C, const int64_t *epi, bool four,
                       double alpha, double beta, int kind, int *status, void *stream, bool c_f32 = false) {
    clear_error();
    DCC_REQUIRE(kind == 0 || kind == 1, DCC_ERR_UNSUPPORTED, "kind must be 0 (bf16x3) or 1 (tf32x3)");
    const int kblk = kind == 0 ? 64 : 32;
    DCC_REQUIRE(M >= 0 && N >= 0 && Kp >= 0 && Kp % kblk == 0, DCC_ERR_SHAPE,
                "Kp (%lld) must be a multiple of %d", (long long)Kp, kblk);
    DCC_REQUIRE(M < (1ll << 31) && N < (1ll << 31), DCC_ERR_SHAPE, "M, N must fit in 31 bits");
    DCC_REQUIRE(lda >= Kp && ldb >= Kp && lda % 8 == 0 && ldb % 8 == 0 && lda < (1ll << 31) && ldb < (1ll << 31),
                DCC_ERR_SHAPE, "row pitches (lda=%lld ldb=%lld) must be >= Kp and multiples of 8", (long long)lda,
                (long long)ldb);
    if (M == 0 || N == 0) return DCC_OK;
    DCC_REQUIRE(A_hi && A_lo && B_hi && B_lo && C && epi && status, DCC_ERR_NULL, "NULL buffer");
    DCC_REQUIRE(Kp > 0, DCC_ERR_SHAPE, "empty contraction");
    GemmEpi ep{map_from(epi, four), map_from(epi + (four ? 7 : 5), four)};
    DCC_REQUIRE(map_ok(ep.row) && map_ok(ep.col), DCC_ERR_SHAPE, "map radices must be >= 1 with products < 2^31");
    const GemmConfig cfg = g_cfg;
    // 128-column tiles have one pipeline for every K and C type: 64-byte k-blocks, 2 stages, 4 epilogue warps
    const bool narrow = cfg.tile_n == 128;
    DCC_REQUIRE(Kp % ((narrow ? 64 : cfg.kb_bytes) / (kind == 0 ? 2 : 4)) == 0, DCC_ERR_SHAPE,
                "Kp (%lld) must be a multiple of the k-block", (long long)Kp);
    // Short contractions are bound by the FP64 epilogue: eight epilogue warps
    // (two per TMEM lane quarter) double its memory parallelism; the ring then
    // is three 64-byte stages to make room for their staging buffers.
    const int esz = kind == 0 ? 2 : 4;
    // an FP32 C always takes the wide epilogue (its only instantiation)
    const bool wide_epi = Kp <= 4096 || c_f32;
    const int kb = (wide_epi || narrow) ? 64 : cfg.kb_bytes;
    const int tn = narrow ? 128 : GN;
    CUtensorMap mAh, mAl, mBh, mBl;
    int rc;
    if ((rc = make_map(&mAh, A_hi, kind, M, Kp, lda, GM, kb)) || (rc = make_map(&mAl, A_lo, kind, M, Kp, lda, GM, kb)) ||
        (rc = make_map(&mBh, B_hi, kind, N, Kp, ldb, tn, kb)) || (rc = make_map(&mBl, B_lo, kind, N, Kp, ldb, tn, kb)))
        return rc;
    cudaStream_t st = as_stream(stream);
    const int nkb = (int)(Kp / (kb / esz));
    const int iM = (int)M, iN = (int)N, gm = cfg.group_m;
    if (narrow) {
        if (c_f32) {
            float *Cf = (float *)C;
            if (kind == 0)
                return gemm_launch<0, 64, 2, 4, float, 128>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cf, ep, alpha, beta, status,
                                                            gm, st);
            return gemm_launch<1, 64, 2, 4, float, 128>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cf, ep, alpha, beta, status, gm,
                                                        st);
        }
        double *Cn = (double *)C;
        if (kind == 0)
            return gemm_launch<0, 64, 2, 4, double, 128>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cn, ep, alpha, beta, status, gm,
                                                         st);
        return gemm_launch<1, 64, 2, 4, double, 128>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cn, ep, alpha, beta, status, gm, st);
    }
    if (c_f32) {
        float *Cf = (float *)C;
        if (kind == 0) return gemm_launch<0, 64, 3, 8>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cf, ep, alpha, beta, status, gm, st);
        return gemm_launch<1, 64, 3, 8>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cf, ep, alpha, beta, status, gm, st);
    }
    double *Cd = (double *)C;
    if (wide_epi) {
        if (kind == 0) return gemm_launch<0, 64, 3, 8>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cd, ep, alpha, beta, status, gm, st);
        return gemm_launch<1, 64, 3, 8>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cd, ep, alpha, beta, status, gm, st);
    }
#define DCC_GEMM_CASE(K_, KB_, ST_)                                                                           \
    if (kind == K_ && cfg.kb_bytes == KB_ && cfg.stages == ST_)                                              \
        return gemm_launch<K_, KB_, ST_, 4>(mAh, mAl, mBh, mBl, iM, iN, nkb, Cd, ep, alpha, beta, status, gm, st);
    DCC_GEMM_CASE(0, 128, 2)
    DCC_GEMM_CASE(0, 64, 4)
    DCC_GEMM_CASE(0, 64, 3)
    DCC_GEMM_CASE(0, 32, 8)
    DCC_GEMM_CASE(1, 128, 2)
    DCC_GEMM_CASE(1, 64, 4)
    DCC_GEMM_CASE(1, 64, 3)
    DCC_GEMM_CASE(1, 32, 8)
#undef DCC_GEMM_CASE
    set_error("no kernel for k-block %d bytes x %d stages", cfg.kb_bytes, cfg.stages);
    return DCC_ERR_UNSUPPORTED;
}

extern "C" int dcc_gemm_split3_ld(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi,
                                  const void *B_lo, int64_t ldb, int64_t M, int64_t N, int64_t Kp, double *C,
                                  const int64_t *epi10, double alpha, double beta, int kind, int *status,
                                  void *stream) {
    return gemm_split3(A_hi, A_lo, lda, B_hi, B_lo, ldb, M, N, Kp, C, epi10, false, alpha, beta, kind, status, stream);
}

extern "C" int dcc_gemm_split3_ld4(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi,
                                   const void *B_lo, int64_t ldb, int64_t M, int64_t N, int64_t Kp, double *C,
                                   const int64_t *epi14, double alpha, double beta, int kind, int *status,
                                   void *stream) {
    return gemm_split3(A_hi, A_lo, lda, B_hi, B_lo, ldb, M, N, Kp, C, epi14, true, alpha, beta, kind, status, stream);
}

extern "C" int dcc_gemm_split3_ld4_f32c(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi,
                                        const void *B_lo, int64_t ldb, int64_t M, int64_t N, int64_t Kp, float *C,
                                        const int64_t *epi14, double alpha, double beta, int kind, int *status,
                                        void *stream) {
    return gemm_split3(A_hi, A_lo, lda, B_hi, B_lo, ldb, M, N, Kp, C, epi14, true, alpha, beta, kind, status, stream,
                       true);
}

extern "C" int dcc_gemm_split3(const void *A_hi, const void *A_lo, const void *B_hi, const void *B_lo, int64_t M,
                               int64_t N, int64_t Kp, double *C, const int64_t *epi10, double alpha, double beta,
                               int kind, int *status, void *stream) {
    return dcc_gemm_split3_ld(A_hi, A_lo, Kp, B_hi, B_lo, Kp, M, N, Kp, C, epi10, alpha, beta, kind, status, stream);
}

extern "C" size_t dcc_gemm_grouped_table_bytes(int nprob) {
    return nprob > 0 ? (size_t)nprob * sizeof(GemmProblem) : 0;
}

extern "C" int dcc_gemm_grouped_table(const int64_t *spec, const double *alpha, int nprob, int kind, void *table,
                                      size_t table_bytes, int64_t *total_tiles) {
    clear_error();
    DCC_REQUIRE(kind == 0 || kind == 1, DCC_ERR_UNSUPPORTED, "kind must be 0 (bf16x3) or 1 (tf32x3)");
    DCC_REQUIRE(nprob >= 1 && nprob <= DCC_GROUP_MAX, DCC_ERR_SHAPE, "nprob must be in [1, %d]", DCC_GROUP_MAX);
    DCC_REQUIRE(spec && alpha && table && total_tiles, DCC_ERR_NULL, "NULL argument");
    DCC_REQUIRE(table_bytes >= dcc_gemm_grouped_table_bytes(nprob), DCC_ERR_WORKSPACE, "table needs %zu bytes",
                dcc_gemm_grouped_table_bytes(nprob));
    DCC_REQUIRE(((uintptr_t)table & 63) == 0, DCC_ERR_SHAPE, "table must be 64-byte aligned");
    const int kb = 64, esz = kind == 0 ? 2 : 4, kblk = kb / esz;
    GemmProblem *h = (GemmProblem *)aligned_alloc(64, sizeof(GemmProblem) * nprob);
    DCC_REQUIRE(h, DCC_ERR_CUDA, "host allocation failed");
    memset((void *)h, 0, sizeof(GemmProblem) * nprob);
    int64_t total = 0;
    int rc = DCC_OK;
    for (int p = 0; p < nprob && rc == DCC_OK; p++) {
        const int64_t *v = spec + (int64_t)p * DCC_GEMM_SPEC;
        const int64_t lda = v[2], ldb = v[5], M = v[6], N = v[7], Kp = v[8];
        // a pitch below Kp stores only the leading lda columns: the tensor map then
        // ends there and the TMA fills the rest of each k-block with zeros
        if (!(M >= 1 && N >= 1 && M < (1ll << 31) && N < (1ll << 31) && Kp >= kblk && Kp % kblk == 0 && lda >= 8 &&
              ldb >= 8 && lda % 8 == 0 && ldb % 8 == 0 && lda < (1ll << 31) && ldb < (1ll << 31))) {
            set_error("problem %d: bad sizes (M=%lld N=%lld Kp=%lld lda=%lld ldb=%lld)", p, (long long)M,
                      (long long)N, (long long)Kp, (long long)lda, (long long)ldb);
            rc = DCC_ERR_SHAPE;
            break;
        }
        if (!(v[0] && v[1] && v[3] && v[4] && v[9]) || !(v[10] == 0 || v[10] == 1)) {
            set_error("problem %d: NULL operand or bad output type", p);
            rc = DCC_ERR_NULL;
            break;
        }
        GemmProblem &g = h[p];
        g.epi = GemmEpi{map_from(v + 11, true), map_from(v + 18, true)};
        if (!map_ok(g.epi.row) || !map_ok(g.epi.col)) {
            set_error("problem %d: map radices must be >= 1 with products < 2^31", p);
            rc = DCC_ERR_SHAPE;
            break;
        }
        const int64_t ka = lda < Kp ? lda : Kp, kb_ = ldb < Kp ? ldb : Kp;
        if ((rc = make_map(&g.tm[0], (void *)v[0], kind, M, ka, lda, GM, kb)) ||
            (rc = make_map(&g.tm[1], (void *)v[1], kind, M, ka, lda, GM, kb)) ||
            (rc = make_map(&g.tm[2], (void *)v[3], kind, N, kb_, ldb, GN, kb)) ||
            (rc = make_map(&g.tm[3], (void *)v[4], kind, N, kb_, ldb, GN, kb)))
            break;
        if (map_span(g.epi.row, M) + map_span(g.epi.col, N) >= (1ll << 31)) {
            set_error("problem %d: output offsets must fit in 31 bits", p);
            rc = DCC_ERR_SHAPE;
            break;
        }
        if (v[10] != spec[10]) {
            set_error("problem %d: every problem of a table has the same output type", p);
            rc = DCC_ERR_SHAPE;
            break;
        }
        int64_t cs, cr, rs, rr;
        fast_digit(g.epi.col, cs, cr);
        fast_digit(g.epi.row, rs, rr);
        g.epi_cols = (cs == 1 || rs != 1) ? 1 : 0;
        g.C = (void *)v[9];
        g.out_f32 = (int)v[10];
        g.alpha = alpha[p];
        g.M = (int)M;
        g.N = (int)N;
        g.nkb = (int)(Kp / kblk);
        g.num_m = (int)ceil_div(M, GM);
        g.num_n = (int)ceil_div(N, GN);
        g.tile_begin = (int)total;
        total += (int64_t)g.num_m * g.num_n;
        if (total >= (1ll << 31)) {
            set_error("too many output tiles");
            rc = DCC_ERR_SHAPE;
        }
    }
    if (rc == DCC_OK) {
        cudaError_t e = cudaMemcpy(table, h, sizeof(GemmProblem) * nprob, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            set_error("table upload failed: %s", cudaGetErrorString(e));
            rc = DCC_ERR_CUDA;
        }
    }
    free(h);
    if (rc == DCC_OK) *total_tiles = total;
    return rc;
}

extern "C" int dcc_gemm_grouped(const void *table, int nprob, int64_t total_tiles, int kind, int out_f32,
                                int *status, void *stream) {
    clear_error();
    DCC_REQUIRE(kind == 0 || kind == 1, DCC_ERR_UNSUPPORTED, "kind must be 0 (bf16x3) or 1 (tf32x3)");
    DCC_REQUIRE(nprob >= 1 && nprob <= DCC_GROUP_MAX, DCC_ERR_SHAPE, "nprob must be in [1, %d]", DCC_GROUP_MAX);
    DCC_REQUIRE(table && status, DCC_ERR_NULL, "NULL argument");
    DCC_REQUIRE(out_f32 == 0 || out_f32 == 1, DCC_ERR_SHAPE, "out_f32 must be 0 or 1");
    DCC_REQUIRE(total_tiles >= 0 && total_tiles < (1ll << 31), DCC_ERR_SHAPE, "bad tile count");
    if (total_tiles == 0) return DCC_OK;
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)(total_tiles < nsm ? total_tiles : nsm);
    constexpr int GE = 16;  // epilogue warps: the reductions, not the MMAs, bound these short-K problems
    const size_t smem = gemm_smem_bytes<3, GE>(64) + (size_t)nprob * sizeof(int);
    const GemmProblem *pr = (const GemmProblem *)table;
    cudaStream_t st = as_stream(stream);
    const int gm = g_cfg.group_m;
#define DCC_GROUPED(K_, T_)                                                                                       \
    do {                                                                                                          \
        cudaFuncSetAttribute(k_gemm_grouped<K_, 64, 3, GE, T_>, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                             (int)smem);                                                                          \
        k_gemm_grouped<K_, 64, 3, GE, T_><<<grid, gemm_threads<GE>(), smem, st>>>(pr, nprob, (int)total_tiles,   \
                                                                                  status, gm);                   \
    } while (0)
    if (kind == 0 && out_f32)
        DCC_GROUPED(0, float);
    else if (kind == 0)
        DCC_GROUPED(0, double);
    else if (out_f32)
        DCC_GROUPED(1, float);
    else
        DCC_GROUPED(1, double);
#undef DCC_GROUPED
    return launch_status("gemm_grouped");
}

extern "C" int dcc_gemm_set_tile_config(int kb_bytes, int stages, int group_m, int tile_n) {
    clear_error();
    DCC_REQUIRE(tile_n == 256 || tile_n == 128, DCC_ERR_UNSUPPORTED, "tile_n must be 256 or 128 (%d)", tile_n);
    const bool ok = tile_n == 128 ? (kb_bytes == 64 && stages == 2)
                                  : ((kb_bytes == 128 && stages == 2) || (kb_bytes == 64 && (stages == 3 || stages == 4)) ||
                                     (kb_bytes == 32 && stages == 8));
    DCC_REQUIRE(ok, DCC_ERR_UNSUPPORTED, "unsupported pipeline (k-block %d bytes, %d stages, %d-column tiles)", kb_bytes,
                stages, tile_n);
    DCC_REQUIRE(group_m >= 1 && group_m <= 4096, DCC_ERR_SHAPE, "group_m must be in [1, 4096]");
    dcc::g_cfg = dcc::GemmConfig{kb_bytes, stages, group_m, tile_n};
    return DCC_OK;
}

extern "C" int dcc_gemm_set_config(int kb_bytes, int stages, int group_m) {
    return dcc_gemm_set_tile_config(kb_bytes, stages, group_m, 256);
}

extern "C" int dcc_gemm_get_tile_config(int *kb_bytes, int *stages, int *group_m, int *tile_n) {
    clear_error();
    DCC_REQUIRE(kb_bytes && stages && group_m && tile_n, DCC_ERR_NULL, "NULL argument");
    *kb_bytes = dcc::g_cfg.kb_bytes;
    *stages = dcc::g_cfg.stages;
    *group_m = dcc::g_cfg.group_m;
    *tile_n = dcc::g_cfg.tile_n;
    return DCC_OK;
}

extern "C" int dcc_gemm_get_config(int *kb_bytes, int *stages, int *group_m) {
    int tn = 0;
    return dcc_gemm_get_tile_config(kb_bytes, stages, group_m, &tn);
}
