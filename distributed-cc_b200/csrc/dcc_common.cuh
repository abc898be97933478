// Shared plumbing for the dcc_b200 CUDA library: status codes, the per-thread
// error string behind dcc_last_error(), stream casts and the non-contracting
// FP64 arithmetic used wherever results must match the reference C helpers
// bit for bit (those were built as ISO C11 without FMA contraction).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/dcc_b200.h"

namespace dcc {

void set_error(const char *fmt, ...);
void clear_error();

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Map the reference's pattern strings to coefficient sets.
// P3 (src/rccsdt.c:135-152): P3_full, P3_422, P3_201.
// P4 (src/rccsdt_q.c:49-85, src/rccsdtq.c:324-350): P4_full, P4_444, P4_442, P4_201.
int p3_pattern(const char *name, double p[5]);
int p4_pattern(const char *name, double p[9]);

// Status after a launch: DCC_ERR_CUDA with the runtime's message on failure.
int launch_status(const char *what);

// A process-unique id of the calling thread's current CUDA context (0 when there is none).
// Caches of device-symbol addresses key on it, so a context created after a device reset
// looks the addresses up again instead of using the dead context's.
unsigned long long current_context_id();

#define DCC_REQUIRE(cond, code, ...)      \
    do {                                  \
        if (!(cond)) {                    \
            ::dcc::set_error(__VA_ARGS__); \
            return (code);                \
        }                                 \
    } while (0)

// Round-to-nearest FP64 operations that the compiler may not fuse into FMA.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Lexicographic rank of a canonical i<=j<=k triple (distr_cc/distribute_t3.py:51-60).
__host__ __device__ __forceinline__ int64_t ijk_linear(int64_t i, int64_t j, int64_t k, int64_t n) {
    int64_t ni = n - i;
    return (n * (n + 1) * (n + 2) - ni * (ni + 1) * (ni + 2)) / 6 + (j - i) * (2 * n - j - i + 1) / 2 + (k - j);
}

// Lexicographic rank of a<=b<=c among all such virtual triplets (src/rccsdt_q.c:657-665).
__host__ __device__ __forceinline__ int64_t abc_linear(int64_t a, int64_t b, int64_t c, int64_t nv) {
    int64_t rem = nv - a;
    return nv * (nv + 1) * (nv + 2) / 6 - rem * (rem + 1) * (rem + 2) / 6 + (b - a) * (2 * nv - a - b + 1) / 2 +
           (c - b);
}

__host__ __device__ __forceinline__ int64_t binom(int64_t n, int64_t r) {
    if (n < r || n < 0) return 0;
    int64_t v = 1;
    for (int64_t t = 0; t < r; t++) v = v * (n - t) / (t + 1);
    return v;
}

// Full triangular rank of i<=j<=k<=l (src/rccsdtq.c:924-929).
__host__ __device__ __forceinline__ int64_t ijkl_linear(int64_t i, int64_t j, int64_t k, int64_t l, int64_t n) {
    return (binom(n + 3, 4) - binom(n - i + 3, 4)) + (binom(n - i + 2, 3) - binom(n - j + 2, 3)) +
           (binom(n - j + 1, 2) - binom(n - k + 1, 2)) + (l - k);
}

// Ordering case of (i,j,k) relative to its sorted form (src/rccsdt.c:41-73).
__host__ __device__ __forceinline__ int order_case3(int64_t i, int64_t j, int64_t k, int64_t s[3]) {
    if (i <= j && j <= k) { s[0] = i; s[1] = j; s[2] = k; return 0; }
    if (i <= k && k < j) { s[0] = i; s[1] = k; s[2] = j; return 1; }
    if (j < i && i <= k) { s[0] = j; s[1] = i; s[2] = k; return 2; }
    if (k < i && i <= j) { s[0] = k; s[1] = i; s[2] = j; return 3; }
    if (j <= k && k < i) { s[0] = j; s[1] = k; s[2] = i; return 4; }
    s[0] = k; s[1] = j; s[2] = i; return 5;
}

// Output axis m of case c takes input axis kPerm3[c][m].
__host__ __device__ __forceinline__ int perm3(int c, int m) {
    // rows {0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}
    switch (c) {
    case 0: return m;
    case 1: return m == 0 ? 0 : (m == 1 ? 2 : 1);
    case 2: return m == 0 ? 1 : (m == 1 ? 0 : 2);
    case 3: return m == 0 ? 1 : (m == 1 ? 2 : 0);
    case 4: return m == 0 ? 2 : (m == 1 ? 0 : 1);
    default: return 2 - m;
    }
}

inline unsigned ceil_div(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace dcc
