// Device DIIS for the unified T1/T2/T3 vector (distr_cc/diis.py:105-177,
// distr_cc/rccsdt.py:1026-1067): the two vector-length passes of one update.
//
// The vector (slots, xprev) holds the segments one after the other, each starting on a
// multiple of 32 elements (dcc_diis_vector_length), the gaps zero, so every slot is read
// and written in aligned 16-byte pairs whatever the segments' lengths.
//
//   push:    v = concat(scale_s * seg_s);  e = v - xprev;  x_slot = v;  e_slot = e;
//            dots[s] = <e, e_other[s]> (s < nother), dots[nother] = <e, e>
//   combine: xnew = sum_s c_s x_s (in slot order, products rounded before each
//            addition as numpy's `xnew += xi * ci`);  delta = |xnew - xprev|^2;
//            xprev = xnew;  seg_s = xnew / scale_s (the unpack of the caller's amplitudes)
//
// Both are HBM-bound single passes; the small B-matrix solve stays on the host
// (numpy eigh / solve, as the reference).  A slot may also live in pinned host memory
// (the out-of-core slots of distr_cc/diis.py:25-103 kept in host RAM instead of files):
// the kernels then read and write it over the host link through its unified address.  Sums are per-CTA partials reduced in
// CTA order by a second kernel, so results do not depend on scheduling.
#include <stdint.h>

#include "dcc_common.cuh"

namespace dcc {

constexpr int DI_THREADS = 256;
constexpr int DI_MAXS = 16;    // DIIS slots
constexpr int DI_MAXSEG = 4;   // amplitude segments in the vector
constexpr int DI_GRID = 148 * 8;
constexpr int64_t DI_PAD = 32; // every segment starts on a multiple of 32 elements of the vector

// The vector's segments: segment s holds n[s] elements at vector positions [off[s], off[s] + n[s]);
// off[s + 1] - off[s] - n[s] padding elements (zero in every slot) follow it.
struct DiisSegs {
    double *p[DI_MAXSEG];
    double scale[DI_MAXSEG];
    int64_t n[DI_MAXSEG];
    int64_t off[DI_MAXSEG + 1];
    int vec[DI_MAXSEG];  // p[s] is 16-byte aligned (pair loads and stores)
    int nseg;
};

struct DiisPtrs {
    const double *p[DI_MAXS];
    double c[DI_MAXS];
    int n;
};

// Segment of vector position j (even): base pointer, length, scale and the local index.
__device__ __forceinline__ int seg_at(const DiisSegs &g, int64_t j, int64_t &l) {
    int s = 0;
#pragma unroll
    for (int q = 1; q < DI_MAXSEG; q++)
        if (q < g.nseg && j >= g.off[q]) s = q;
    l = j - g.off[s];
    return s;
}

// The two segment elements at local index l, l + 1 (zero past the segment's end).
__device__ __forceinline__ double2 seg_load(const DiisSegs &g, int s, int64_t l) {
    const double *p = g.p[s];
    const int64_t n = g.n[s];
    if (g.vec[s] && l + 1 < n) return *reinterpret_cast<const double2 *>(p + l);
    return make_double2(l < n ? p[l] : 0.0, l + 1 < n ? p[l + 1] : 0.0);
}

__device__ __forceinline__ void seg_store(const DiisSegs &g, int s, int64_t l, double2 v) {
    double *p = g.p[s];
    const int64_t n = g.n[s];
    if (g.vec[s] && l + 1 < n) {
        *reinterpret_cast<double2 *>(p + l) = v;
        return;
    }
    if (l < n) p[l] = v.x;
    if (l + 1 < n) p[l + 1] = v.y;
}

__device__ __forceinline__ double2 ld2(const double *p, int64_t j) { return *reinterpret_cast<const double2 *>(p + j); }
__device__ __forceinline__ void st2(double *p, int64_t j, double2 v) { *reinterpret_cast<double2 *>(p + j) = v; }

// Block-wide sums of v[0..N) into partial[blockIdx.x * stride + s] for s < n,
// and of `last` into partial[blockIdx.x * stride + n] (thread 0 writes).
template <int N>
__device__ __forceinline__ void block_sums(const double (&v)[N], double last, int n, double *partial, int stride) {
    __shared__ double red[DI_THREADS / 32][N + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int s = 0; s <= N; s++) {
        double x = s < N ? v[s] : last;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[w][s] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s <= n; s++) {
            double x = 0.0;
            for (int q = 0; q < DI_THREADS / 32; q++) x += red[q][s < n ? s : N];
            partial[(int64_t)blockIdx.x * stride + s] = x;
        }
    }
}

// One pass over the vector in element pairs (16-byte loads and stores of every slot).
__global__ void __launch_bounds__(DI_THREADS) k_diis_push(DiisSegs x, double *xprev, double *xslot, double *eslot,
                                                          DiisPtrs eo, double *partial) {
    double acc[DI_MAXS];
    double ee = 0.0;
#pragma unroll
    for (int s = 0; s < DI_MAXS; s++) acc[s] = 0.0;
    const int64_t npair = x.off[x.nseg] / 2, stride = (int64_t)gridDim.x * DI_THREADS;
    for (int64_t q = (int64_t)blockIdx.x * DI_THREADS + threadIdx.x; q < npair; q += stride) {
        const int64_t j = 2 * q;
        int64_t l;
        const int s = seg_at(x, j, l);
        const double2 a = seg_load(x, s, l), xp = ld2(xprev, j);
        const double sc = x.scale[s];
        const double2 v = make_double2(dmul(sc, a.x), dmul(sc, a.y));
        const double2 e = make_double2(dsub(v.x, xp.x), dsub(v.y, xp.y));
        st2(xslot, j, v);
        st2(eslot, j, e);
#pragma unroll
        for (int t = 0; t < DI_MAXS; t++)
            if (t < eo.n) {
                const double2 o = ld2(eo.p[t], j);
                acc[t] = fma(e.y, o.y, fma(e.x, o.x, acc[t]));
            }
        ee = fma(e.y, e.y, fma(e.x, e.x, ee));
    }
    block_sums(acc, ee, eo.n, partial, DI_MAXS + 1);  // <e, e_s> then <e, e>
}

__global__ void __launch_bounds__(DI_THREADS) k_diis_combine(DiisPtrs xs, double *xprev, DiisSegs out,
                                                             double *partial) {
    double dd = 0.0;
    const int64_t npair = out.off[out.nseg] / 2, stride = (int64_t)gridDim.x * DI_THREADS;
    for (int64_t q = (int64_t)blockIdx.x * DI_THREADS + threadIdx.x; q < npair; q += stride) {
        const int64_t j = 2 * q;
        double2 xi[DI_MAXS];
#pragma unroll
        for (int t = 0; t < DI_MAXS; t++)
            if (t < xs.n) xi[t] = ld2(xs.p[t], j);
        const double2 xp = ld2(xprev, j);
        double vx = 0.0, vy = 0.0;
#pragma unroll
        for (int t = 0; t < DI_MAXS; t++)
            if (t < xs.n) {
                vx = dadd(vx, dmul(xi[t].x, xs.c[t]));
                vy = dadd(vy, dmul(xi[t].y, xs.c[t]));
            }
        const double dx = dsub(vx, xp.x), dy = dsub(vy, xp.y);
        dd = fma(dy, dy, fma(dx, dx, dd));
        st2(xprev, j, make_double2(vx, vy));
        int64_t l;
        const int s = seg_at(out, j, l);
        const double sc = out.scale[s];
        seg_store(out, s, l, sc == 1.0 ? make_double2(vx, vy) : make_double2(__ddiv_rn(vx, sc), __ddiv_rn(vy, sc)));
    }
    const double none[1] = {0.0};
    block_sums(none, dd, 0, partial, DI_MAXS + 1);
}

// out[s] = sum over CTAs of partial[cta][s], CTAs in order.
__global__ void k_diis_finish(const double *partial, int nblk, int nsum, double *out) {
    const int s = threadIdx.x;
    if (s >= nsum) return;
    double x = 0.0;
    for (int b = 0; b < nblk; b++) x += partial[(int64_t)b * (DI_MAXS + 1) + s];
    out[s] = x;
}

static int make_segs(DiisSegs &g, double *const *seg, const int64_t *seg_n, const double *scale, int nseg,
                     int64_t &n) {
    DCC_REQUIRE(nseg >= 1 && nseg <= DI_MAXSEG, DCC_ERR_SHAPE, "1..%d segments", DI_MAXSEG);
    DCC_REQUIRE(seg && seg_n && scale, DCC_ERR_NULL, "NULL segment table");
    g = DiisSegs{};
    g.nseg = nseg;
    n = 0;
    for (int s = 0; s < nseg; s++) {
        DCC_REQUIRE(seg_n[s] >= 0 && (seg[s] || seg_n[s] == 0), DCC_ERR_NULL, "segment %d is NULL", s);
        DCC_REQUIRE(scale[s] != 0.0, DCC_ERR_SHAPE, "segment %d has scale 0", s);
        g.p[s] = seg[s];
        g.scale[s] = scale[s];
        g.n[s] = seg_n[s];
        g.off[s] = n;
        g.vec[s] = ((uintptr_t)seg[s] & 15) == 0;
        n += (seg_n[s] + DI_PAD - 1) / DI_PAD * DI_PAD;
    }
    for (int s = nseg; s <= DI_MAXSEG; s++) g.off[s] = n;
    return DCC_OK;
}

}  // namespace dcc

using namespace dcc;

extern "C" size_t dcc_diis_workspace_bytes(void) { return (size_t)DI_GRID * (DI_MAXS + 1) * sizeof(double); }

extern "C" int64_t dcc_diis_vector_length(const int64_t *seg_n, int nseg, int64_t *seg_off) {
    clear_error();
    if (!seg_n || nseg < 1 || nseg > DI_MAXSEG) {
        set_error("1..%d segments", DI_MAXSEG);
        return -1;
    }
    int64_t n = 0;
    for (int s = 0; s < nseg; s++) {
        if (seg_n[s] < 0) {
            set_error("segment %d has a negative length", s);
            return -1;
        }
        if (seg_off) seg_off[s] = n;
        n += (seg_n[s] + DI_PAD - 1) / DI_PAD * DI_PAD;
    }
    return n;
}

static bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// A slot pointer the kernels can dereference: device, managed or pinned (page-locked) host
// memory.  Pageable host memory is refused before any launch.
static int check_slot(const void *p, const char *what, int s) {
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("%s %d: cudaPointerGetAttributes: %s", what, s, cudaGetErrorString(e));
        return DCC_ERR_CUDA;
    }
    DCC_REQUIRE(a.type != cudaMemoryTypeUnregistered, DCC_ERR_UNSUPPORTED,
                "%s %d is pageable host memory; slots must be device or pinned host memory", what, s);
    DCC_REQUIRE(a.type != cudaMemoryTypeHost || a.devicePointer == p, DCC_ERR_UNSUPPORTED,
                "%s %d: pinned host memory whose device address differs from its host address", what, s);
    return DCC_OK;
}

extern "C" int dcc_diis_push(double *const *seg, const int64_t *seg_n, const double *seg_scale, int nseg,
                             double *xprev, double *x_slot, double *e_slot, const double *const *e_other, int nother,
                             double *dots, void *workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    DiisSegs g;
    int64_t n = 0;
    int rc = make_segs(g, seg, seg_n, seg_scale, nseg, n);
    if (rc) return rc;
    DCC_REQUIRE(nother >= 0 && nother < DI_MAXS, DCC_ERR_SHAPE, "0..%d other slots", DI_MAXS - 1);
    DCC_REQUIRE(xprev && x_slot && e_slot && dots && workspace && (nother == 0 || e_other), DCC_ERR_NULL,
                "NULL buffer");
    DCC_REQUIRE(workspace_bytes >= dcc_diis_workspace_bytes(), DCC_ERR_SHAPE, "workspace too small");
    DiisPtrs eo{};
    eo.n = nother;
    for (int s = 0; s < nother; s++) {
        DCC_REQUIRE(e_other[s], DCC_ERR_NULL, "other slot %d is NULL", s);
        if ((rc = check_slot(e_other[s], "other error slot", s))) return rc;
        eo.p[s] = e_other[s];
    }
    if ((rc = check_slot(x_slot, "x slot", 0)) || (rc = check_slot(e_slot, "error slot", 0))) return rc;
    DCC_REQUIRE(aligned16(xprev) && aligned16(x_slot) && aligned16(e_slot), DCC_ERR_UNSUPPORTED,
                "xprev and the slots must be 16-byte aligned");
    for (int s = 0; s < nother; s++)
        DCC_REQUIRE(aligned16(e_other[s]), DCC_ERR_UNSUPPORTED, "other slot %d is not 16-byte aligned", s);
    cudaStream_t st = as_stream(stream);
    double *partial = (double *)workspace;
    k_diis_push<<<DI_GRID, DI_THREADS, 0, st>>>(g, xprev, x_slot, e_slot, eo, partial);
    k_diis_finish<<<1, 32, 0, st>>>(partial, DI_GRID, nother + 1, dots);
    return launch_status("diis_push");
}

extern "C" int dcc_diis_combine(const double *const *xs, const double *coef, int nd, double *xprev,
                                double *const *out_seg, const int64_t *seg_n, const double *seg_scale, int nseg,
                                double *delta, void *workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    DiisSegs g;
    int64_t n = 0;
    int rc = make_segs(g, out_seg, seg_n, seg_scale, nseg, n);
    if (rc) return rc;
    DCC_REQUIRE(nd >= 1 && nd <= DI_MAXS, DCC_ERR_SHAPE, "1..%d slots", DI_MAXS);
    DCC_REQUIRE(xs && coef && xprev && delta && workspace, DCC_ERR_NULL, "NULL buffer");
    DCC_REQUIRE(workspace_bytes >= dcc_diis_workspace_bytes(), DCC_ERR_SHAPE, "workspace too small");
    DiisPtrs p{};
    p.n = nd;
    for (int s = 0; s < nd; s++) {
        DCC_REQUIRE(xs[s], DCC_ERR_NULL, "slot %d is NULL", s);
        if ((rc = check_slot(xs[s], "x slot", s))) return rc;
        DCC_REQUIRE(aligned16(xs[s]), DCC_ERR_UNSUPPORTED, "slot %d is not 16-byte aligned", s);
        p.p[s] = xs[s];
        p.c[s] = coef[s];
    }
    DCC_REQUIRE(aligned16(xprev), DCC_ERR_UNSUPPORTED, "xprev must be 16-byte aligned");
    cudaStream_t st = as_stream(stream);
    double *partial = (double *)workspace;
    k_diis_combine<<<DI_GRID, DI_THREADS, 0, st>>>(p, xprev, g, partial);
    k_diis_finish<<<1, 32, 0, st>>>(partial, DI_GRID, 1, delta);
    return launch_status("diis_combine");
}
