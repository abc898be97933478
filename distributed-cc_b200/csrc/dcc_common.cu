// Error reporting and small shared tables of the dcc_b200 library.
#include <cuda.h>
#include <stdarg.h>
#include <string.h>

#include "dcc_common.cuh"

namespace dcc {

static thread_local char g_err[512];

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void clear_error() { g_err[0] = '\0'; }

int launch_status(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return DCC_ERR_CUDA;
    }
    return DCC_OK;
}

unsigned long long current_context_id() {
    typedef CUresult (*GetCurrentFn)(CUcontext *);
    typedef CUresult (*GetIdFn)(CUcontext, unsigned long long *);
    static GetCurrentFn get_current = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess) ? (GetCurrentFn)p : (GetCurrentFn)nullptr;
    }();
    static GetIdFn get_id = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
                q == cudaDriverEntryPointSuccess) ? (GetIdFn)p : (GetIdFn)nullptr;
    }();
    CUcontext ctx = nullptr;
    if (!get_current || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    unsigned long long id = 0;
    if (get_id && get_id(ctx, &id) == CUDA_SUCCESS) return id + 1;
    return (unsigned long long)(uintptr_t)ctx;
}

int p4_pattern(const char *name, double p[9]) {
    static const struct {
        const char *n;
        double c[9];
    } tab[] = {{"P4_full", {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0}},
               {"P4_444", {2.0, -1.0, -1.0, -1.0, 2.0, -1.0, -1.0, 2.0, -1.0}},
               {"P4_442", {2.0, -1.0, -1.0, -1.0, 2.0, -1.0, -1.0, 1.0, 0.0}},
               {"P4_201", {2.0, -1.0, -1.0, -1.0, 1.0, 0.0, 0.0, 1.0, 0.0}}};
    if (!name) return -1;
    for (auto &t : tab)
        if (strcmp(name, t.n) == 0) {
            memcpy(p, t.c, sizeof(t.c));
            return 0;
        }
    return -1;
}

}  // namespace dcc

extern "C" const char *dcc_last_error(void) { return dcc::g_err; }

extern "C" int dcc_version(void) { return 100; }
