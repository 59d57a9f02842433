// Library-level C ABI: version and per-thread error reporting.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace inc {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: CUDA launch failed: %s", what, cudaGetErrorString(e));
        return INC_E_LAUNCH;
    }
    return INC_OK;
}

}  // namespace inc

extern "C" int32_t inc_version(void) { return 10000 * 0 + 100 * 1 + 0; }

extern "C" const char* inc_last_error_string(void) { return inc::g_err; }
