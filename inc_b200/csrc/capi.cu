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

// ---- FP32 FMA throughput probe (measurement utility for the roofline) -------
// Eight independent FMA chains per thread; out[] keeps the result live.
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters) {
    float a0 = threadIdx.x * 1e-3f, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
    const float b = 0.999999f, c = 1e-6f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

extern "C" int inc_bench_fma(float* out, int32_t blocks, int32_t iters, void* stream) {
    if (!out || blocks <= 0 || iters <= 0) {
        inc::set_error("bench_fma: bad arguments");
        return INC_E_INVALID;
    }
    k_fma_peak<<<blocks, 256, 0, inc::as_stream(stream)>>>(out, iters);
    return inc::check_launch("bench_fma");
}
