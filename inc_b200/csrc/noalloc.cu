// Burgers rollout forward + backward that needs no device allocation.
//
// inc_burgers_rollout + inc_burgers_rollout_bwd want the caller to allocate the
// checkpoint buffer that carries states from the forward launch to the backward
// one.  Some callers cannot allocate device memory while they run this op: a
// host framework that owns all device memory and forbids allocation inside a
// foreign-function call, or an application running within a fixed memory
// budget.  This entry point keeps the checkpoints in a fixed array compiled
// into the library instead, so the caller passes only its inputs and outputs.
#include <mutex>

#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {
int fill_args(const inc_burgers_desc* d, Args& a);
int dispatch(Kind kind, const Args& a, int cpt, cudaStream_t st);
}  // namespace burgers
}  // namespace inc

namespace {

// The checkpoint area: INC_NOALLOC_CKPT_FLOATS floats (8 MiB).  Every GPU that
// loads the library holds one copy until the process exits.
static __device__ __align__(256) float g_ckpt_area[INC_NOALLOC_CKPT_FLOATS];

constexpr int kMaxDevices = 64;
float* g_area_ptr[kMaxDevices] = {};
std::mutex g_area_mu;

// Device address of g_ckpt_area in the current context.  In host code the
// array's name is only a host-side stand-in, so the kernels must be given this
// address.  It is looked up again on every call whose stream is not capturing
// (the context may have been reset, or be another one than last time, and the
// module then lives at another address); a call on a capturing stream uses the
// address the last uncapturing call on this device found.
int area_on_current_device(cudaStream_t st, float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        inc::set_error("rollout_grad_noalloc: cudaGetDevice failed: %s", cudaGetErrorString(e));
        return INC_E_LAUNCH;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        inc::set_error("rollout_grad_noalloc: device %d out of range", dev);
        return INC_E_UNSUPPORTED;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        cudaGetLastError();  // e.g. the legacy stream while another stream captures
        cap = cudaStreamCaptureStatusActive;
    }
    std::lock_guard<std::mutex> lock(g_area_mu);
    if (cap == cudaStreamCaptureStatusNone) {
        float* p = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_ckpt_area);
        if (e != cudaSuccess || p == nullptr) {
            inc::set_error("rollout_grad_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return INC_E_LAUNCH;
        }
        g_area_ptr[dev] = p;
    } else if (!g_area_ptr[dev]) {
        inc::set_error("rollout_grad_noalloc: the first call on device %d must come before stream capture", dev);
        return INC_E_INVALID;
    }
    *out = g_area_ptr[dev];
    return INC_OK;
}

}  // namespace

using namespace inc;
using namespace inc::burgers;

extern "C" int inc_burgers_rollout_grad_noalloc(const inc_burgers_desc* d, const float* u0, const float* s,
                                                const float* t_rows, double t0, int32_t steps, int32_t ckpt_every,
                                                const float* g_frames, const float* g_final, float* frames,
                                                float* u_final, float* g_u0, float* g_s, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!u0 || !g_u0 || steps <= 0 || ckpt_every <= 0) {
        set_error("rollout_grad_noalloc: need u0, g_u0, steps > 0 and ckpt_every > 0");
        return INC_E_INVALID;
    }
    const int64_t nseg = (steps + ckpt_every - 1) / ckpt_every;
    const int64_t need = (int64_t)d->rows * nseg * d->n;
    if (need > INC_NOALLOC_CKPT_FLOATS) {
        set_error("rollout_grad_noalloc: rows * ceil(steps / ckpt_every) * n = %lld floats exceeds the built-in "
                  "checkpoint area of %d floats; raise ckpt_every or split the batch",
                  (long long)need, INC_NOALLOC_CKPT_FLOATS);
        return INC_E_INVALID;
    }
    cudaStream_t st = as_stream(stream);
    float* area = nullptr;
    rc = area_on_current_device(st, &area);
    if (rc) return rc;
    // forward: frames / final state for the caller, checkpoints into the area
    a.u = u0; a.s = s; a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.frames = frames; a.out = u_final;
    a.ckpt_every = ckpt_every; a.ckpts = area;
    rc = dispatch(Kind::Rollout, a, d->cells_per_thread, st);
    if (rc) return rc;
    // backward: every checkpoint it reads was written by the launch above
    Args b;
    fill_args(d, b);
    b.s = s; b.t_rows = t_rows; b.t0 = (float)t0; b.steps = steps; b.ckpt_every = ckpt_every; b.ckpts = area;
    b.g_frames = g_frames; b.g_final = g_final; b.g_u = g_u0; b.g_s = g_s;
    return dispatch(Kind::RolloutBwd, b, d->cells_per_thread, st);
}
