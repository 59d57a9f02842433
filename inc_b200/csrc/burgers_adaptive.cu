// Adaptive-CFL Burgers stepping (solver_1d.py:148-179) across the whole GPU, and
// its adjoint with the substep sizes held constant.
//
// The reference loops in Python: per substep the global max |u| (a host round
// trip through .item()), dt_local = min(remaining, CFL dx / max|u|), one Euler
// substep, and a stop once ceil(remaining / dt_local) exceeds 1000.  Here one
// cooperative launch (all CTAs resident at once) runs that loop: each CTA
// advances its rows, folds the new max |u| of its rows into one atomic maximum,
// and a grid barrier separates the substeps, so every CTA derives the same
// dt_local from the same maximum.  No host synchronisation, no second launch.
//
// The barrier is a generation counter in the caller's work buffer.  Its waits
// are bounded: a CTA that waits longer than kBarrierSpins polls records an error
// in the control block and leaves the loop, so a kernel never spins forever.
//
// The adjoint (autograd of the reference treats dt_local as a constant: it comes
// from .item()) replays the recorded substeps from u, storing every substep's
// state in caller scratch, then runs the Euler substeps' adjoints in reverse.
#include <algorithm>

#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

// Control block at the start of the work buffer (zeroed by the launching call).
struct AdaptCtl {
    unsigned count;       // CTAs arrived at the current barrier
    unsigned gen;         // barrier generation
    unsigned maxbits[3];  // max |u| of substep i in slot i % 3 (float bit patterns)
    int err;              // 1: a barrier wait gave up; 2: the recorded-substep capacity was reached
    int executed;         // substeps run (the entries of dts)
    int pad[9];
};
static_assert(sizeof(AdaptCtl) == 64, "control block layout");

constexpr long kBarrierSpins = 1L << 22;  // x 256 ns sleep: about a second

struct AdaptArgs {
    Args a;
    AdaptCtl* ctl;
    double* dts;        // [capacity] dt_local of every substep run
    double* tss;        // [capacity] the time offset at the start of each (sum of the earlier dt_local)
    float* t_out;       // [rows] or null
    int* substeps_out;  // the reference's substep count, or null
    float cfl;
    int max_substeps;
    int capacity;
    double dt_total;
};

// All CTAs of the (cooperative) grid reach this point before any leaves it.
// Returns false, with ctl->err set, if this CTA's wait ran out.
INC_DEV bool grid_barrier(AdaptCtl* ctl) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* vgen = &ctl->gen;
        const unsigned g = *vgen;
        __threadfence();  // this CTA's row stores and atomics before its arrival
        if (atomicAdd(&ctl->count, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->count, 0u);
            __threadfence();
            atomicAdd(&ctl->gen, 1u);
            ok = 1;
        } else {
            ok = 0;
            for (long it = 0; it < kBarrierSpins; ++it) {
                if (*vgen != g) { ok = 1; break; }
                __nanosleep(256);
            }
            if (!ok) atomicExch(&ctl->err, 1);
        }
        __threadfence();
        if (ok && *reinterpret_cast<volatile int*>(&ctl->err) == 1) ok = 0;  // another CTA gave up
    }
    __syncthreads();
    return ok != 0;
}

// max(m, |x|) on the bit patterns: a NaN wins, as in torch.max (solver_1d.py:158)
INC_DEV float absmax(float m, float x) {
    return __uint_as_float(max(__float_as_uint(m), __float_as_uint(fabsf(x))));
}

// max |u| of a warp's rows folded into one block maximum, then into *dst
INC_DEV void block_max_to(unsigned* smax, float m, unsigned* dst) {
    const unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
    if ((threadIdx.x & 31) == 0) atomicMax(smax, bits);
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(dst, *smax);
}

template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_adaptive_grid(AdaptArgs ad) {
    __shared__ unsigned smax;
    const Args& a = ad.a;
    AdaptCtl* ctl = ad.ctl;
    const int lane = threadIdx.x & 31;
    const int rpw = 32 / TPR;  // rows per warp
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int g = lane % TPR;
    const int left = (g + TPR - 1) & (TPR - 1), right = (g + 1) & (TPR - 1);
    // max |u| of the input (solver_1d.py:158) into slot 0
    if (threadIdx.x == 0) smax = 0u;
    __syncthreads();
    float m = 0.f;
    for (int r0 = gwarp * rpw; r0 < a.rows; r0 += nwarps * rpw) {
        const int row = r0 + lane / TPR;
        float u[CPT];
        load_row_chunk<CPT>(u, a.out + (int64_t)(row < a.rows ? row : 0) * a.n + g * CPT, row < a.rows);
#pragma unroll
        for (int c = 0; c < CPT; ++c) m = absmax(m, u[c]);
    }
    block_max_to(&smax, m, &ctl->maxbits[0]);
    double target = ad.dt_total, tacc = 0.0;
    int substeps = 0, executed = 0;
    for (int i = 0;; ++i) {
        if (!grid_barrier(ctl)) break;
        const float mx = __uint_as_float(*reinterpret_cast<volatile unsigned*>(&ctl->maxbits[i % 3]));
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->maxbits[(i + 2) % 3] = 0u;  // read by all: barrier i
        if (!(target > 0.0)) break;
        const double allowed = mx > 0.f ? (double)ad.cfl * (double)a.dx / (double)mx : target;
        const double dtl = target < allowed ? target : allowed;
        if (i >= ad.capacity) {  // more substeps than the buffer records: stop, flagged
            if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&ctl->err, 2);
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ad.dts[i] = dtl;
            ad.tss[i] = tacc;
        }
        if (threadIdx.x == 0) smax = 0u;
        __syncthreads();
        m = 0.f;
        for (int r0 = gwarp * rpw; r0 < a.rows; r0 += nwarps * rpw) {
            const int row = r0 + lane / TPR;
            const bool valid = row < a.rows;
            Ctx<CPT> cx;
            make_ctx<CPT, TPR>(a, row, g, valid, cx);
            cx.dt = (float)dtl;
            float u[CPT];
            float* p = a.out + (int64_t)(valid ? row : 0) * a.n + g * CPT;
            load_row_chunk<CPT>(u, p, valid);
            advance<CPT, TPR>(a, cx, u, cx.t + (float)tacc, left, right);
            store_row_chunk<CPT>(p, u, valid);
#pragma unroll
            for (int c = 0; c < CPT; ++c) m = valid ? absmax(m, u[c]) : m;
        }
        block_max_to(&smax, m, &ctl->maxbits[(i + 1) % 3]);
        ++executed;
        tacc += dtl;
        target -= dtl;
        if (target > 0.0 && (int)ceil(target / dtl) > ad.max_substeps) break;  // solver_1d.py:173-176
        ++substeps;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        ctl->executed = executed;
        if (ad.substeps_out) *ad.substeps_out = substeps;
    }
    if (ad.t_out) {
        for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < a.rows; r += gridDim.x * blockDim.x) {
            const float t0 = a.t_rows ? a.t_rows[r] : a.t0;
            ad.t_out[r] = (float)((double)t0 + tacc);
        }
    }
}

// The adjoint of the recorded substeps, one warp per row group: replay storing every
// substep's start state in `states` [executed][rows][n], then the Euler substeps'
// vector-Jacobian products in reverse (advance_bwd with that substep's dt).
template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_adaptive_bwd(Args a, const double* __restrict__ dts,
                                                      const double* __restrict__ tss, int executed,
                                                      float* __restrict__ states) {
    int row, g, left, right;
    bool valid;
    lane_setup<CPT, TPR>(row, g, left, right, valid, a.rows);
    Ctx<CPT> cx;
    make_ctx<CPT, TPR>(a, row, g, valid, cx);
    const float t_row = cx.t;
    const int64_t base = (int64_t)(valid ? row : 0) * a.n + g * CPT;
    const int64_t plane = (int64_t)a.rows * a.n;
    float u[CPT];
    load_row_chunk<CPT>(u, a.u + base, valid);
    for (int k = 0; k < executed; ++k) {  // as k_adaptive_grid's substeps
        store_row_chunk<CPT>(states + k * plane + base, u, valid);
        cx.dt = (float)dts[k];
        advance<CPT, TPR>(a, cx, u, t_row + (float)tss[k], left, right);
    }
    float gu[CPT], gs[CPT];
    load_row_chunk<CPT>(gu, a.g_out + base, valid);
#pragma unroll
    for (int c = 0; c < CPT; ++c) gs[c] = 0.f;
    for (int k = executed - 1; k >= 0; --k) {
        load_row_chunk<CPT>(u, states + k * plane + base, valid);
        cx.dt = (float)dts[k];
        advance_bwd<CPT, TPR>(a, cx, u, gu, gs, t_row + (float)tss[k], g, left, right);
    }
    store_row_chunk<CPT>(a.g_u + base, gu, valid);
    if (a.g_s) store_row_chunk<CPT>(a.g_s + base, gs, valid);
}

}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

namespace inc {
namespace burgers {
int fill_args(const inc_burgers_desc* d, Args& a);
}
}  // namespace inc

namespace {

// Work buffer: the control block, then dt_local and the time offset of every
// substep run (max_substeps + 1 entries each: the reference may run one substep
// past its cap before it stops).
int64_t capacity_of(int max_substeps) { return (int64_t)max_substeps + 1; }
int64_t work_bytes(int max_substeps) {
    return ((int64_t)sizeof(AdaptCtl) + 2 * 8 * capacity_of(max_substeps) + 255) & ~int64_t(255);
}

int cells_per_lane(int n) { return n <= 128 ? 4 : (n <= 256 ? 8 : 16); }

template <int CPT, int TPR>
int launch_adaptive(AdaptArgs& ad, cudaStream_t st) {
    const int threads = 256;
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adaptive_grid<CPT, TPR>, threads, 0);
    if (per_sm <= 0) { set_error("step_adaptive: kernel does not fit on an SM"); return INC_E_LAUNCH; }
    const int64_t groups = (ad.a.rows + (32 / TPR) - 1) / (32 / TPR);
    const int64_t need = (groups + threads / 32 - 1) / (threads / 32);
    const int grid = (int)std::min<int64_t>(need, (int64_t)per_sm * sms);
    void* args[] = {&ad};
    cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_adaptive_grid<CPT, TPR>),
                                                dim3(grid), dim3(threads), args, 0, st);
    if (e != cudaSuccess) { set_error("step_adaptive: %s", cudaGetErrorString(e)); return INC_E_LAUNCH; }
    return INC_OK;
}

template <int CPT, int TPR>
int launch_adaptive_bwd(const Args& a, const double* dts, const double* tss, int executed, float* states,
                        cudaStream_t st) {
    const int rpb = 256 / TPR;
    const int grid = (a.rows + rpb - 1) / rpb;
    k_adaptive_bwd<CPT, TPR><<<grid, 256, 0, st>>>(a, dts, tss, executed, states);
    return check_launch("step_adaptive_bwd");
}

}  // namespace

#define INC_ADAPTIVE_SHAPES(X) X(4, 2) X(4, 4) X(4, 8) X(4, 16) X(4, 32) X(8, 32) X(16, 32)

extern "C" int64_t inc_burgers_step_adaptive_work_size(int32_t max_substeps) {
    return max_substeps > 0 ? work_bytes(max_substeps) : -1;
}

extern "C" int inc_burgers_step_adaptive(const inc_burgers_desc* d, float cfl, int32_t max_substeps, const float* u,
                                         const float* s, const float* t_rows, double t0, float* u_out, float* t_out,
                                         void* work, int32_t* substeps_out, void* stream) {
    AdaptArgs ad;
    int rc = fill_args(d, ad.a);
    if (rc) return rc;
    if (!u || !u_out || !(cfl > 0.f) || max_substeps <= 0) { set_error("step_adaptive: bad arguments"); return INC_E_INVALID; }
    if (!work || (reinterpret_cast<uintptr_t>(work) & 255u)) {
        set_error("step_adaptive: work needs inc_burgers_step_adaptive_work_size(max_substeps) bytes, 256-byte aligned");
        return INC_E_INVALID;
    }
    if (d->scheme != INC_TS_EULER) { set_error("step_adaptive: the reference sub-steps with forward Euler only"); return INC_E_INVALID; }
    const int n = d->n;
    if (!is_pow2(n) || n < 8 || n > 512) { set_error("step_adaptive: n must be a power of two in [8,512]"); return INC_E_UNSUPPORTED; }
    ad.a.s = s; ad.a.t_rows = t_rows; ad.a.t0 = (float)t0; ad.a.out = u_out;
    ad.ctl = static_cast<AdaptCtl*>(work);
    ad.dts = reinterpret_cast<double*>(static_cast<char*>(work) + sizeof(AdaptCtl));
    ad.tss = ad.dts + capacity_of(max_substeps);
    ad.t_out = t_out; ad.substeps_out = substeps_out; ad.cfl = cfl; ad.max_substeps = max_substeps;
    ad.capacity = (int)capacity_of(max_substeps);
    ad.dt_total = (double)d->dt;
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaSuccess;
    if (u != u_out) e = cudaMemcpyAsync(u_out, u, (size_t)d->rows * n * sizeof(float), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(work, 0, sizeof(AdaptCtl), st);
    if (e != cudaSuccess) { set_error("step_adaptive: %s", cudaGetErrorString(e)); return INC_E_LAUNCH; }
    const int cpt = cells_per_lane(n), tpr = n / cpt;
#define INC_A(C, T) \
    if (cpt == C && tpr == T) return launch_adaptive<C, T>(ad, st);
    INC_ADAPTIVE_SHAPES(INC_A)
#undef INC_A
    set_error("step_adaptive: no kernel for n=%d", n);
    return INC_E_UNSUPPORTED;
}

extern "C" int inc_burgers_step_adaptive_bwd(const inc_burgers_desc* d, const float* u, const float* s,
                                             const float* t_rows, double t0, const void* work, int32_t max_substeps,
                                             int32_t executed, const float* g_out, float* g_u, float* g_s,
                                             float* states, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!u || !g_out || !g_u || !work || max_substeps <= 0 || executed < 0 || executed > capacity_of(max_substeps) ||
        (executed > 0 && !states)) {
        set_error("step_adaptive_bwd: bad arguments");
        return INC_E_INVALID;
    }
    if (d->scheme != INC_TS_EULER) { set_error("step_adaptive_bwd: forward Euler only"); return INC_E_INVALID; }
    const int n = d->n;
    if (!is_pow2(n) || n < 8 || n > 512) { set_error("step_adaptive_bwd: n must be a power of two in [8,512]"); return INC_E_UNSUPPORTED; }
    a.u = u; a.s = s; a.t_rows = t_rows; a.t0 = (float)t0; a.g_out = g_out; a.g_u = g_u; a.g_s = g_s;
    const double* dts = reinterpret_cast<const double*>(static_cast<const char*>(work) + sizeof(AdaptCtl));
    const double* tss = dts + capacity_of(max_substeps);
    cudaStream_t st = as_stream(stream);
    const int cpt = cells_per_lane(n), tpr = n / cpt;
#define INC_A(C, T) \
    if (cpt == C && tpr == T) return launch_adaptive_bwd<C, T>(a, dts, tss, executed, states, st);
    INC_ADAPTIVE_SHAPES(INC_A)
#undef INC_A
    set_error("step_adaptive_bwd: no kernel for n=%d", n);
    return INC_E_UNSUPPORTED;
}
