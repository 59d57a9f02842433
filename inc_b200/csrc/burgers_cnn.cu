// Hybrid Burgers rollout with a periodic CNN corrector evaluated inside the
// kernel: per step s = CNN(u), then u = step(u, s) -- the per-step loop of
// trainer/trainer_1d.py:154-183 (simulate_rollout with correction "INC") for
// the convolutional corrector, forward only (evaluation rollouts).
//
// The network is the benchmark's PeriodicCNN1D: four Conv1d layers
// 1 -> 32 -> 32 -> 32 -> 1, kernel 5, circular padding 2, exact (erf) GELU
// between layers.  torch's Conv1d is a cross-correlation:
//   out[co][x] = b[co] + sum_ci sum_k W[co][ci][k] in[ci][(x + k - 2) mod N].
//
// Layout: one CTA holds R = max(1, 512 / N) rows, N threads per row.  The
// solver stage keeps one cell per thread (the wide-row layout of
// burgers_kernels.cuh, stages through a shared row).  In the convolution
// stages thread g computes 4 output channels (group g / (N/8)) x 8 contiguous
// cells (8 * (g % (N/8)) ...): per input channel it reads 12 activations as
// three float4 and 20 weights as five broadcast float4, then does 160 FMAs.
// Activations live in shared memory, two buffers of [R][32][row], cell x of a
// row at apad(x + 2) with x in [-2, N + 2) (the circular halo is stored); the
// 4-float pad per 32 makes the float4 reads conflict-free.  All weights
// (42.6 KB) sit in shared memory for the whole launch.
#include "burgers_cnn.cuh"

namespace inc {
namespace burgers {
namespace cnn {

template <int N>
__global__ void __launch_bounds__(512) k_cnn_rollout(Args a, const float* __restrict__ wts,
                                                     float* __restrict__ corr, float* __restrict__ acts) {
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem<N>& S = *reinterpret_cast<Smem<N>*>(smraw);
    constexpr int R = rows_per_cta<N>();
    constexpr int LPG = N / 8;  // lanes per channel group
    const int rl = threadIdx.x / N;
    const int g = threadIdx.x % N;
    const int cg = g / LPG;
    const int L = g % LPG;
    const int row = blockIdx.x * R + rl;
    const bool valid = row < a.rows;
    for (int i = threadIdx.x; i < W_FLOATS; i += blockDim.x) S.w[i] = __ldg(wts + i);
    Ctx<1> cx;
    make_ctx<1, N>(a, valid ? row : 0, g, true, cx);
    cx.has_s = true;
    float u[1], cmp[1] = {0.f};  // cmp: compensation carried from step to step (see advance)
    u[0] = valid ? __ldg(a.u + (int64_t)row * N + g) : 0.f;
    int parity = 0;
    float (*act0)[row_len<N>()] = S.act[0][rl];
    float (*act1)[row_len<N>()] = S.act[1][rl];
    const int nseg = a.ckpt_every > 0 ? (a.steps + a.ckpt_every - 1) / a.ckpt_every : 0;
    for (int k = 0; k < a.steps; ++k) {
        if (a.ckpts && valid && k % a.ckpt_every == 0)
            a.ckpts[((int64_t)row * nseg + k / a.ckpt_every) * N + g] = u[0];
        put_cell<N>(act0[0], g, u[0]);
        __syncthreads();  // also: the weights are in place (first step)
        conv_first<N>(S.w, act0[0], act1, cg, L);
        __syncthreads();
        if (acts) {  // training: the hidden layers' pre-activations recorded for the backward
            float acc[4][8];
            conv_mid_acc<N>(S.w + OFF_W2, S.w + OFF_B2, act1, acc, cg, L);
            if (valid) put_acts(acts, row, a.steps, k, 0, acc, cg, L, N);
            store_tile<N, true>(act0, acc, cg, L);
            __syncthreads();
            conv_mid_acc<N>(S.w + OFF_W3, S.w + OFF_B3, act0, acc, cg, L);
            if (valid) put_acts(acts, row, a.steps, k, 1, acc, cg, L, N);
            store_tile<N, true>(act1, acc, cg, L);
        } else {
            conv_mid<N>(S.w + OFF_W2, S.w + OFF_B2, act1, act0, cg, L);
            __syncthreads();
            conv_mid<N>(S.w + OFF_W3, S.w + OFF_B3, act0, act1, cg, L);
        }
        __syncthreads();
        conv_last_partial<N>(S.w + OFF_W4, act1, act0, cg, L);
        __syncthreads();
        float s = S.w[OFF_B4];
#pragma unroll
        for (int q = 0; q < 8; ++q) s += act0[q][apad(g + 2)];
        cx.s[0] = s;
        const int64_t at = ((int64_t)row * a.steps + k) * N + g;
        if (corr && valid) corr[at] = s;
        // the stage's first barrier also orders these reads of act0 before the next step's writes
        advance_wide<1, N>(a, cx, u, cmp, cx.t + k * cx.dt, S.sh[rl], parity, g);
        if (a.frames && valid) a.frames[at] = u[0];
    }
    if (a.out && valid) a.out[(int64_t)row * N + g] = u[0];
}

template <int N>
int launch(const Args& a, const float* w, float* corr, float* acts, cudaStream_t st) {
    constexpr int R = rows_per_cta<N>();
    const size_t smem = sizeof(Smem<N>);
    static_assert(sizeof(Smem<N>) <= 227 * 1024, "shared memory");
    cudaFuncSetAttribute(k_cnn_rollout<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cnn_rollout<N><<<(a.rows + R - 1) / R, R * N, smem, st>>>(a, w, corr, acts);
    return check_launch("burgers_cnn_rollout");
}

}  // namespace cnn
}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

static int cnn_rollout(const inc_burgers_desc* d, const float* weights, const float* u0, const float* t_rows,
                       double t0, int32_t steps, float* frames, float* corrections, float* u_final,
                       int32_t ckpt_every, float* ckpts, float* acts, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!weights || !u0 || steps < 0) { set_error("cnn_rollout: bad arguments"); return INC_E_INVALID; }
    if (ckpts && ckpt_every <= 0) { set_error("cnn_rollout: ckpt_every must be positive with ckpts"); return INC_E_INVALID; }
    a.ckpt_every = ckpt_every;
    a.ckpts = ckpts;
    if (((reinterpret_cast<uintptr_t>(weights)) & 15u) != 0) {
        set_error("cnn_rollout: weights must be 16-byte aligned");
        return INC_E_INVALID;
    }
    if (acts && ((reinterpret_cast<uintptr_t>(acts)) & 15u) != 0) {
        set_error("cnn_rollout: acts must be 16-byte aligned");
        return INC_E_INVALID;
    }
    a.u = u0; a.s = nullptr; a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.frames = frames; a.out = u_final;
    cudaStream_t st = as_stream(stream);
    switch (d->n) {
        case 64: return cnn::launch<64>(a, weights, corrections, acts, st);
        case 128: return cnn::launch<128>(a, weights, corrections, acts, st);
        case 256: return cnn::launch<256>(a, weights, corrections, acts, st);
        case 512: return cnn::launch<512>(a, weights, corrections, acts, st);
        default:
            set_error("cnn_rollout: n must be 64, 128, 256 or 512 (got %d)", d->n);
            return INC_E_UNSUPPORTED;
    }
}

extern "C" int inc_burgers_cnn_rollout(const inc_burgers_desc* d, const float* weights, const float* u0,
                                       const float* t_rows, double t0, int32_t steps, float* frames,
                                       float* corrections, float* u_final, int32_t ckpt_every, float* ckpts,
                                       void* stream) {
    return cnn_rollout(d, weights, u0, t_rows, t0, steps, frames, corrections, u_final, ckpt_every, ckpts, nullptr,
                       stream);
}

extern "C" int inc_burgers_cnn_rollout_acts(const inc_burgers_desc* d, const float* weights, const float* u0,
                                            const float* t_rows, double t0, int32_t steps, float* frames,
                                            float* corrections, float* u_final, int32_t ckpt_every, float* ckpts,
                                            float* acts, void* stream) {
    if (!acts) { set_error("cnn_rollout_acts: acts must not be NULL"); return INC_E_INVALID; }
    return cnn_rollout(d, weights, u0, t_rows, t0, steps, frames, corrections, u_final, ckpt_every, ckpts, acts,
                       stream);
}
