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
#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

int fill_args(const inc_burgers_desc* d, Args& a);  // burgers_api.cu

namespace cnn {

constexpr int C = 32;   // hidden channels
constexpr int KW = 5;   // kernel width
// Packed weights (inc_burgers_cnn_rollout): w1[co][k], b1[co], w2[ci][co][k],
// b2[co], w3[ci][co][k], b3[co], w4[ci][k], b4.
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + C * KW;
constexpr int OFF_W2 = OFF_B1 + C;
constexpr int OFF_B2 = OFF_W2 + C * C * KW;
constexpr int OFF_W3 = OFF_B2 + C;
constexpr int OFF_B3 = OFF_W3 + C * C * KW;
constexpr int OFF_W4 = OFF_B3 + C;
constexpr int OFF_B4 = OFF_W4 + C * KW;
constexpr int W_FLOATS = OFF_B4 + 1;
constexpr int W_SMEM = (W_FLOATS + 3) / 4 * 4;
static_assert(INC_CNN_WEIGHT_FLOATS == W_FLOATS, "packed weight size");
static_assert(OFF_W2 % 4 == 0 && OFF_W3 % 4 == 0 && OFF_B1 % 4 == 0 && OFF_B2 % 4 == 0 && OFF_B3 % 4 == 0,
              "float4 weight loads");

INC_DEV constexpr int apad(int p) { return p + ((p >> 5) << 2); }
template <int N>
INC_DEV constexpr int row_len() { return (apad(N + 3) + 1 + 3) / 4 * 4; }
template <int N>
INC_DEV constexpr int rows_per_cta() { return N >= 512 ? 1 : 512 / N; }

template <int N>
struct Smem {
    float w[W_SMEM];
    float act[2][rows_per_cta<N>()][C][row_len<N>()];
    WideSmem<1, N> sh[rows_per_cta<N>()];
};

// torch.nn.functional.gelu, approximate='none'
INC_DEV float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }

INC_DEV float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }

// cells 8L-2 .. 8L+9 of one activation row
INC_DEV void load12(float (&a)[12], const float* row, int L) {
    const float4 v0 = lds4(row + apad(8 * L)), v1 = lds4(row + apad(8 * L + 4)), v2 = lds4(row + apad(8 * L + 8));
    a[0] = v0.x; a[1] = v0.y; a[2] = v0.z; a[3] = v0.w;
    a[4] = v1.x; a[5] = v1.y; a[6] = v1.z; a[7] = v1.w;
    a[8] = v2.x; a[9] = v2.y; a[10] = v2.z; a[11] = v2.w;
}

// cells 8L .. 8L+7 of one row, plus the halo copies the row's ends own
template <int N>
INC_DEV void store8(float* row, int L, const float (&v)[8]) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
        *reinterpret_cast<float2*>(row + apad(8 * L + 2 + 2 * i)) = make_float2(v[2 * i], v[2 * i + 1]);
    if (L == 0) {  // x = 0, 1 -> x = N, N + 1
        row[apad(N + 2)] = v[0];
        row[apad(N + 3)] = v[1];
    }
    if (L == N / 8 - 1) {  // x = N - 2, N - 1 -> x = -2, -1
        row[apad(0)] = v[6];
        row[apad(1)] = v[7];
    }
}

template <int N>
INC_DEV void put_cell(float* row, int g, float v) {
    row[apad(g + 2)] = v;
    if (g < 2) row[apad(N + 2 + g)] = v;
    if (g >= N - 2) row[apad(g - N + 2)] = v;
}

// Layer 1: one input channel -> channels 4 cg .. 4 cg + 3, GELU.
template <int N>
INC_DEV void conv_first(const float* w, const float* in, float (*out)[row_len<N>()], int cg, int L) {
    float a[12];
    load12(a, in, L);
    const float4 b = lds4(w + OFF_B1 + 4 * cg);
    const float bias[4] = {b.x, b.y, b.z, b.w};
    float wv[20];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const float4 q = lds4(w + OFF_W1 + 20 * cg + 4 * i);
        wv[4 * i] = q.x; wv[4 * i + 1] = q.y; wv[4 * i + 2] = q.z; wv[4 * i + 3] = q.w;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float acc = bias[c];
#pragma unroll
            for (int k = 0; k < KW; ++k) acc = fmaf(wv[c * KW + k], a[j + k], acc);
            o[j] = gelu(acc);
        }
        store8<N>(out[4 * cg + c], L, o);
    }
}

// Layers 2 and 3: 32 -> channels 4 cg .. 4 cg + 3, GELU.  wt is [ci][co][k].
template <int N>
INC_DEV void conv_mid(const float* wt, const float* bias_p, float (*in)[row_len<N>()],
                      float (*out)[row_len<N>()], int cg, int L) {
    float acc[4][8];
    {
        const float4 b = lds4(bias_p + 4 * cg);
        const float bias[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[c][j] = bias[c];
    }
#pragma unroll 2
    for (int ci = 0; ci < C; ++ci) {
        float a[12], wv[20];
        load12(a, in[ci], L);
        const float* wp = wt + ci * C * KW + 20 * cg;
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            const float4 q = lds4(wp + 4 * i);
            wv[4 * i] = q.x; wv[4 * i + 1] = q.y; wv[4 * i + 2] = q.z; wv[4 * i + 3] = q.w;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < KW; ++k)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[c][j] = fmaf(wv[c * KW + k], a[j + k], acc[c][j]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = gelu(acc[c][j]);
        store8<N>(out[4 * cg + c], L, o);
    }
}

// Layer 4: channels 4 cg .. 4 cg + 3 -> partial sums of the single output
// channel, stored in row cg of `part` (the other buffer); no bias, no GELU.
template <int N>
INC_DEV void conv_last_partial(const float* w4, float (*in)[row_len<N>()], float (*part)[row_len<N>()], int cg,
                               int L) {
    float acc[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j] = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int ci = 4 * cg + c;
        float a[12];
        load12(a, in[ci], L);
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            const float wk = w4[ci * KW + k];
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] = fmaf(wk, a[j + k], acc[j]);
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
        *reinterpret_cast<float2*>(part[cg] + apad(8 * L + 2 + 2 * i)) = make_float2(acc[2 * i], acc[2 * i + 1]);
}

template <int N>
__global__ void __launch_bounds__(512) k_cnn_rollout(Args a, const float* __restrict__ wts,
                                                     float* __restrict__ corr) {
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
    float u[1];
    u[0] = valid ? __ldg(a.u + (int64_t)row * N + g) : 0.f;
    int parity = 0;
    float (*act0)[row_len<N>()] = S.act[0][rl];
    float (*act1)[row_len<N>()] = S.act[1][rl];
    for (int k = 0; k < a.steps; ++k) {
        put_cell<N>(act0[0], g, u[0]);
        __syncthreads();  // also: the weights are in place (first step)
        conv_first<N>(S.w, act0[0], act1, cg, L);
        __syncthreads();
        conv_mid<N>(S.w + OFF_W2, S.w + OFF_B2, act1, act0, cg, L);
        __syncthreads();
        conv_mid<N>(S.w + OFF_W3, S.w + OFF_B3, act0, act1, cg, L);
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
        advance_wide<1, N>(a, cx, u, cx.t + k * cx.dt, S.sh[rl], parity, g);
        if (a.frames && valid) a.frames[at] = u[0];
    }
    if (a.out && valid) a.out[(int64_t)row * N + g] = u[0];
}

template <int N>
int launch(const Args& a, const float* w, float* corr, cudaStream_t st) {
    constexpr int R = rows_per_cta<N>();
    const size_t smem = sizeof(Smem<N>);
    static_assert(sizeof(Smem<N>) <= 227 * 1024, "shared memory");
    cudaFuncSetAttribute(k_cnn_rollout<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_cnn_rollout<N><<<(a.rows + R - 1) / R, R * N, smem, st>>>(a, w, corr);
    return check_launch("burgers_cnn_rollout");
}

}  // namespace cnn
}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

extern "C" int inc_burgers_cnn_rollout(const inc_burgers_desc* d, const float* weights, const float* u0,
                                       const float* t_rows, double t0, int32_t steps, float* frames,
                                       float* corrections, float* u_final, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!weights || !u0 || steps < 0) { set_error("cnn_rollout: bad arguments"); return INC_E_INVALID; }
    if (((reinterpret_cast<uintptr_t>(weights)) & 15u) != 0) {
        set_error("cnn_rollout: weights must be 16-byte aligned");
        return INC_E_INVALID;
    }
    a.u = u0; a.s = nullptr; a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.frames = frames; a.out = u_final;
    cudaStream_t st = as_stream(stream);
    switch (d->n) {
        case 64: return cnn::launch<64>(a, weights, corrections, st);
        case 128: return cnn::launch<128>(a, weights, corrections, st);
        case 256: return cnn::launch<256>(a, weights, corrections, st);
        case 512: return cnn::launch<512>(a, weights, corrections, st);
        default:
            set_error("cnn_rollout: n must be 64, 128, 256 or 512 (got %d)", d->n);
            return INC_E_UNSUPPORTED;
    }
}
