// Periodic CNN corrector (PeriodicCNN1D: Conv1d 1 -> 32 -> 32 -> 32 -> 1,
// kernel 5, circular padding 2, erf GELU between layers) evaluated from shared
// memory inside the Burgers rollout kernels: constants, the packed weight
// layout, the activation row layout and the convolution stages shared by the
// forward rollout (burgers_cnn.cu) and its backward (burgers_cnn_bwd.cu).
// torch's Conv1d is a cross-correlation:
//   out[co][x] = b[co] + sum_ci sum_k W[co][ci][k] in[ci][(x + k - 2) mod N].
#pragma once
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

// Layer 1, accumulation: acc[c][j] = pre-activation of channel 4 cg + c at cell
// 8 L + j, from one input row.
template <int N>
INC_DEV void conv_first_acc(const float* w, const float* in, float (&acc)[4][8], int cg, int L) {
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
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float acc1 = bias[c];
#pragma unroll
            for (int k = 0; k < KW; ++k) acc1 = fmaf(wv[c * KW + k], a[j + k], acc1);
            acc[c][j] = acc1;
        }
}

// Layers 2 and 3, accumulation: acc[c][j] = pre-activation of channel 4 cg + c
// at cell 8 L + j.  wt is [ci][co][k].
template <int N>
INC_DEV void conv_mid_acc(const float* wt, const float* bias_p, float (*in)[row_len<N>()], float (&acc)[4][8],
                          int cg, int L) {
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
}

// a 4-channel x 8-cell tile into rows 4 cg .. 4 cg + 3 of `out` (GELU applied or not)
template <int N, bool GELU_OUT>
INC_DEV void store_tile(float (*out)[row_len<N>()], const float (&acc)[4][8], int cg, int L) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = GELU_OUT ? gelu(acc[c][j]) : acc[c][j];
        store8<N>(out[4 * cg + c], L, o);
    }
}

// Layer 1: one input channel -> channels 4 cg .. 4 cg + 3, GELU (or, with
// GELU_OUT = false, the pre-activations).
template <int N, bool GELU_OUT = true>
INC_DEV void conv_first(const float* w, const float* in, float (*out)[row_len<N>()], int cg, int L) {
    float acc[4][8];
    conv_first_acc<N>(w, in, acc, cg, L);
    store_tile<N, GELU_OUT>(out, acc, cg, L);
}

// Layers 2 and 3: 32 -> channels 4 cg .. 4 cg + 3, GELU (or the
// pre-activations).
template <int N, bool GELU_OUT = true>
INC_DEV void conv_mid(const float* wt, const float* bias_p, float (*in)[row_len<N>()],
                      float (*out)[row_len<N>()], int cg, int L) {
    float acc[4][8];
    conv_mid_acc<N>(wt, bias_p, in, acc, cg, L);
    store_tile<N, GELU_OUT>(out, acc, cg, L);
}

// The hidden layers' pre-activations of every step, recorded by the forward for
// its backward: acts[row][step][layer: 0 = z2, 1 = z3][channel][cell].
INC_DEV float* acts_tile(float* acts, int64_t row, int steps, int k, int layer, int ch, int n) {
    return acts + ((((row * steps + k) * 2 + layer) * C + ch) * (int64_t)n);
}

// this thread's 4-channel x 8-cell tile to / from the record (two float4 a channel)
INC_DEV void put_acts(float* acts, int64_t row, int steps, int k, int layer, const float (&acc)[4][8], int cg,
                      int L, int n) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float4* p = reinterpret_cast<float4*>(acts_tile(acts, row, steps, k, layer, 4 * cg + c, n) + 8 * L);
        p[0] = make_float4(acc[c][0], acc[c][1], acc[c][2], acc[c][3]);
        p[1] = make_float4(acc[c][4], acc[c][5], acc[c][6], acc[c][7]);
    }
}
INC_DEV void get_acts(const float* __restrict__ acts, int64_t row, int steps, int k, int layer, float (&acc)[4][8],
                      int cg, int L, int n) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float4* p = reinterpret_cast<const float4*>(
            acts_tile(const_cast<float*>(acts), row, steps, k, layer, 4 * cg + c, n) + 8 * L);
        const float4 v0 = __ldg(p), v1 = __ldg(p + 1);
        acc[c][0] = v0.x; acc[c][1] = v0.y; acc[c][2] = v0.z; acc[c][3] = v0.w;
        acc[c][4] = v1.x; acc[c][5] = v1.y; acc[c][6] = v1.z; acc[c][7] = v1.w;
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

}  // namespace cnn
}  // namespace burgers
}  // namespace inc
