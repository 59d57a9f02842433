// y = gelu(h + bias[c]) over [rows][n] activations whose row r is channel
// r % channels (the FNO corrector's projection layer, models/models_1d/fno.py:
// 101-102: fc1 then gelu), and its backward: dh = dy * gelu'(h + bias[c]) with
// the per-row sums of dh for the bias gradient.  GELU is the exact (erf) form of
// torch.nn.functional.gelu:
//   gelu(z)  = z Phi(z),            Phi(z) = (1 + erf(z / sqrt 2)) / 2,
//   gelu'(z) = Phi(z) + z phi(z),   phi(z) = exp(-z^2 / 2) / sqrt(2 pi).
// One warp per row, float4 loads and stores (n a multiple of 4 keeps every row
// 16-byte aligned); the row sums make the bias gradient a fixed-order
// reduction.
#include "common.cuh"

namespace inc {
namespace act {

constexpr int BG_BLOCK = 256;
constexpr float kInvSqrt2 = 0.70710678118654752f;
constexpr float kInvSqrt2Pi = 0.39894228040143268f;

INC_DEV float gelu_phi(float z) { return 0.5f * (1.f + erff(z * kInvSqrt2)); }

__global__ void __launch_bounds__(BG_BLOCK) k_bias_gelu(const float4* __restrict__ h, const float* __restrict__ bias,
                                                       float4* __restrict__ y, int rows, int n4, int channels) {
    const int warps = gridDim.x * (BG_BLOCK / 32);
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (BG_BLOCK / 32) + (threadIdx.x >> 5); r < rows; r += warps) {
        const float b = __ldg(bias + r % channels);
        const float4* hr = h + (int64_t)r * n4;
        float4* yr = y + (int64_t)r * n4;
        for (int i = lane; i < n4; i += 32) {
            const float4 v = __ldg(hr + i);
            float4 o;
            o.x = (v.x + b) * gelu_phi(v.x + b);
            o.y = (v.y + b) * gelu_phi(v.y + b);
            o.z = (v.z + b) * gelu_phi(v.z + b);
            o.w = (v.w + b) * gelu_phi(v.w + b);
            yr[i] = o;
        }
    }
}

INC_DEV float gelu_grad(float z) { return gelu_phi(z) + z * kInvSqrt2Pi * expf(-0.5f * z * z); }

__global__ void __launch_bounds__(BG_BLOCK) k_bias_gelu_bwd(const float4* __restrict__ dy,
                                                           const float4* __restrict__ h,
                                                           const float* __restrict__ bias, float4* __restrict__ dh,
                                                           float* __restrict__ row_sums, int rows, int n4,
                                                           int channels) {
    const int warps = gridDim.x * (BG_BLOCK / 32);
    const int lane = threadIdx.x & 31;
    for (int r = blockIdx.x * (BG_BLOCK / 32) + (threadIdx.x >> 5); r < rows; r += warps) {
        const float b = __ldg(bias + r % channels);
        const float4* hr = h + (int64_t)r * n4;
        const float4* gr = dy + (int64_t)r * n4;
        float4* dr = dh + (int64_t)r * n4;
        float s = 0.f;
        for (int i = lane; i < n4; i += 32) {
            const float4 v = __ldg(hr + i), g = __ldg(gr + i);
            float4 o;
            o.x = g.x * gelu_grad(v.x + b);
            o.y = g.y * gelu_grad(v.y + b);
            o.z = g.z * gelu_grad(v.z + b);
            o.w = g.w * gelu_grad(v.w + b);
            dr[i] = o;
            s += (o.x + o.y) + (o.z + o.w);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) row_sums[r] = s;
    }
}

int grid_for(int rows) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int want = (rows + BG_BLOCK / 32 - 1) / (BG_BLOCK / 32);
    const int cap = sms * 8;
    return want < cap ? want : cap;
}

int check_shape(const void* a, const void* b, const void* c, int32_t rows, int32_t n, int32_t channels) {
    if (!a || !b || !c || rows <= 0 || channels <= 0 || rows % channels != 0) {
        set_error("bias_gelu: bad arguments");
        return INC_E_INVALID;
    }
    if (n <= 0 || n % 4 != 0) {
        set_error("bias_gelu: n must be a positive multiple of 4 (got %d)", n);
        return INC_E_UNSUPPORTED;
    }
    return INC_OK;
}

}  // namespace act
}  // namespace inc

using namespace inc;

extern "C" int inc_bias_gelu(const float* h, const float* bias, float* y, int32_t rows, int32_t n, int32_t channels,
                             void* stream) {
    int rc = act::check_shape(h, bias, y, rows, n, channels);
    if (rc) return rc;
    act::k_bias_gelu<<<act::grid_for(rows), act::BG_BLOCK, 0, as_stream(stream)>>>(
        reinterpret_cast<const float4*>(h), bias, reinterpret_cast<float4*>(y), rows, n / 4, channels);
    return check_launch("bias_gelu");
}

extern "C" int inc_bias_gelu_bwd(const float* g_y, const float* h, const float* bias, float* g_h, float* row_sums,
                                 int32_t rows, int32_t n, int32_t channels, void* stream) {
    int rc = act::check_shape(g_y, h, bias, rows, n, channels);
    if (rc) return rc;
    if (!g_h || !row_sums) {
        set_error("bias_gelu_bwd: bad arguments");
        return INC_E_INVALID;
    }
    act::k_bias_gelu_bwd<<<act::grid_for(rows), act::BG_BLOCK, 0, as_stream(stream)>>>(
        reinterpret_cast<const float4*>(g_y), reinterpret_cast<const float4*>(h), bias,
        reinterpret_cast<float4*>(g_h), row_sums, rows, n / 4, channels);
    return check_launch("bias_gelu_bwd");
}
