// Shared device/host helpers for the INC 1D time-stepper kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/inc_b200.h"

#define INC_DEV __device__ __forceinline__

namespace inc {

// ---- host-side error reporting ---------------------------------------------
// The message of the last failed call on this host thread.
void set_error(const char* fmt, ...);

// Turns the launch status of the kernel just issued into an INC status code.
int check_launch(const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool is_pow2(int64_t v) { return v > 0 && (v & (v - 1)) == 0; }

// SMs of the current device, looked up once per device
inline int sm_count() {
    static int cache[64] = {0};
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && cache[dev] > 0) return cache[dev];
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (dev >= 0 && dev < 64) cache[dev] = n;
    return n;
}

// ---- warp helpers ------------------------------------------------------------
// All shuffles are issued by the full warp: every kernel here keeps all 32 lanes
// on the same control path (rows past the end are masked, never skipped).
template <int W>
INC_DEV float shfl(float v, int src) { return __shfl_sync(0xffffffffu, v, src, W); }

template <int W>
INC_DEV float group_max(float v) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o, W));
    return v;
}

template <int W>
INC_DEV float group_sum(float v) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, W);
    return v;
}

// Max of |v| with the smallest index among ties (torch.max(dim) returns the
// first occurrence on the CPU reference).
template <int W>
INC_DEV void group_argmax(float& v, int& idx) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) {
        float ov = __shfl_xor_sync(0xffffffffu, v, o, W);
        int oi = __shfl_xor_sync(0xffffffffu, idx, o, W);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
}

// Lanes of this thread's group of W consecutive lanes.
template <int W>
INC_DEV unsigned group_mask() {
    if constexpr (W == 32) return 0xffffffffu;
    else return ((1u << W) - 1u) << ((threadIdx.x & 31) & ~(W - 1));
}

// Max over a group of non-negative values (|u|) in one redux.sync on the bit
// patterns, which order like the values for non-negative floats.  A NaN is
// larger than every finite pattern, so it wins, as in torch.max.
template <int W>
INC_DEV float group_max_nonneg(float v) {
    return __uint_as_float(__reduce_max_sync(group_mask<W>(), __float_as_uint(v)));
}

// group_argmax for non-negative values: the max by redux.sync, then the lowest
// lane holding it (lanes own consecutive cells, so the lowest lane holds the
// first index; torch.max(dim) returns the first occurrence on the CPU).
template <int W>
INC_DEV void group_argmax_nonneg(float& v, int& idx) {
    const unsigned best = __reduce_max_sync(group_mask<W>(), __float_as_uint(v));
    const unsigned hit = __ballot_sync(0xffffffffu, __float_as_uint(v) == best) & group_mask<W>();
    idx = __shfl_sync(0xffffffffu, idx, __ffs(hit) - 1);
    v = __uint_as_float(best);
}

// ---- vector memory helpers ---------------------------------------------------
template <int C>
INC_DEV void load_row_chunk(float (&r)[C], const float* __restrict__ p, bool valid) {
    if (!valid) {
#pragma unroll
        for (int c = 0; c < C; ++c) r[c] = 0.f;
        return;
    }
    const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
    for (int c = 0; c < C / 4; ++c) {
        float4 v = __ldg(q + c);
        r[4 * c] = v.x; r[4 * c + 1] = v.y; r[4 * c + 2] = v.z; r[4 * c + 3] = v.w;
    }
}

template <int C>
INC_DEV void store_row_chunk(float* __restrict__ p, const float (&r)[C], bool valid) {
    if (!valid) return;
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int c = 0; c < C / 4; ++c) q[c] = make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
}

// Streaming store (frames are written once and not re-read by this kernel).
template <int C>
INC_DEV void store_row_chunk_cs(float* __restrict__ p, const float (&r)[C], bool valid) {
    if (!valid) return;
    float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
    for (int c = 0; c < C / 4; ++c) __stcs(q + c, make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]));
}

}  // namespace inc
