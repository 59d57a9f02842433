// Backward of the hybrid Burgers rollout with the periodic CNN corrector
// (inc_burgers_cnn_rollout): the training step of simulate_rollout
// (trainer/trainer_1d.py:154-183) for that corrector, in one kernel.
//
// Forward per step k: s_k = CNN(u_k), u_{k+1} = S(u_k, s_k), frame k = u_{k+1}.
// Backward, one CTA (256 threads) per row, segments of ckpt_every steps in
// reverse order:
//   * replay: all threads re-run the solver from the segment's checkpoint (one
//     cell per thread, the wide forward) with the forward's saved corrections
//     s_k, keeping every u_k in shared memory;
//   * per step k (last first): u_bar += dL/dframe_k; the CNN's pre-activations
//     z1..z3 at u_k are recomputed into shared memory; all threads run the
//     solver step's adjoint (advance_bwd_wide, the SSP-RK3/Euler VJP one cell
//     per thread), giving u_bar through S and s_bar = dL/ds_k
//     (+ dL/dcorrection_k); then the network's backward layer by layer: weight
//     gradients (kept in registers for the whole launch) and input adjoints,
//     GELU' applied in place over z; finally u_bar += dCNN/du^T s_bar.
// Weight gradients go to a per-row slot of `work` (the warps' partials summed in
// a fixed order), and a second kernel adds the rows in a fixed order.
//
// Thread maps (256 threads = 8 warps, N = 256 cells):
//   convolution tiles: warp w = channel group (4 channels), lane = 8 cells;
//   weight gradients of the hidden layers: warp w = 4 output channels, lane =
//   input channel, 4 cells per step with float4 windows (the row stride is
//   4 mod 32, so eight lanes' float4 reads of eight rows hit 32 distinct banks);
//   first/last layer and biases: lane = channel, warp = 32-cell part of the row.
#include "burgers_cnn.cuh"

namespace inc {
namespace burgers {
namespace cnn {

constexpr int BN = 256;                // row width of the backward kernel
constexpr int BRL = row_len<BN>();     // activation row stride (floats)
constexpr int BKMAX = 32;              // largest ckpt_every
static_assert(BRL % 32 == 4, "row stride must be 4 mod 32 for conflict-free float4 reads across rows");
static_assert(BN / 8 == 32, "one channel group per warp");

struct BwdSmem {
    float w[W_SMEM];
    float z[3][C][BRL];  // pre-activations of layers 1-3, replaced in place by their adjoints
    float x[C][BRL];     // GELU outputs of the layer being differentiated / partial sums
    float u[BRL];        // the network's input row u_k (with its halo)
    float d[BRL];        // adjoint row: s_bar (layer 4 output), then the network's input adjoint
    float seg[1][BN];    // [ckpt_every][BN] states of the current segment (sized at launch)
};
constexpr size_t bwd_smem_bytes(int K) { return sizeof(BwdSmem) + (size_t)(K - 1) * BN * sizeof(float); }

// d gelu(z) / dz = Phi(z) + z phi(z)
INC_DEV float gelu_grad(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// out = gelu(in) over every slot of a [C][BRL] buffer (halo copies included),
// by threads first .. first + count - 1, four slots at a time
INC_DEV void gelu_rows(float (*out)[BRL], float (*in)[BRL], int first = 0, int count = 256) {
    float4* o = reinterpret_cast<float4*>(&out[0][0]);
    const float4* i = reinterpret_cast<const float4*>(&in[0][0]);
    for (int e = (int)threadIdx.x - first; e < C * BRL / 4; e += count) {
        const float4 v = i[e];
        o[e] = make_float4(gelu(v.x), gelu(v.y), gelu(v.z), gelu(v.w));
    }
}

INC_DEV float2 lds2(const float* p) { return *reinterpret_cast<const float2*>(p); }

// Hidden layer (wt = [ci][co][k]): adjoint of its input, fused with GELU' of the
// previous layer: zprev[ci][x] <- (sum_co sum_k W[co][ci][k] dz[co][x-k+2]) * gelu'(zprev[ci][x])
// for ci in 4 cg .. 4 cg + 3, x in 8 L .. 8 L + 7 (this thread's tile, in place).
INC_DEV void dgrad_mid(const float* wt, float (*dz)[BRL], float (*zprev)[BRL], int cg, int L) {
    float acc[4][8];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[c][j] = 0.f;
#pragma unroll 2
    for (int co = 0; co < C; ++co) {
        float a[12];
        load12(a, dz[co], L);
        float wv[4][KW];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < KW; ++k) wv[c][k] = wt[((4 * cg + c) * C + co) * KW + k];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < KW; ++k)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[c][j] = fmaf(wv[c][k], a[j + 4 - k], acc[c][j]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float* row = zprev[4 * cg + c];
        float o[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 z = lds2(row + apad(8 * L + 2 + 2 * i));
            o[2 * i] = acc[c][2 * i] * gelu_grad(z.x);
            o[2 * i + 1] = acc[c][2 * i + 1] * gelu_grad(z.y);
        }
        store8<BN>(row, L, o);
    }
}

// Hidden layer weight gradient: acc[c][k] += sum_x dz[4 w + c][x] a[lane][x + k - 2].
INC_DEV void wgrad_mid(float (&acc)[4][KW], float (*a)[BRL], float (*dz)[BRL], int w, int lane) {
    const float* ar = a[lane];
    float4 lo = *reinterpret_cast<const float4*>(ar + apad(0));
#pragma unroll 2
    for (int x0 = 0; x0 < BN; x0 += 4) {
        const float4 hi = *reinterpret_cast<const float4*>(ar + apad(x0 + 4));
        const float win[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};  // cells x0-2 .. x0+5
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float* dr = dz[4 * w + c];
            const float2 d01 = lds2(dr + apad(x0 + 2)), d23 = lds2(dr + apad(x0 + 4));
            const float dv[4] = {d01.x, d01.y, d23.x, d23.y};
#pragma unroll
            for (int k = 0; k < KW; ++k)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[c][k] = fmaf(dv[j], win[j + k], acc[c][k]);
        }
        lo = hi;
    }
}

// sum over the 32 cells of part w of row r (bias gradients)
INC_DEV float row_part_sum(const float* r, int w) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float2 v = lds2(r + apad(32 * w + 2 + 2 * i));
        s += v.x + v.y;
    }
    return s;
}

// acc[k] += sum over the 32 cells of part w of  dr[x] * ar[x + k - 2]
INC_DEV void wgrad_part(float (&acc)[KW], const float* dr, const float* ar, int w) {
    float win[36];  // cells 32 w - 2 .. 32 w + 33
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float4 v = *reinterpret_cast<const float4*>(ar + apad(32 * w + 4 * i));
        win[4 * i] = v.x; win[4 * i + 1] = v.y; win[4 * i + 2] = v.z; win[4 * i + 3] = v.w;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float2 d = lds2(dr + apad(32 * w + 2 + 2 * i));
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            acc[k] = fmaf(d.x, win[2 * i + k], acc[k]);
            acc[k] = fmaf(d.y, win[2 * i + 1 + k], acc[k]);
        }
    }
}

__global__ void __launch_bounds__(256) k_cnn_rollout_bwd(Args a, const float* __restrict__ wts,
                                                         const float* __restrict__ corr,
                                                         const float* __restrict__ g_corr,
                                                         float* __restrict__ work) {
    extern __shared__ __align__(16) unsigned char smraw[];
    BwdSmem& S = *reinterpret_cast<BwdSmem*>(smraw);
    float(*seg)[BN] = S.seg;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int row = blockIdx.x;
    const int K = a.ckpt_every;
    const int nseg = (a.steps + K - 1) / K;
    for (int i = t; i < W_FLOATS; i += blockDim.x) S.w[i] = __ldg(wts + i);
    // persistent weight-gradient sums
    float g2[4][KW], g3[4][KW], g1[KW], g4[KW], gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, gb4 = 0.f;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < KW; ++k) { g2[c][k] = 0.f; g3[c][k] = 0.f; }
#pragma unroll
    for (int k = 0; k < KW; ++k) { g1[k] = 0.f; g4[k] = 0.f; }
    // The solver, one cell per thread (the wide-row layout): all eight warps run the
    // segment replay and the step adjoints.  Its shared scratch is S.x, which holds
    // no activations while the solver runs.
    WideAdjSmem<BN>& SW = *reinterpret_cast<WideAdjSmem<BN>*>(&S.x[0][0]);
    Ctx<1> cx;
    make_ctx<1, BN>(a, row, t, true, cx);
    cx.has_s = true;
    int parity = 0;
    const int64_t cell = (int64_t)row * BN + t;
    float gu = a.g_final ? __ldg(a.g_final + cell) : 0.f;
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        {  // replay the segment's states from its checkpoint
            float u[1] = {__ldg(a.ckpts + ((int64_t)row * nseg + sidx) * BN + t)};
            for (int j = 0; j < len; ++j) {
                seg[j][t] = u[0];
                if (j + 1 < len) {
                    cx.s[0] = __ldg(corr + ((int64_t)row * a.steps + k0 + j) * BN + t);
                    advance_wide<1, BN>(a, cx, u, cx.t + (k0 + j) * cx.dt, SW.fw, parity, t);
                }
            }
        }
        __syncthreads();
        for (int j = len - 1; j >= 0; --j) {
            const int k = k0 + j;
            // ---- the network's pre-activations at u_k
            put_cell<BN>(S.u, t, seg[j][t]);
            __syncthreads();
            conv_first<BN, false>(S.w, S.u, S.z[0], w, lane);
            __syncthreads();
            gelu_rows(S.x, S.z[0]);
            __syncthreads();
            conv_mid<BN, false>(S.w + OFF_W2, S.w + OFF_B2, S.x, S.z[1], w, lane);
            __syncthreads();
            gelu_rows(S.x, S.z[1]);
            __syncthreads();
            conv_mid<BN, false>(S.w + OFF_W3, S.w + OFF_B3, S.x, S.z[2], w, lane);
            __syncthreads();
            // ---- the solver step's adjoint, all threads: u_bar through S and s_bar
            {
                const int64_t at = ((int64_t)row * a.steps + k) * BN + t;
                if (a.g_frames) gu += __ldg(a.g_frames + at);
                float gs = 0.f;
                cx.s[0] = __ldg(corr + at);
                advance_bwd_wide<BN>(a, cx, seg[j][t], gu, gs, cx.t + k * cx.dt, SW, parity, t);
                if (g_corr) gs += __ldg(g_corr + at);
                put_cell<BN>(S.d, t, gs);
            }
            __syncthreads();
            gelu_rows(S.x, S.z[2]);  // layer 4's input gelu(z3), after the solver's use of S.x
            __syncthreads();
            // ---- layer 4 (32 -> 1, no activation): dW4, db4, then dz3 in place of z3
            wgrad_part(g4, S.d, S.x[lane], w);
            gb4 += row_part_sum(S.d, w);
            {
                float dd[12];
                load12(dd, S.d, lane);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int ci = 4 * w + c;
                    float* zr = S.z[2][ci];
                    float o[8];
#pragma unroll
                    for (int j2 = 0; j2 < 8; ++j2) {
                        float acc = 0.f;
#pragma unroll
                        for (int kk = 0; kk < KW; ++kk) acc = fmaf(S.w[OFF_W4 + ci * KW + kk], dd[j2 + 4 - kk], acc);
                        o[j2] = acc;
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const float2 z = lds2(zr + apad(8 * lane + 2 + 2 * i));
                        o[2 * i] *= gelu_grad(z.x);
                        o[2 * i + 1] *= gelu_grad(z.y);
                    }
                    store8<BN>(zr, lane, o);
                }
            }
            __syncthreads();
            // ---- layer 3: dW3, db3 (input gelu(z2)), dz2 in place of z2
            gelu_rows(S.x, S.z[1]);
            __syncthreads();
            wgrad_mid(g3, S.x, S.z[2], w, lane);
            gb3 += row_part_sum(S.z[2][lane], w);
            dgrad_mid(S.w + OFF_W3, S.z[2], S.z[1], w, lane);
            __syncthreads();
            // ---- layer 2: dW2, db2 (input gelu(z1)), dz1 in place of z1
            gelu_rows(S.x, S.z[0]);
            __syncthreads();
            wgrad_mid(g2, S.x, S.z[1], w, lane);
            gb2 += row_part_sum(S.z[1][lane], w);
            dgrad_mid(S.w + OFF_W2, S.z[1], S.z[0], w, lane);
            __syncthreads();
            // ---- layer 1 (1 -> 32): dW1, db1 (input u_k), and the input adjoint as partial sums
            wgrad_part(g1, S.z[0][lane], S.u, w);
            gb1 += row_part_sum(S.z[0][lane], w);
            {
                float part[8];
#pragma unroll
                for (int j2 = 0; j2 < 8; ++j2) part[j2] = 0.f;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int co = 4 * w + c;
                    float dd[12];
                    load12(dd, S.z[0][co], lane);
#pragma unroll
                    for (int kk = 0; kk < KW; ++kk) {
                        const float wk = S.w[OFF_W1 + co * KW + kk];
#pragma unroll
                        for (int j2 = 0; j2 < 8; ++j2) part[j2] = fmaf(wk, dd[j2 + 4 - kk], part[j2]);
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    *reinterpret_cast<float2*>(S.x[w] + apad(8 * lane + 2 + 2 * i)) = make_float2(part[2 * i], part[2 * i + 1]);
            }
            __syncthreads();
            {
                float du = 0.f;
#pragma unroll
                for (int q = 0; q < 8; ++q) du += S.x[q][apad(t + 2)];
                S.d[apad(t + 2)] = du;
            }
            __syncthreads();
            gu += S.d[apad(t + 2)];
            // the next step's first writes (S.u) are ordered after these reads by its first barrier
        }
        __syncthreads();  // segment states are rewritten by the next replay
    }
    a.g_u[cell] = gu;
    // ---- weight gradients: per-thread sums -> shared -> this row's slot of work.
    // W2, W3: one slot per thread.  W1, W4 and the biases: one partial per warp,
    // summed over the warps in a fixed order (the result does not depend on timing).
    float* acc = &S.z[0][0][0];
    constexpr int NP = 2 * KW + 4;
    float* part = &S.z[2][0][0];  // [8 warps][32 lanes][NP], past acc's W_FLOATS
    __syncthreads();
    for (int i = t; i < W_FLOATS; i += blockDim.x) acc[i] = 0.f;
    {
        float* p = part + (w * 32 + lane) * NP;
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            p[k] = g1[k];
            p[KW + k] = g4[k];
        }
        p[2 * KW] = gb1;
        p[2 * KW + 1] = gb2;
        p[2 * KW + 2] = gb3;
        p[2 * KW + 3] = gb4;
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            const int co = 4 * w + c;
            acc[OFF_W2 + (lane * C + co) * KW + k] = g2[c][k];
            acc[OFF_W3 + (lane * C + co) * KW + k] = g3[c][k];
        }
    if (w == 0) {
        float s[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) s[i] = 0.f;
        for (int q = 0; q < 8; ++q) {
            const float* p = part + (q * 32 + lane) * NP;
#pragma unroll
            for (int i = 0; i < NP; ++i) s[i] += p[i];
        }
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            acc[OFF_W1 + lane * KW + k] = s[k];
            acc[OFF_W4 + lane * KW + k] = s[KW + k];
        }
        acc[OFF_B1 + lane] = s[2 * KW];
        acc[OFF_B2 + lane] = s[2 * KW + 1];
        acc[OFF_B3 + lane] = s[2 * KW + 2];
        if (lane == 0) acc[OFF_B4] = s[2 * KW + 3];  // each warp's gb4 is the same on all its lanes
    }
    __syncthreads();
    for (int i = t; i < W_FLOATS; i += blockDim.x) work[(int64_t)row * W_FLOATS + i] = acc[i];
}

// g[i] = sum over rows of work[row][i], rows in order
__global__ void __launch_bounds__(256) k_sum_rows(const float* __restrict__ work, float* __restrict__ g, int rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W_FLOATS) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += work[(int64_t)r * W_FLOATS + i];
    g[i] = s;
}

}  // namespace cnn
}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

extern "C" int inc_burgers_cnn_rollout_bwd(const inc_burgers_desc* d, const float* weights, const float* ckpts,
                                           const float* corrections, const float* t_rows, double t0, int32_t steps,
                                           int32_t ckpt_every, const float* g_frames, const float* g_corrections,
                                           const float* g_final, float* g_u0, float* g_weights, float* work,
                                           void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!weights || !ckpts || !corrections || !g_u0 || !g_weights || !work || steps <= 0 || ckpt_every <= 0) {
        set_error("cnn_rollout_bwd: bad arguments");
        return INC_E_INVALID;
    }
    if (ckpt_every > cnn::BKMAX) {
        set_error("cnn_rollout_bwd: ckpt_every must be <= %d (got %d)", cnn::BKMAX, ckpt_every);
        return INC_E_INVALID;
    }
    if (d->n != cnn::BN) {
        set_error("cnn_rollout_bwd: n must be %d (got %d)", cnn::BN, d->n);
        return INC_E_UNSUPPORTED;
    }
    if ((reinterpret_cast<uintptr_t>(weights) & 15u) != 0) {
        set_error("cnn_rollout_bwd: weights must be 16-byte aligned");
        return INC_E_INVALID;
    }
    a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.ckpt_every = ckpt_every;
    a.ckpts = const_cast<float*>(ckpts); a.g_frames = g_frames; a.g_final = g_final; a.g_u = g_u0;
    cudaStream_t st = as_stream(stream);
    const size_t smem = cnn::bwd_smem_bytes(ckpt_every);
    cudaFuncSetAttribute(cnn::k_cnn_rollout_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cnn::k_cnn_rollout_bwd<<<a.rows, 256, smem, st>>>(a, weights, corrections, g_corrections, work);
    rc = check_launch("burgers_cnn_rollout_bwd");
    if (rc) return rc;
    cnn::k_sum_rows<<<(cnn::W_FLOATS + 255) / 256, 256, 0, st>>>(work, g_weights, a.rows);
    return check_launch("burgers_cnn_rollout_bwd (sum)");
}
