// Backward of the hybrid Burgers rollout with the periodic CNN corrector
// (inc_burgers_cnn_rollout): the training step of simulate_rollout
// (trainer/trainer_1d.py:154-183) for that corrector, in one kernel, for rows
// of n = 64, 128, 256 or 512 cells.
//
// Forward per step k: s_k = CNN(u_k), u_{k+1} = S(u_k, s_k), frame k = u_{k+1}.
// Backward, one CTA of T threads holding R rows (T = 256, R = 256 / n for
// n <= 256; T = n = 512, R = 1), segments of ckpt_every steps in reverse order:
//   * replay: the solver re-runs from the segment's checkpoint (one cell per
//     thread, the wide forward) with the forward's saved corrections s_k,
//     keeping every u_k in shared memory;
//   * per step k (last first): u_bar += dL/dframe_k; the network's activations
//     at u_k are recomputed; the solver step's adjoint (advance_bwd_wide, the
//     SSP-RK3/Euler VJP one cell per thread) gives u_bar through S and
//     s_bar = dL/ds_k (+ dL/dcorrection_k); then the network's backward layer
//     by layer, and u_bar += dCNN/du^T s_bar.
//
// Shared memory holds two activation buffers per row (A, B: [32][row]), the
// input row u_k, the adjoint row, one scratch area (the solver's rows, later
// the first layer's partial sums) and the segment's states: about 89 KB at
// n = 256 and ckpt_every = 8, so two CTAs share an SM.  The weights are read
// through the L1 cache.  The schedule of one step (=> marks a block barrier):
//   A = gelu(z1) => B = z2 => A = gelu(z2) => z3 accumulated from A => A = z3,
//   solver adjoint, d = s_bar =>
//   layer 4: dW4, db4 (gelu(z3) formed on the fly from A) => A = dz3 in place =>
//   layer 3: dz2 accumulated from A (registers), times gelu'(z2), B = gelu(z2)
//            => dW3, db3 from B and A => A = dz2, B = gelu(z1) =>
//   layer 2: dz1 accumulated from A (registers), times gelu'(z1) (z1 recomputed
//            from u), dW2, db2 from B and A => A = dz1 =>
//   layer 1: dW1, db1, partial sums of the input adjoint => u_bar.
// Weight gradients: the hidden layers' (32 x 32 x 5 each) are summed per step
// into this CTA's slot of `work` (thread-major, one owner per entry, so the
// order of additions is fixed); the first and last layers' and the biases' are
// kept per warp in registers and summed over the warps in a fixed order at the
// end.  A second kernel adds the CTAs' slots in a fixed order.
//
// Thread maps:
//   convolution tiles: thread g of a row: channel group g / (n/8) (4 channels),
//   8 cells from 8 (g % (n/8));
//   hidden-layer weight gradients: warp w = CO output channels (CO = 32 / warps),
//   lane = input channel, all cells of the CTA's rows, 4 cells per step with
//   float4 windows (a row stride of 4 mod 8 floats makes eight lanes' float4
//   reads of eight rows hit 32 distinct banks);
//   first/last layer and biases: lane = channel, warp = 32 cells of the CTA's
//   rows.
#include "burgers_cnn.cuh"

namespace inc {
namespace burgers {
namespace cnn {

constexpr int BKMAX = 32;  // largest ckpt_every

template <int N>
struct BwdCfg {
    static constexpr int T = N >= 256 ? N : 256;  // threads per CTA
    static constexpr int R = T / N;               // rows per CTA
    static constexpr int RL = row_len<N>();       // activation row stride (floats)
    static constexpr int NW = T / 32;             // warps
    static constexpr int CO = C / NW;             // output channels per warp (hidden weight gradients)
    static constexpr int NG = 2 * CO * KW;        // hidden weight-gradient entries per thread
    static_assert((RL / 4) % 2 == 1, "row stride must be 4 mod 8 floats for conflict-free float4 reads across rows");
    static_assert(N % 32 == 0 && CO * NW == C, "thread maps");
};

template <int N>
struct BwdSmem {
    static constexpr int R = BwdCfg<N>::R, RL = BwdCfg<N>::RL;
    float A[R][C][RL];
    float B[R][C][RL];
    float u[R][RL];  // the network's input row u_k (with its halo)
    float d[R][RL];  // s_bar (layer 4's output adjoint)
    union Scratch {
        WideAdjSmem<N> sol[R];  // the solver's rows (replay and step adjoint)
        float part[R][8][RL];   // layer 1: the input adjoint's partial sums per channel group
    } P;
    float seg[1][R][N];  // [ckpt_every][R][N] states of the current segment (sized at launch)
};
template <int N>
constexpr size_t bwd_smem_bytes(int K) {
    return sizeof(BwdSmem<N>) + (size_t)(K - 1) * BwdCfg<N>::R * N * sizeof(float);
}
constexpr size_t kSmemLimit = 227 * 1024;

// gelu(z) and d gelu(z) / dz = Phi(z) + z phi(z), from one erf
INC_DEV void gelu_both(float z, float& g, float& gp) {
    const float e = erff(z * 0.70710678118654752f);
    g = 0.5f * z * (1.f + e);
    gp = fmaf(z * 0.39894228040143268f, expf(-0.5f * z * z), 0.5f * (1.f + e));
}
INC_DEV float gelu_grad(float z) {
    float g, gp;
    gelu_both(z, g, gp);
    return gp;
}

INC_DEV float2 lds2(const float* p) { return *reinterpret_cast<const float2*>(p); }

// out = gelu(in) over every slot of a [R][C][RL] buffer (halo copies included)
template <int N>
INC_DEV void gelu_buf(float* out, const float* in) {
    constexpr int NV = BwdCfg<N>::R * C * BwdCfg<N>::RL / 4;
    float4* o = reinterpret_cast<float4*>(out);
    const float4* i = reinterpret_cast<const float4*>(in);
    for (int e = threadIdx.x; e < NV; e += BwdCfg<N>::T) {
        const float4 v = i[e];
        o[e] = make_float4(gelu(v.x), gelu(v.y), gelu(v.z), gelu(v.w));
    }
}

// Hidden layer (wt = [ci][co][k]), input adjoint before GELU':
// acc[c][j] = sum_co sum_k W[co][4 cg + c][k] dz[co][8 L + j - k + 2]
template <int N>
INC_DEV void dgrad_acc(const float* __restrict__ wt, float (*dz)[BwdCfg<N>::RL], float (&acc)[4][8], int cg, int L) {
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
            for (int k = 0; k < KW; ++k) wv[c][k] = __ldg(wt + ((4 * cg + c) * C + co) * KW + k);
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < KW; ++k)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[c][j] = fmaf(wv[c][k], a[j + 4 - k], acc[c][j]);
    }
}

// Hidden layer weight gradient over the CTA's rows:
// acc[c][k] = sum_r sum_x dz[r][CO w + c][x] a[r][lane][x + k - 2]
template <int N>
INC_DEV void wgrad_mid(float (&acc)[BwdCfg<N>::CO][KW], float (*a)[C][BwdCfg<N>::RL],
                       float (*dz)[C][BwdCfg<N>::RL], int w, int lane) {
    constexpr int CO = BwdCfg<N>::CO, R = BwdCfg<N>::R;
#pragma unroll
    for (int c = 0; c < CO; ++c)
#pragma unroll
        for (int k = 0; k < KW; ++k) acc[c][k] = 0.f;
    for (int r = 0; r < R; ++r) {
        const float* ar = a[r][lane];
        float4 lo = lds4(ar + apad(0));
#pragma unroll 2
        for (int x0 = 0; x0 < N; x0 += 4) {
            const float4 hi = lds4(ar + apad(x0 + 4));
            const float win[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};  // cells x0-2 .. x0+5
#pragma unroll
            for (int c = 0; c < CO; ++c) {
                const float* dr = dz[r][CO * w + c];
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
}

// this thread's hidden-layer weight-gradient entries (layer l = 0: W2, 1: W3) in
// the CTA's slot, thread-major: slot[(l * CO * KW + i) * T + t] += acc
template <int N>
INC_DEV void slot_add(float* __restrict__ slot, int l, const float (&acc)[BwdCfg<N>::CO][KW], int t) {
    constexpr int CO = BwdCfg<N>::CO, T = BwdCfg<N>::T;
    float* p = slot + (l * CO * KW) * T + t;
    float old[CO * KW];
#pragma unroll
    for (int i = 0; i < CO * KW; ++i) old[i] = p[i * T];
#pragma unroll
    for (int c = 0; c < CO; ++c)
#pragma unroll
        for (int k = 0; k < KW; ++k) p[(c * KW + k) * T] = old[c * KW + k] + acc[c][k];
}

// sum over the 32 cells x0 .. x0 + 31 of row r (bias gradients)
INC_DEV float part_sum(const float* r, int x0) {
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float2 v = lds2(r + apad(x0 + 2 + 2 * i));
        s += v.x + v.y;
    }
    return s;
}

// acc[k] += sum over the 32 cells x0 .. x0 + 31 of  dr[x] * f(ar[x + k - 2]),
// f = gelu (GELU_IN) or the identity
template <bool GELU_IN>
INC_DEV void wgrad_part(float (&acc)[KW], const float* dr, const float* ar, int x0) {
    float win[36];  // cells x0 - 2 .. x0 + 33
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        const float4 v = lds4(ar + apad(x0 + 4 * i));
        win[4 * i] = v.x; win[4 * i + 1] = v.y; win[4 * i + 2] = v.z; win[4 * i + 3] = v.w;
    }
    if (GELU_IN) {
#pragma unroll
        for (int i = 0; i < 36; ++i) win[i] = gelu(win[i]);
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float2 d = lds2(dr + apad(x0 + 2 + 2 * i));
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            acc[k] = fmaf(d.x, win[2 * i + k], acc[k]);
            acc[k] = fmaf(d.y, win[2 * i + 1 + k], acc[k]);
        }
    }
}

template <int N>
__global__ void __launch_bounds__(BwdCfg<N>::T, 256 / N > 0 ? 2 : 1)
    k_cnn_rollout_bwd(Args a, const float* __restrict__ wts, const float* __restrict__ corr,
                      const float* __restrict__ g_corr, float* __restrict__ work, const float* __restrict__ acts) {
    using Cfg = BwdCfg<N>;
    constexpr int T = Cfg::T, R = Cfg::R, RL = Cfg::RL, NW = Cfg::NW, CO = Cfg::CO;
    constexpr int LPG = N / 8;  // lanes per channel group in the tile map
    extern __shared__ __align__(16) unsigned char smraw[];
    BwdSmem<N>& S = *reinterpret_cast<BwdSmem<N>*>(smraw);
    float(*seg)[R][N] = S.seg;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int rl = t / N, g = t % N;                 // this thread's row and cell
    const int cg = g / LPG, L = g % LPG;             // its convolution tile
    const int pr = (32 * w) / N, px = (32 * w) % N;  // its warp's 32-cell part: row, first cell
    const int row = blockIdx.x * R + rl;
    const bool valid = row < a.rows;
    const int src = valid ? row : 0;  // a row past the batch replays row 0 with zero adjoints
    const int K = a.ckpt_every;
    const int nseg = (a.steps + K - 1) / K;
    float* slot = work + (int64_t)blockIdx.x * W_FLOATS;
#pragma unroll
    for (int i = 0; i < Cfg::NG; ++i) slot[i * T + t] = 0.f;
    float g1[KW], g4[KW], gb1 = 0.f, gb2 = 0.f, gb3 = 0.f, gb4 = 0.f;
#pragma unroll
    for (int k = 0; k < KW; ++k) { g1[k] = 0.f; g4[k] = 0.f; }
    Ctx<1> cx;
    make_ctx<1, N>(a, src, g, true, cx);
    cx.has_s = true;
    WideAdjSmem<N>& SW = S.P.sol[rl];
    int parity = 0;
    const int64_t cell = (int64_t)src * N + g;
    float gu = (a.g_final && valid) ? __ldg(a.g_final + cell) : 0.f;
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        {  // replay the segment's states from its checkpoint
            float u[1] = {__ldg(a.ckpts + ((int64_t)src * nseg + sidx) * N + g)};
            for (int j = 0; j < len; ++j) {
                seg[j][rl][g] = u[0];
                if (j + 1 < len) {
                    cx.s[0] = __ldg(corr + ((int64_t)src * a.steps + k0 + j) * N + g);
                    advance_wide<1, N>(a, cx, u, cx.t + (k0 + j) * cx.dt, SW.fw, parity, g);
                }
            }
        }
        __syncthreads();
        for (int j = len - 1; j >= 0; --j) {
            const int k = k0 + j;
            float acc[4][8];
            // ---- the network's activations at u_k
            put_cell<N>(S.u[rl], g, seg[j][rl][g]);
            if (acts) {  // z2, z3 as the forward recorded them (this thread's tiles)
                get_acts(acts, src, a.steps, k, 0, acc, cg, L, N);
                store_tile<N, false>(S.B[rl], acc, cg, L);  // B = z2
                get_acts(acts, src, a.steps, k, 1, acc, cg, L, N);
                store_tile<N, false>(S.A[rl], acc, cg, L);  // A = z3
            } else {
                __syncthreads();
                conv_first<N, true>(wts, S.u[rl], S.A[rl], cg, L);  // A = gelu(z1)
                __syncthreads();
                conv_mid<N, false>(wts + OFF_W2, wts + OFF_B2, S.A[rl], S.B[rl], cg, L);  // B = z2
                __syncthreads();
                gelu_buf<N>(&S.A[0][0][0], &S.B[0][0][0]);  // A = gelu(z2)
                __syncthreads();
                conv_mid_acc<N>(wts + OFF_W3, wts + OFF_B3, S.A[rl], acc, cg, L);
                __syncthreads();
                store_tile<N, false>(S.A[rl], acc, cg, L);  // A = z3
            }
            // ---- the solver step's adjoint: u_bar through S and s_bar
            {
                const int64_t at = ((int64_t)src * a.steps + k) * N + g;
                if (a.g_frames && valid) gu += __ldg(a.g_frames + at);
                float gs = 0.f;
                cx.s[0] = __ldg(corr + at);
                advance_bwd_wide<N>(a, cx, seg[j][rl][g], gu, gs, cx.t + k * cx.dt, SW, parity, g);
                if (g_corr && valid) gs += __ldg(g_corr + at);
                put_cell<N>(S.d[rl], g, gs);
            }
            __syncthreads();
            // ---- layer 4 (32 -> 1, no activation): dW4, db4 with gelu(z3) formed on the fly
            wgrad_part<true>(g4, S.d[pr], S.A[pr][lane], px);
            gb4 += part_sum(S.d[pr], px);
            {  // dz3 = (W4^T s_bar) gelu'(z3), this thread's tile
                float dd[12];
                load12(dd, S.d[rl], L);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int ci = 4 * cg + c;
#pragma unroll
                    for (int j2 = 0; j2 < 8; ++j2) {
                        float s = 0.f;
#pragma unroll
                        for (int kk = 0; kk < KW; ++kk) s = fmaf(__ldg(wts + OFF_W4 + ci * KW + kk), dd[j2 + 4 - kk], s);
                        acc[c][j2] = s;
                    }
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const float2 z = lds2(S.A[rl][ci] + apad(8 * L + 2 + 2 * i));
                        acc[c][2 * i] *= gelu_grad(z.x);
                        acc[c][2 * i + 1] *= gelu_grad(z.y);
                    }
                }
            }
            __syncthreads();  // the windows of z3 read above, before it is overwritten
            store_tile<N, false>(S.A[rl], acc, cg, L);  // A = dz3
            __syncthreads();
            // ---- layer 3: dz2 = (W3^T dz3) gelu'(z2) into registers, B = gelu(z2) in place
            dgrad_acc<N>(wts + OFF_W3, S.A[rl], acc, cg, L);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float* zr = S.B[rl][4 * cg + c];
                float o[8];
#pragma unroll
                for (int i = 0; i < 8; i += 2) {
                    const float2 z = lds2(zr + apad(8 * L + 2 + i));
                    float gp0, gp1;
                    gelu_both(z.x, o[i], gp0);
                    gelu_both(z.y, o[i + 1], gp1);
                    acc[c][i] *= gp0;
                    acc[c][i + 1] *= gp1;
                }
                store8<N>(zr, L, o);
            }
            __syncthreads();
            {  // dW3, db3 from gelu(z2) and dz3
                float gw[CO][KW];
                wgrad_mid<N>(gw, S.B, S.A, w, lane);
                slot_add<N>(slot, 1, gw, t);
            }
            gb3 += part_sum(S.A[pr][lane], px);
            __syncthreads();
            store_tile<N, false>(S.A[rl], acc, cg, L);  // A = dz2
            conv_first<N, true>(wts, S.u[rl], S.B[rl], cg, L);  // B = gelu(z1)
            __syncthreads();
            // ---- layer 2: dz1 = (W2^T dz2) gelu'(z1) into registers; dW2, db2 from gelu(z1), dz2
            dgrad_acc<N>(wts + OFF_W2, S.A[rl], acc, cg, L);
            {
                float z1[4][8];
                conv_first_acc<N>(wts, S.u[rl], z1, cg, L);
#pragma unroll
                for (int c = 0; c < 4; ++c)
#pragma unroll
                    for (int j2 = 0; j2 < 8; ++j2) acc[c][j2] *= gelu_grad(z1[c][j2]);
            }
            {
                float gw[CO][KW];
                wgrad_mid<N>(gw, S.B, S.A, w, lane);
                slot_add<N>(slot, 0, gw, t);
            }
            gb2 += part_sum(S.A[pr][lane], px);
            __syncthreads();
            store_tile<N, false>(S.A[rl], acc, cg, L);  // A = dz1
            __syncthreads();
            // ---- layer 1 (1 -> 32): dW1, db1 (input u_k), the input adjoint as partial sums
            wgrad_part<false>(g1, S.A[pr][lane], S.u[pr], px);
            gb1 += part_sum(S.A[pr][lane], px);
            {
                float part[8];
#pragma unroll
                for (int j2 = 0; j2 < 8; ++j2) part[j2] = 0.f;
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int co = 4 * cg + c;
                    float dd[12];
                    load12(dd, S.A[rl][co], L);
#pragma unroll
                    for (int kk = 0; kk < KW; ++kk) {
                        const float wk = __ldg(wts + OFF_W1 + co * KW + kk);
#pragma unroll
                        for (int j2 = 0; j2 < 8; ++j2) part[j2] = fmaf(wk, dd[j2 + 4 - kk], part[j2]);
                    }
                }
#pragma unroll
                for (int i = 0; i < 4; ++i)
                    *reinterpret_cast<float2*>(S.P.part[rl][cg] + apad(8 * L + 2 + 2 * i)) =
                        make_float2(part[2 * i], part[2 * i + 1]);
            }
            __syncthreads();
            {
                float du = 0.f;
#pragma unroll
                for (int q = 0; q < 8; ++q) du += S.P.part[rl][q][apad(g + 2)];
                gu += du;
            }
            // the next step's first writes (S.u) and the solver's use of S.P come after
            // barriers that order them behind these reads
        }
        __syncthreads();  // segment states are rewritten by the next replay
    }
    if (valid) a.g_u[cell] = gu;
    // ---- this CTA's slot in the packed layout.  Hidden layers: this thread's
    // thread-major entries, moved to their packed places; first/last layers and
    // biases: one partial per warp, summed over the warps in a fixed order.
    float gh[Cfg::NG];
#pragma unroll
    for (int i = 0; i < Cfg::NG; ++i) gh[i] = slot[i * T + t];
    constexpr int NP = 2 * KW + 4;
    float* part = &S.A[0][0][0];  // [NW warps][32 lanes][NP]
    static_assert(NW * 32 * NP <= R * C * RL, "partials fit in one activation buffer");
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
    __syncthreads();  // every thread holds its hidden-layer entries before the slot is rewritten
#pragma unroll
    for (int c = 0; c < CO; ++c)
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            const int co = CO * w + c;
            slot[OFF_W2 + (lane * C + co) * KW + k] = gh[c * KW + k];
            slot[OFF_W3 + (lane * C + co) * KW + k] = gh[CO * KW + c * KW + k];
        }
    if (w == 0) {
        float s[NP];
#pragma unroll
        for (int i = 0; i < NP; ++i) s[i] = 0.f;
        for (int q = 0; q < NW; ++q) {
            const float* p = part + (q * 32 + lane) * NP;
#pragma unroll
            for (int i = 0; i < NP; ++i) s[i] += p[i];
        }
#pragma unroll
        for (int k = 0; k < KW; ++k) {
            slot[OFF_W1 + lane * KW + k] = s[k];
            slot[OFF_W4 + lane * KW + k] = s[KW + k];
        }
        slot[OFF_B1 + lane] = s[2 * KW];
        slot[OFF_B2 + lane] = s[2 * KW + 1];
        slot[OFF_B3 + lane] = s[2 * KW + 2];
        if (lane == 0) slot[OFF_B4] = s[2 * KW + 3];  // each warp's gb4 is the same on all its lanes
    }
}

// g[i] = sum over slots of work[slot][i], slots in order
__global__ void __launch_bounds__(256) k_sum_rows(const float* __restrict__ work, float* __restrict__ g, int slots) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W_FLOATS) return;
    float s = 0.f;
    for (int r = 0; r < slots; ++r) s += work[(int64_t)r * W_FLOATS + i];
    g[i] = s;
}

template <int N>
int max_ckpt_every() {
    int k = BKMAX;
    while (k > 1 && bwd_smem_bytes<N>(k) > kSmemLimit) --k;
    return k;
}

// the backward kernel; *slots = the number of work slots it fills
template <int N>
int launch_bwd(const Args& a, const float* w, const float* corr, const float* g_corr, float* work,
               const float* acts, cudaStream_t st, int* slots) {
    constexpr int R = BwdCfg<N>::R, T = BwdCfg<N>::T;
    if (a.ckpt_every > max_ckpt_every<N>()) {
        set_error("cnn_rollout_bwd: ckpt_every must be <= %d for n = %d (got %d)", max_ckpt_every<N>(), N,
                  a.ckpt_every);
        return INC_E_INVALID;
    }
    const size_t smem = bwd_smem_bytes<N>(a.ckpt_every);
    cudaFuncSetAttribute(k_cnn_rollout_bwd<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    *slots = (a.rows + R - 1) / R;
    k_cnn_rollout_bwd<N><<<*slots, T, smem, st>>>(a, w, corr, g_corr, work, acts);
    return check_launch("burgers_cnn_rollout_bwd");
}

}  // namespace cnn
}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

static int cnn_rollout_bwd(const inc_burgers_desc* d, const float* weights, const float* ckpts,
                           const float* corrections, const float* t_rows, double t0, int32_t steps,
                           int32_t ckpt_every, const float* g_frames, const float* g_corrections,
                           const float* g_final, float* g_u0, float* g_weights, float* work, const float* acts,
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
    if ((reinterpret_cast<uintptr_t>(weights) & 15u) != 0 || (reinterpret_cast<uintptr_t>(acts) & 15u) != 0) {
        set_error("cnn_rollout_bwd: weights and acts must be 16-byte aligned");
        return INC_E_INVALID;
    }
    a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.ckpt_every = ckpt_every;
    a.ckpts = const_cast<float*>(ckpts); a.g_frames = g_frames; a.g_final = g_final; a.g_u = g_u0;
    cudaStream_t st = as_stream(stream);
    int slots = 0;
    switch (d->n) {
        case 64: rc = cnn::launch_bwd<64>(a, weights, corrections, g_corrections, work, acts, st, &slots); break;
        case 128: rc = cnn::launch_bwd<128>(a, weights, corrections, g_corrections, work, acts, st, &slots); break;
        case 256: rc = cnn::launch_bwd<256>(a, weights, corrections, g_corrections, work, acts, st, &slots); break;
        case 512: rc = cnn::launch_bwd<512>(a, weights, corrections, g_corrections, work, acts, st, &slots); break;
        default:
            set_error("cnn_rollout_bwd: n must be 64, 128, 256 or 512 (got %d)", d->n);
            return INC_E_UNSUPPORTED;
    }
    if (rc) return rc;
    cnn::k_sum_rows<<<(cnn::W_FLOATS + 255) / 256, 256, 0, st>>>(work, g_weights, slots);
    return check_launch("burgers_cnn_rollout_bwd (sum)");
}

extern "C" int inc_burgers_cnn_rollout_bwd(const inc_burgers_desc* d, const float* weights, const float* ckpts,
                                           const float* corrections, const float* t_rows, double t0, int32_t steps,
                                           int32_t ckpt_every, const float* g_frames, const float* g_corrections,
                                           const float* g_final, float* g_u0, float* g_weights, float* work,
                                           void* stream) {
    return cnn_rollout_bwd(d, weights, ckpts, corrections, t_rows, t0, steps, ckpt_every, g_frames, g_corrections,
                           g_final, g_u0, g_weights, work, nullptr, stream);
}

extern "C" int inc_burgers_cnn_rollout_bwd_acts(const inc_burgers_desc* d, const float* weights, const float* ckpts,
                                                const float* corrections, const float* t_rows, double t0,
                                                int32_t steps, int32_t ckpt_every, const float* g_frames,
                                                const float* g_corrections, const float* g_final, float* g_u0,
                                                float* g_weights, float* work, const float* acts, void* stream) {
    if (!acts) { set_error("cnn_rollout_bwd_acts: acts must not be NULL"); return INC_E_INVALID; }
    return cnn_rollout_bwd(d, weights, ckpts, corrections, t_rows, t0, steps, ckpt_every, g_frames, g_corrections,
                           g_final, g_u0, g_weights, work, acts, stream);
}
