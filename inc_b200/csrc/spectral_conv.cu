// FNO spectral convolution (SpectralConv1d of the FNO corrector,
// models/models_1d/fno.py:6-37 of tum-pbs/INC) on the KS row-pair FFT:
//   y[b][o] = irfft( sum_c rfft(x[b][c])[k] * W[c][o][k]  for k < modes, 0 above ).
// The [B][W][n] activations are a flat matrix of B*W rows; W is even, so pair p
// (rows 2p, 2p+1) never straddles two trajectories.  Three kernels:
//   k_sc_modes   - streaming: one row pair per group shares one complex FFT
//                  (z = x_a + i x_b); the split storage of ks_kernels.cuh hands
//                  each row its half spectrum; the first `modes` coefficients go
//                  to a [B*W][modes] complex array.  Persistent loop over pairs,
//                  the next pair's rows loaded before the current transform.
//   k_sc_mix     - the mode mixing, for each mode k a complex [tile x W] by
//                  [W x W] product: the weights' k-slice (laid out mode-major
//                  by k_sc_weights) is staged in shared memory once per tile of
//                  trajectories, not read per trajectory.
//   k_sc_inverse - streaming: pairs of output rows from one inverse FFT of the
//                  packed spectrum Z = F_a + i F_b, built from the mixed modes
//                  with their Hermitian mirrors and zeros above `modes` (irfft's
//                  convention: the DC coefficient's imaginary part is ignored),
//                  plus a per-channel bias and an addend tensor (the FNO layer's
//                  1x1 convolution), so the layer's sum is one pass.
// The backward (adjoint w.r.t. x) runs the same kernels on dL/dy: its FFT gives
// dL/dF = (c_k / n) FFT(dL/dy)[k] (c_0 = 1 with the imaginary part dropped,
// c_k = 2), the mixing uses conj(W) transposed, and the inverse builds
// dL/dx[n] = sum_k Re(dL/dX[k] e^{2 pi i k n / N}) (modes k >= 1 halved: the
// Hermitian packing counts them twice).  dL/dF is the weight gradient's input,
// sum over the batch of dL/dF[o][k] conj(X[c][k]).
#include "ks_kernels.cuh"

namespace inc {
namespace ks {

constexpr int SC_BLOCK = 256;

template <int P, int T>
INC_DEV Twiddles<P, T> sc_twiddles(float2* sm, int t) {
    Twiddles<P, T> tw;
    tw.sm = sm;
    if constexpr (twiddles_in_registers<P, T>()) {
        compute_lane_twiddles<P, T>(tw, t);
    } else {
        fill_twiddle_table<P, T>(sm);
        __syncthreads();
    }
    return tw;
}

// rows 2p and 2p+1 of a [rows][N] matrix as (row 2p, row 2p+1) pairs; zeros
// for a pair past the end.
template <int P, int T>
INC_DEV void sc_load_pair(const float* __restrict__ rows, int p, bool live, int t, float2 (&v)[P]) {
    constexpr int N = P * T;
    const float* ra = rows + (int64_t)(live ? p : 0) * 2 * N;
#pragma unroll
    for (int m = 0; m < P; ++m)
        v[m] = live ? make_float2(__ldg(ra + t + T * m), __ldg(ra + N + t + T * m)) : make_float2(0.f, 0.f);
}

// in [2*npairs][N] -> modes [2*npairs][M].  BWD scales to dL/dF.
template <int P, int T, bool BWD>
__global__ void __launch_bounds__(SC_BLOCK) k_sc_modes(const float* __restrict__ in, float2* __restrict__ modes,
                                                       int npairs, int M) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    constexpr int G = SC_BLOCK / T;
    const int t = threadIdx.x % T, grp = threadIdx.x / T;
    const Twiddles<P, T> tw = sc_twiddles<P, T>(sm, t);
    const Buf<P, T> buf = group_buf<P, T>(sm + tw_size<P, T>() + grp * fwd_group_smem<P, T>(), t);
    const float sc = BWD ? 2.f / (float)N : 1.f;
    const float sc0 = BWD ? 1.f / (float)N : 1.f;
    // Every group of the block runs the same trip count (sub-warp groups share
    // their warp's __syncwarp).
    const int stride = gridDim.x * G;
    int p = blockIdx.x * G + grp;
    float2 nxt[P];
    sc_load_pair<P, T>(in, p, p < npairs, t, nxt);
    for (int p0 = blockIdx.x * G; p0 < npairs; p0 += stride, p += stride) {
        float2 v[P];
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = nxt[m];
        sc_load_pair<P, T>(in, p + stride, p + stride < npairs, t, nxt);
        fft_fwd<P, T>(v, buf, tw, t);
        if (M <= T) {
            // Z[k], k < M, is register 0 of lane k and Z[N-k] register P-1 of lane
            // T-k: one exchange gives lane k both rows' coefficients,
            // A = (Z[k] + conj Z[N-k]) / 2, B = (Z[k] - conj Z[N-k]) / 2i.
            const int partner = (T - t) & (T - 1);
            const float2 zm = make_float2(shfl<T>(v[P - 1].x, partner), shfl<T>(v[P - 1].y, partner));
            if (p >= npairs || t >= M) continue;
            const float2 z = v[0];
            float2* ma = modes + (int64_t)(2 * p) * M;
            if (t == 0) {  // (A[0], B[0]) real
                ma[0] = make_float2(z.x * sc0, 0.f);
                ma[M] = make_float2(z.y * sc0, 0.f);
            } else {
                const float h = 0.5f * sc;
                ma[t] = make_float2(h * (z.x + zm.x), h * (z.y - zm.y));
                ma[M + t] = make_float2(h * (z.y + zm.y), -h * (z.x - zm.x));
            }
            continue;
        }
        to_split<P, T>(v, t, buf.a);
        if (p >= npairs) continue;
        float2* ma = modes + (int64_t)(2 * p) * M;
        float2* mb = ma + M;
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const int k = t + T * m;
            const float2 z = v[m];
            if (k == 0) {  // (A[0], B[0]) real
                ma[0] = make_float2(z.x * sc0, 0.f);
                mb[0] = make_float2(z.y * sc0, 0.f);
            } else if (k < M) {  // A[k]
                ma[k] = cscale(z, sc);
            } else if (k > N / 2 && N - k < M) {  // B[N-k] = conj(slot k)
                mb[N - k] = make_float2(z.x * sc, -z.y * sc);
            }
        }
    }
}

// out[b][r][k] = s_k * sum_j in[b][j][k] * S[j][r], S[j][r] = W[j][r][k] (forward)
// or conj(W[r][j][k]) (backward); s_k = 1/n forward, 1 (k = 0) or 1/2 backward.
// Block: one mode k and a tile of MIX_TB trajectories, S and the tile's modes
// staged in shared memory.  Thread: output rows r0, r0 + 1 (one 16-byte load of
// S per j) for MIX_RB trajectories bsub, bsub + bstep, ... (each a broadcast
// load).  The tile's rows are padded with zeros to whole rounds of
// bstep * MIX_RB, so the inner loop has no bounds checks; results for the
// padding are not stored.  The weights arrive mode-major and complex
// interleaved (k_sc_weights), so a block's slice is one contiguous 16-byte-load
// copy.
constexpr int MIX_TB = 32;
constexpr int MIX_RB = 4;

__host__ __device__ constexpr int mix_bstep(int W) { return SC_BLOCK / (W / 2); }
__host__ __device__ constexpr int mix_xrows(int W) {
    return (MIX_TB + mix_bstep(W) * MIX_RB - 1) / (mix_bstep(W) * MIX_RB) * (mix_bstep(W) * MIX_RB);
}

// S for every mode: wt[k][j][r] = W[j][r][k] (forward) or conj(W[r][j][k])
// (backward), complex interleaved.  Thread: one weight entry, read in the
// weights' own order (mode fastest).
template <bool BWD>
__global__ void __launch_bounds__(SC_BLOCK) k_sc_weights(const float* __restrict__ w_re,
                                                         const float* __restrict__ w_im, float2* __restrict__ wt,
                                                         int W, int M) {
    const int e = blockIdx.x * SC_BLOCK + threadIdx.x;  // (c * W + o) * M + k
    if (e >= W * W * M) return;
    const int k = e % M, co = e / M;
    const int c = co / W, o = co - c * W;
    const float re = __ldg(w_re + e), im = __ldg(w_im + e);
    const int i = BWD ? o * W + c : co;  // S[j][r]: (j, r) = (c, o) forward, (o, c) backward
    wt[(int64_t)k * W * W + i] = make_float2(re, BWD ? -im : im);
}

template <bool BWD>
__global__ void __launch_bounds__(SC_BLOCK) k_sc_mix(const float2* __restrict__ in, const float2* __restrict__ wt,
                                                     float2* __restrict__ out, int B, int W, int M,
                                                     float fwd_scale) {
    extern __shared__ float4 sm4[];
    float2* S = reinterpret_cast<float2*>(sm4);  // [W][W]: S[j * W + r]
    float2* X = S + W * W;                       // [mix_xrows(W)][W], zero past the tile
    const int k = blockIdx.x;
    const int b0 = blockIdx.y * MIX_TB;
    const int nb = min(MIX_TB, B - b0);
    const float4* src = reinterpret_cast<const float4*>(wt + (int64_t)k * W * W);
#pragma unroll 4
    for (int i = threadIdx.x; i < W * W / 2; i += SC_BLOCK) sm4[i] = __ldg(src + i);
    // the tile's modes: gathers with stride M, unrolled so that several are in flight
#pragma unroll 8
    for (int i = threadIdx.x; i < nb * W; i += SC_BLOCK) X[i] = __ldg(in + ((int64_t)b0 * W + i) * M + k);
    for (int i = nb * W + threadIdx.x; i < mix_xrows(W) * W; i += SC_BLOCK) X[i] = make_float2(0.f, 0.f);
    __syncthreads();
    const float s = BWD ? (k == 0 ? 1.f : 0.5f) : fwd_scale;
    const int half = W / 2;  // threads per trajectory
    const int bstep = mix_bstep(W);
    const int r0 = 2 * (threadIdx.x % half);
    const int bsub = threadIdx.x / half;
    if (bsub >= bstep) return;  // the block's last threads when W / 2 does not divide it
    const float4* S4 = reinterpret_cast<const float4*>(S) + r0 / 2;
    for (int base = bsub; base < nb; base += bstep * MIX_RB) {
        float acc[MIX_RB][4];
#pragma unroll
        for (int q = 0; q < MIX_RB; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.f;
        const float2* xq = X + base * W;
#pragma unroll 4
        for (int j = 0; j < W; ++j) {
            const float4 w = S4[j * half];  // S[j][r0], S[j][r0 + 1]
#pragma unroll
            for (int q = 0; q < MIX_RB; ++q) {
                const float2 x = xq[q * bstep * W + j];
                acc[q][0] = fmaf(x.x, w.x, fmaf(-x.y, w.y, acc[q][0]));
                acc[q][1] = fmaf(x.x, w.y, fmaf(x.y, w.x, acc[q][1]));
                acc[q][2] = fmaf(x.x, w.z, fmaf(-x.y, w.w, acc[q][2]));
                acc[q][3] = fmaf(x.x, w.w, fmaf(x.y, w.z, acc[q][3]));
            }
        }
#pragma unroll
        for (int q = 0; q < MIX_RB; ++q) {
            const int bb = base + q * bstep;
            if (bb < nb) {
                float2* o = out + ((int64_t)(b0 + bb) * W + r0) * M + k;
                o[0] = make_float2(acc[q][0] * s, acc[q][1] * s);
                o[M] = make_float2(acc[q][2] * s, acc[q][3] * s);
            }
        }
    }
}

// With M <= T the packed spectrum of a pair is nonzero in two registers of a
// lane only: register 0 of lane t holds slot t (F[t] for t < M), register P-1
// slot N - (T - t) (the mirror of F[T - t] for 0 < T - t < M).  These are the
// four coefficients lane t needs, loaded one pair ahead.
struct LaneModes {
    float2 a0, b0, a1, b1;
};

template <int T>
INC_DEV LaneModes sc_lane_modes(const float2* __restrict__ fm, int p, bool live, int t, int M) {
    LaneModes c;
    c.a0 = c.b0 = c.a1 = c.b1 = make_float2(0.f, 0.f);
    if (live) {
        const float2* fa = fm + (int64_t)(2 * p) * M;
        if (t < M) {
            c.a0 = fa[t];
            c.b0 = fa[M + t];
        }
        if (t > 0 && T - t < M) {
            c.a1 = fa[T - t];
            c.b1 = fa[M + T - t];
        }
    }
    return c;
}

// mixed modes [2*npairs][M] -> out [2*npairs][N] (+ bias[row % W] + addend).
template <int P, int T>
__global__ void __launch_bounds__(SC_BLOCK) k_sc_inverse(const float2* __restrict__ fm, float* __restrict__ out,
                                                         const float* __restrict__ bias,
                                                         const float* __restrict__ addend, int npairs, int W,
                                                         int M) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    constexpr int G = SC_BLOCK / T;
    const int t = threadIdx.x % T, grp = threadIdx.x / T;
    const Twiddles<P, T> tw = sc_twiddles<P, T>(sm, t);
    const Buf<P, T> buf = group_buf<P, T>(sm + tw_size<P, T>() + grp * fwd_group_smem<P, T>(), t);
    const int stride = gridDim.x * G;
    const bool sparse = M <= T;
    int p = blockIdx.x * G + grp;
    LaneModes nxt = sc_lane_modes<T>(fm, p, sparse && p < npairs, t, M);
    for (int p0 = blockIdx.x * G; p0 < npairs; p0 += stride, p += stride) {
        const bool live = p < npairs;
        // the epilogue's addend first: its loads overlap the transform
        float2 add[P];
        if (addend) sc_load_pair<P, T>(addend, p, live, t, add);
        // packed spectrum F_a + i F_b (mirrors: conj(F_a) + i conj(F_b)), swapped:
        // the inverse transform is swap(FFT(swap(z)))
        float2 v[P];
        if (sparse) {
            const LaneModes c = nxt;
            nxt = sc_lane_modes<T>(fm, p + stride, p + stride < npairs, t, M);
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = make_float2(0.f, 0.f);
            v[0] = cswap(t == 0 ? make_float2(c.a0.x, c.b0.x) : make_float2(c.a0.x - c.b0.y, c.a0.y + c.b0.x));
            v[P - 1] = cswap(make_float2(c.a1.x + c.b1.y, c.b1.x - c.a1.y));
        } else {
            const float2* fa = fm + (int64_t)(2 * (live ? p : 0)) * M;
            const float2* fb = fa + M;
#pragma unroll
            for (int m = 0; m < P; ++m) {
                const int k = t + T * m;
                float2 z = make_float2(0.f, 0.f);
                if (!live) {
                } else if (k == 0) {
                    z = make_float2(fa[0].x, fb[0].x);
                } else if (k < M) {
                    const float2 a = fa[k], b = fb[k];
                    z = make_float2(a.x - b.y, a.y + b.x);
                } else if (N - k < M) {
                    const float2 a = fa[N - k], b = fb[N - k];
                    z = make_float2(a.x + b.y, b.x - a.y);
                }
                v[m] = cswap(z);
            }
        }
        fft_fwd<P, T>(v, buf, tw, t);
        if (!live) continue;
        float ba = 0.f, bb = 0.f;
        if (bias) {
            ba = __ldg(bias + (2 * p) % W);
            bb = __ldg(bias + (2 * p + 1) % W);
        }
        float* ya = out + (int64_t)(2 * p) * N;
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const int i = t + T * m;
            const float2 y = cswap(v[m]);
            float y0 = y.x + ba, y1 = y.y + bb;
            if (addend) {
                y0 += add[m].x;
                y1 += add[m].y;
            }
            ya[i] = y0;
            ya[N + i] = y1;
        }
    }
}

template <int P, int T>
constexpr size_t sc_fft_smem() {
    return ((size_t)tw_size<P, T>() + (size_t)(SC_BLOCK / T) * fwd_group_smem<P, T>()) * sizeof(float2);
}

template <typename K>
void sc_allow_smem(K kernel, size_t smem) {
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// Resident blocks of a streaming kernel on the whole device (SM count times
// blocks per SM), queried once per kernel instance: the smem size is fixed per
// instance and the devices of a process are alike.
template <typename K>
int sc_resident(K kernel, size_t smem) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, SC_BLOCK, smem);
    return sms * (per_sm > 0 ? per_sm : 1);
}

// Grid of the streaming kernels: every SM's resident blocks, at most one block
// per SC_BLOCK / T pairs.
inline int sc_grid(int resident, int npairs, int G) {
    const int want = (npairs + G - 1) / G;
    return want < resident ? want : resident;
}

template <int P, int T, bool BWD>
int run_spectral_conv(const float* in, float* out, const float* w_re, const float* w_im, const float* bias,
                      const float* addend, float2* modes, float2* mixed, int batch, int W, int M, cudaStream_t st) {
    constexpr int N = P * T;
    constexpr int G = SC_BLOCK / T;
    const int npairs = batch * W / 2;
    const size_t fsm = sc_fft_smem<P, T>();
    sc_allow_smem(k_sc_modes<P, T, BWD>, fsm);
    sc_allow_smem(k_sc_inverse<P, T>, fsm);
    // (after the smem opt-in, which the occupancy query depends on)
    static const int res1 = sc_resident(k_sc_modes<P, T, BWD>, fsm);
    static const int res3 = sc_resident(k_sc_inverse<P, T>, fsm);
    const int g1 = sc_grid(res1, npairs, G);
    k_sc_modes<P, T, BWD><<<g1, SC_BLOCK, fsm, st>>>(in, modes, npairs, M);
    float2* wt = mixed + (int64_t)batch * W * M;
    k_sc_weights<BWD><<<(W * W * M + SC_BLOCK - 1) / SC_BLOCK, SC_BLOCK, 0, st>>>(w_re, w_im, wt, W, M);
    const size_t msm = ((size_t)W * W + (size_t)mix_xrows(W) * W) * sizeof(float2);
    sc_allow_smem(k_sc_mix<BWD>, msm);
    const dim3 g2(M, (batch + MIX_TB - 1) / MIX_TB);
    k_sc_mix<BWD><<<g2, SC_BLOCK, msm, st>>>(modes, wt, mixed, batch, W, M, 1.f / (float)N);
    const int g3 = sc_grid(res3, npairs, G);
    k_sc_inverse<P, T><<<g3, SC_BLOCK, fsm, st>>>(mixed, out, BWD ? nullptr : bias, BWD ? nullptr : addend, npairs,
                                                  W, M);
    return check_launch("spectral_conv");
}

template <bool BWD>
int spectral_conv_dispatch(const float* in, float* out, const float* w_re, const float* w_im, const float* bias,
                           const float* addend, float* modes, float* mixed, int32_t batch, int32_t width,
                           int32_t n, int32_t nm, void* stream) {
    if (!in || !out || !w_re || !w_im || !modes || !mixed || batch <= 0) {
        set_error("spectral_conv: bad arguments");
        return INC_E_INVALID;
    }
    if (width < 2 || width % 2 != 0 || width > 128) {
        set_error("spectral_conv: width must be even and <= 128 (got %d)", width);
        return INC_E_UNSUPPORTED;
    }
    if (nm < 1 || nm > 32 || nm > n / 2) {
        set_error("spectral_conv: modes must be in [1, min(32, n/2)] (got %d, n=%d)", nm, n);
        return INC_E_UNSUPPORTED;
    }
    float2* mo = reinterpret_cast<float2*>(modes);
    float2* mx = reinterpret_cast<float2*>(mixed);
    cudaStream_t st = as_stream(stream);
    switch (n) {
        case 16: return run_spectral_conv<4, 4, BWD>(in, out, w_re, w_im, bias, addend, mo, mx, batch, width, nm, st);
        case 32: return run_spectral_conv<4, 8, BWD>(in, out, w_re, w_im, bias, addend, mo, mx, batch, width, nm, st);
        case 64: return run_spectral_conv<4, 16, BWD>(in, out, w_re, w_im, bias, addend, mo, mx, batch, width, nm, st);
        case 128: return run_spectral_conv<4, 32, BWD>(in, out, w_re, w_im, bias, addend, mo, mx, batch, width, nm, st);
        case 256: return run_spectral_conv<8, 32, BWD>(in, out, w_re, w_im, bias, addend, mo, mx, batch, width, nm, st);
        case 512:
            return run_spectral_conv<16, 32, BWD>(in, out, w_re, w_im, bias, addend, mo, mx, batch, width, nm, st);
        default:
            set_error("spectral_conv: n must be a power of two in [16, 512] (got %d)", n);
            return INC_E_UNSUPPORTED;
    }
}

}  // namespace ks
}  // namespace inc

extern "C" int inc_spectral_conv1d(const float* x, const float* w_re, const float* w_im, const float* bias,
                                   const float* addend, float* y, float* x_modes, float* work, int32_t batch,
                                   int32_t width, int32_t n, int32_t modes, void* stream) {
    return inc::ks::spectral_conv_dispatch<false>(x, y, w_re, w_im, bias, addend, x_modes, work, batch, width, n,
                                                  modes, stream);
}

extern "C" int inc_spectral_conv1d_bwd(const float* g_y, const float* w_re, const float* w_im, float* g_x,
                                       float* g_modes, float* work, int32_t batch, int32_t width, int32_t n,
                                       int32_t modes, void* stream) {
    return inc::ks::spectral_conv_dispatch<true>(g_y, g_x, w_re, w_im, nullptr, nullptr, g_modes, work, batch, width,
                                                 n, modes, stream);
}
