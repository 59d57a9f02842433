// Energy spectrum of many real rows: |FFT(u)|^2 over the half spectrum with the
// interior bins doubled (analysis/Plot_KS.py:196-235 of tum-pbs/INC), on the
// KS row-pair FFT.  Rows a, b share one complex FFT; the split storage of
// ks_kernels.cuh hands each row its own half spectrum.  Lane twiddles are
// computed in FP64 here, so no plan is needed.
#include "ks_kernels.cuh"

namespace inc {
namespace ks {

template <int P, int T>
__global__ void __launch_bounds__(128) k_spectrum(const float* __restrict__ v, float* __restrict__ out, int rows) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    constexpr int H = N / 2 + 1;
    const int t = threadIdx.x % T;
    Twiddles<P, T> tw;
    tw.sm = nullptr;
    compute_lane_twiddles<P, T>(tw, t);
    const Buf<P, T> buf = group_buf<P, T>(sm + (threadIdx.x / T) * fwd_group_smem<P, T>(), t);
    const int pair = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    const int ra = 2 * pair, rb = 2 * pair + 1 < rows ? 2 * pair + 1 : -1;
    const bool valid = ra < rows;
    float2 x[P];
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int i = t + T * m;
        x[m].x = valid ? __ldg(v + (int64_t)ra * N + i) : 0.f;
        x[m].y = (valid && rb >= 0) ? __ldg(v + (int64_t)rb * N + i) : 0.f;
    }
    fft_fwd<P, T>(x, buf, tw, t);
    to_split<P, T>(x, t, buf.a);
    if (!valid) return;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int k = t + T * m;
        const float2 z = x[m];
        if (k == 0 || k == N / 2) {  // (A, B) real: DC or Nyquist of both rows, not doubled
            out[(int64_t)ra * H + k] = z.x * z.x;
            if (rb >= 0) out[(int64_t)rb * H + k] = z.y * z.y;
        } else if (k < N / 2) {
            out[(int64_t)ra * H + k] = 2.f * (z.x * z.x + z.y * z.y);
        } else if (rb >= 0) {  // B[k] = conj(B[N-k])
            out[(int64_t)rb * H + (N - k)] = 2.f * (z.x * z.x + z.y * z.y);
        }
    }
}

template <int P, int T>
int launch_spectrum(const float* v, float* out, int rows, cudaStream_t st) {
    const int npairs = (rows + 1) / 2;
    const int block = T > 32 ? T : 128;
    const int gpb = block / T;
    const int grid = (npairs + gpb - 1) / gpb;
    const size_t smem = (size_t)gpb * fwd_group_smem<P, T>() * sizeof(float2);
    k_spectrum<P, T><<<grid, block, smem, st>>>(v, out, rows);
    return check_launch("energy_spectrum");
}

// Full complex spectra of real rows for the reference's term methods:
// mode 0: FFT(u), mode 1: FFT(u^2) (calc_nonlinear's transform, solver_1d.py:225-233),
// both unnormalised as torch.fft.fft, out [rows][n] complex (re, im interleaved);
// mode 2: the real part of the unnormalised inverse DFT of complex rows
// (sum_k z_k exp(+2 pi i k j / n)), out [rows][n] real: the adjoint of a real
// row's FFT.  Modes 0/1 pair rows a, b in one complex FFT and unpack each row's
// spectrum from the split storage; mode 2 takes one complex row per group and
// inverts it as swap(FFT(swap(z))).
template <int P, int T>
__global__ void __launch_bounds__(128) k_fft_rows(const float* __restrict__ v, float* __restrict__ out, int rows,
                                                   int mode) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    Twiddles<P, T> tw;
    tw.sm = nullptr;
    compute_lane_twiddles<P, T>(tw, t);
    const Buf<P, T> buf = group_buf<P, T>(sm + (threadIdx.x / T) * fwd_group_smem<P, T>(), t);
    const int grp = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    float2 x[P];
    if (mode == 2) {
        const bool valid = grp < rows;
        const float2* z = reinterpret_cast<const float2*>(v) + (int64_t)(valid ? grp : 0) * N;
#pragma unroll
        for (int m = 0; m < P; ++m) x[m] = valid ? cswap(z[t + T * m]) : make_float2(0.f, 0.f);
        fft_fwd<P, T>(x, buf, tw, t);
        if (!valid) return;
#pragma unroll
        for (int m = 0; m < P; ++m) out[(int64_t)grp * N + t + T * m] = x[m].y;  // real part of swap(.)
        return;
    }
    const int ra = 2 * grp, rb = 2 * grp + 1 < rows ? 2 * grp + 1 : -1;
    const bool valid = ra < rows;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int i = t + T * m;
        const float a = valid ? __ldg(v + (int64_t)ra * N + i) : 0.f;
        const float b = (valid && rb >= 0) ? __ldg(v + (int64_t)rb * N + i) : 0.f;
        x[m] = mode == 1 ? make_float2(a * a, b * b) : make_float2(a, b);
    }
    fft_fwd<P, T>(x, buf, tw, t);
    to_split<P, T>(x, t, buf.a);
    if (!valid) return;
    float2* oa = reinterpret_cast<float2*>(out) + (int64_t)ra * N;
    float2* ob = reinterpret_cast<float2*>(out) + (int64_t)(rb >= 0 ? rb : ra) * N;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int k = t + T * m;
        const float2 z = x[m];
        if (k == 0 || k == N / 2) {  // (A, B) real at DC and Nyquist
            oa[k] = make_float2(z.x, 0.f);
            if (rb >= 0) ob[k] = make_float2(z.y, 0.f);
        } else if (k < N / 2) {      // A[k]; A[N-k] = conj(A[k])
            oa[k] = z;
            oa[N - k] = make_float2(z.x, -z.y);
        } else if (rb >= 0) {        // B[k]; B[N-k] = conj(B[k])
            ob[k] = z;
            ob[N - k] = make_float2(z.x, -z.y);
        }
    }
}

template <int P, int T>
int launch_fft_rows(const float* v, float* out, int rows, int mode, cudaStream_t st) {
    const int groups = mode == 2 ? rows : (rows + 1) / 2;
    const int block = T > 32 ? T : 128;
    const int gpb = block / T;
    const int grid = (groups + gpb - 1) / gpb;
    const size_t smem = (size_t)gpb * fwd_group_smem<P, T>() * sizeof(float2);
    k_fft_rows<P, T><<<grid, block, smem, st>>>(v, out, rows, mode);
    return check_launch("ks_fft_rows");
}

}  // namespace ks
}  // namespace inc

extern "C" int inc_ks_fft_rows(const float* v, float* out, int32_t rows, int32_t n, int32_t mode, void* stream) {
    using namespace inc;
    using namespace inc::ks;
    if (!v || !out || rows <= 0 || mode < 0 || mode > 2) { set_error("ks_fft_rows: bad arguments"); return INC_E_INVALID; }
    if ((reinterpret_cast<uintptr_t>(out) & 7u) || (mode == 2 && (reinterpret_cast<uintptr_t>(v) & 7u))) {
        set_error("ks_fft_rows: complex arrays must be 8-byte aligned");
        return INC_E_INVALID;
    }
    cudaStream_t st = as_stream(stream);
    switch (n) {
        case 16: return launch_fft_rows<4, 4>(v, out, rows, mode, st);
        case 32: return launch_fft_rows<4, 8>(v, out, rows, mode, st);
        case 64: return launch_fft_rows<4, 16>(v, out, rows, mode, st);
        case 128: return launch_fft_rows<4, 32>(v, out, rows, mode, st);
        case 256: return launch_fft_rows<8, 32>(v, out, rows, mode, st);
        case 512: return launch_fft_rows<8, 64>(v, out, rows, mode, st);
        default:
            set_error("ks_fft_rows: n must be a power of two in [16, 512] (got %d)", n);
            return INC_E_UNSUPPORTED;
    }
}

extern "C" int inc_energy_spectrum(const float* v, float* out, int32_t rows, int32_t n, void* stream) {
    using namespace inc;
    using namespace inc::ks;
    if (!v || !out || rows <= 0) { set_error("energy_spectrum: bad arguments"); return INC_E_INVALID; }
    cudaStream_t st = as_stream(stream);
    switch (n) {
        case 16: return launch_spectrum<4, 4>(v, out, rows, st);
        case 32: return launch_spectrum<4, 8>(v, out, rows, st);
        case 64: return launch_spectrum<4, 16>(v, out, rows, st);
        case 128: return launch_spectrum<4, 32>(v, out, rows, st);
        case 256: return launch_spectrum<8, 32>(v, out, rows, st);
        case 512: return launch_spectrum<8, 64>(v, out, rows, st);
        default:
            set_error("energy_spectrum: n must be a power of two in [16, 512] (got %d)", n);
            return INC_E_UNSUPPORTED;
    }
}
