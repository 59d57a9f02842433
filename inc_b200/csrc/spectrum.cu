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

}  // namespace ks
}  // namespace inc

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
