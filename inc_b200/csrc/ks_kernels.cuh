// Kuramoto-Sivashinsky pseudo-spectral ETRK2 / ETD1 stepper for sm_100a.
//
// Two rows a, b share one complex FFT of length N: z = u_a + i u_b.  A row pair
// is owned by a group of T lanes (T <= 64; a group wider than a warp syncs on the CTA barrier); lane t holds the
// P = N/T values z[t + T*m] in register m, for physical and spectral data
// alike.  An FFT is a P-point DFT in registers followed by Stockham passes
// of radix <= P, each reading the previous pass's output through a padded
// shared-memory buffer, with FP64-derived twiddles.  Every operator of the step is a
// Fourier multiplier or a pointwise product, so the whole step (both
// substeps) runs in registers with four FFTs per substep.
//
// Spectral storage: "packed" (the FFT of z) when both rows of a pair have the
// same domain size; otherwise "split": slot k < N/2 holds row a's spectrum
// A[k], slot k > N/2 holds row b's B[k], slots 0 and N/2 hold (A, B) as
// (re, im).  Converting costs one mirror exchange (k <-> N-k) by shuffles.
// Spectra are stored scaled by 1/N so the inverse FFT needs no scaling.
//
// Reference (tum-pbs/INC solvers/solver_1d.py): calc_nonlinear :225-233,
// calc_linear :235-240, etd1_step :242-255, etrk2_step :257-278,
// etd1/etrk2 (double step, correction_u) :280-288.  The derivative multiplier
// is zero at the Nyquist bin: the reference's value there is purely imaginary
// and is discarded by ifft(.).real, so the two are the same map.
#pragma once
#include <utility>

#include "common.cuh"

namespace inc {
namespace ks {

// Compile-time loop: f(std::integral_constant<int, i>) for i in [0, N), so
// that indices derived from i are constant expressions (shared-memory offsets).
template <typename F, int... I>
INC_DEV void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
INC_DEV void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// ---- complex helpers ---------------------------------------------------------
INC_DEV float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
INC_DEV float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
INC_DEV float2 cmul(float2 a, float2 b) { return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x)); }
INC_DEV float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
INC_DEV float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// cos(2*pi*m/32), sin(2*pi*m/32) for m in [0, 16), rounded from FP64.
INC_DEV float cos32(int m) {
    switch (m) {
        case 0: return 1.0f;
        case 1: return 0.9807852506637573f;
        case 2: return 0.9238795042037964f;
        case 3: return 0.8314695954322815f;
        case 4: return 0.7071067690849304f;
        case 5: return 0.5555702447891235f;
        case 6: return 0.3826834261417389f;
        case 7: return 0.19509032368659973f;
        case 8: return 0.0f;
        case 9: return -0.19509032368659973f;
        case 10: return -0.3826834261417389f;
        case 11: return -0.5555702447891235f;
        case 12: return -0.7071067690849304f;
        case 13: return -0.8314695954322815f;
        case 14: return -0.9238795042037964f;
        default: return -0.9807852506637573f;
    }
}
INC_DEV float sin32(int m) {
    switch (m) {
        case 0: return 0.0f;
        case 1: return 0.19509032368659973f;
        case 2: return 0.3826834261417389f;
        case 3: return 0.5555702447891235f;
        case 4: return 0.7071067690849304f;
        case 5: return 0.8314695954322815f;
        case 6: return 0.9238795042037964f;
        case 7: return 0.9807852506637573f;
        case 8: return 1.0f;
        case 9: return 0.9807852506637573f;
        case 10: return 0.9238795042037964f;
        case 11: return 0.8314695954322815f;
        case 12: return 0.7071067690849304f;
        case 13: return 0.5555702447891235f;
        case 14: return 0.3826834261417389f;
        default: return 0.19509032368659973f;
    }
}

// a + w b and a - w b in six FMAs (the difference as 2a - (a + w b)).
INC_DEV void bfly_w(float2 a, float2 b, float2 w, float2& s, float2& d) {
    s.x = fmaf(w.x, b.x, fmaf(-w.y, b.y, a.x));
    s.y = fmaf(w.x, b.y, fmaf(w.y, b.x, a.y));
    d.x = fmaf(2.f, a.x, -s.x);
    d.y = fmaf(2.f, a.y, -s.y);
}

// a +- b * exp(-+ 2 pi i m / 32) (forward: minus, inverse: plus).  m = 0 and
// m = 8 need no multiply; m = 4, 12 scale a sum of +-b.x, +-b.y by cos(pi/4).
template <bool INV>
INC_DEV void bfly_rot32(float2 a, float2 b, int m, float2& s, float2& d) {
    if (m == 0) {
        s = cadd(a, b);
        d = csub(a, b);
        return;
    }
    if (m == 8) {
        const float2 r = INV ? make_float2(-b.y, b.x) : make_float2(b.y, -b.x);
        s = cadd(a, r);
        d = csub(a, r);
        return;
    }
    const float c = cos32(m), sn = INV ? sin32(m) : -sin32(m);
    if (m == 4 || m == 12) {
        const float k = cos32(4);
        const float cs = c > 0.f ? 1.f : -1.f, ss = sn > 0.f ? 1.f : -1.f;
        const float tr = cs * b.x - ss * b.y, ti = ss * b.x + cs * b.y;
        s = make_float2(fmaf(k, tr, a.x), fmaf(k, ti, a.y));
        d = make_float2(fmaf(-k, tr, a.x), fmaf(-k, ti, a.y));
        return;
    }
    bfly_w(a, b, make_float2(c, sn), s, d);
}

// In-register DFT of P <= 32 points, natural order in and out: radix-2
// Stockham autosort (every index is arithmetic on unrolled loop counters, so
// the whole transform stays in registers), from the stage of span NS0 on.
template <int P, bool INV, int NS0 = 1>
INC_DEV void dft_reg(float2 (&v)[P]) {
#pragma unroll
    for (int ns = NS0; ns < P; ns *= 2) {
        float2 w[P];
#pragma unroll
        for (int j = 0; j < P / 2; ++j) {
            const int k = j % ns;
            const int idx = (j / ns) * ns * 2 + k;
            bfly_rot32<INV>(v[j], v[j + P / 2], k * (16 / ns), w[idx], w[idx + ns]);
        }
#pragma unroll
        for (int i = 0; i < P; ++i) v[i] = w[i];
    }
}

// R-point forward DFT of tw[r] * y[r] (tw[0] = 1, not read): the twiddles of
// the first stage's second operands are applied inside its butterflies.
template <int R>
INC_DEV void dft_tw(float2 (&y)[R], const float2 (&tw)[R]) {
    float2 w[R];
#pragma unroll
    for (int j = 0; j < R / 2; ++j) {
        const float2 a = j == 0 ? y[0] : cmul(y[j], tw[j]);
        bfly_w(a, y[j + R / 2], tw[j + R / 2], w[2 * j], w[2 * j + 1]);
    }
#pragma unroll
    for (int i = 0; i < R; ++i) y[i] = w[i];
    dft_reg<R, false, 2>(y);
}

// ---- FFT -------------------------------------------------------------------------
// Length-N (= P*T) FFT of a row pair held as z[t + T*m] in v[m] (same layout
// out), as Stockham passes: pass 1 is a P-point DFT in registers; every later
// pass (span NS, radix R = min(P, N/NS), P/R butterflies per lane) reads the
// previous pass's output from shared memory, applies its twiddles, runs R-point
// DFTs in registers and writes the next buffer -- or, in the last pass, the
// registers.  Two buffers per group alternate, so one barrier per pass
// suffices.  Shared indices are padded by one slot per 16 (padx), which
// spreads the strided accesses over the banks and keeps every address a
// per-lane base plus a compile-time constant.
INC_DEV constexpr int pass_radix(int P, int T, int ns) { return P < (P * T) / ns ? P : (P * T) / ns; }
INC_DEV constexpr int num_later_passes(int P, int T) {
    int n = 0;
    for (int ns = P; ns < P * T; ns *= pass_radix(P, T, ns)) ++n;
    return n;
}
// index of the later pass with span ns (0 for the first later pass)
INC_DEV constexpr int pass_index(int P, int T, int ns) {
    int i = 0;
    for (int x = P; x < ns; x *= pass_radix(P, T, x)) ++i;
    return i;
}
// twiddles one lane applies in all later passes, and before the pass with span ns
INC_DEV constexpr int lane_twiddles(int P, int T) {
    int c = 0;
    for (int ns = P; ns < P * T; ns *= pass_radix(P, T, ns)) c += (P / pass_radix(P, T, ns)) * (pass_radix(P, T, ns) - 1);
    return c;
}
INC_DEV constexpr int lane_twiddle_offset(int P, int T, int ns) {
    int c = 0;
    for (int x = P; x < ns; x *= pass_radix(P, T, x)) c += (P / pass_radix(P, T, x)) * (pass_radix(P, T, x) - 1);
    return c;
}
// a lane keeps its twiddles in registers when it needs at most 16
template <int P, int T>
INC_DEV constexpr bool twiddles_in_registers() { return lane_twiddles(P, T) <= 16; }
template <int P, int T>
INC_DEV constexpr int reg_twiddles() { return twiddles_in_registers<P, T>() ? lane_twiddles(P, T) : 1; }

// Shared-memory layout of the exchanges.  Exchange e is the buffer written by
// the pass with span ex_span(e) (e = 0: the register pass) and read by the
// next pass.  Each exchange has its own linear map lay(e, i) = sum of
// weight(e, j) over the set bits j of the logical index i: the weights are
// superincreasing (so the map is injective) and, modulo the 16 float2 banks,
// send the index bits that vary across the lanes of a half-warp to distinct
// bank bits for both the write pattern and the read pattern of that exchange.
// Every access is then conflict-free, and because the map is additive over
// disjoint bits, every address is a per-lane base plus a compile-time constant.
// Groups narrower than 16 lanes share a half-warp; their stride supplies the
// remaining bank bits (group_stride).
INC_DEV constexpr int ilog2(int x) {
    int r = 0;
    while ((2 << r) <= x) ++r;
    return r;
}
INC_DEV constexpr int ex_span(int P, int T, int e) {
    int ns = 1, R = P;
    for (int k = 0; k < e; ++k) { ns *= R; R = pass_radix(P, T, ns); }
    return ns;
}
INC_DEV constexpr int ex_radix(int P, int T, int e) {
    int ns = 1, R = P;
    for (int k = 0; k < e; ++k) { ns *= R; R = pass_radix(P, T, ns); }
    return R;
}
// lane-varying bits of one half-warp: 4, or log2(T) for narrower groups
INC_DEV constexpr int lane_bits(int T) { return T >= 16 ? 4 : ilog2(T); }
// bank weight (a power of two, or 0) of index bit j in exchange e
INC_DEV constexpr int lay_bank(int P, int T, int e, int j) {
    const int lgNS = ilog2(ex_span(P, T, e)), lgR = ilog2(ex_radix(P, T, e)), nb = lane_bits(T);
    int sw = 0;  // index bits the write pattern varies across a half-warp
    for (int b = 0; b < nb; ++b) sw |= 1 << (b < lgNS ? b : b + lgR);
    if (j < nb) return 1 << j;  // the read pattern varies bits [0, nb)
    if (!((sw >> j) & 1)) return 0;
    int used = sw & ((1 << nb) - 1);
    for (int k = nb; k <= j; ++k) {
        if (!((sw >> k) & 1)) continue;
        int nx = 0;
        while ((used >> nx) & 1) ++nx;
        if (k == j) return 1 << nx;
        used |= 1 << nx;
    }
    return 0;
}
INC_DEV constexpr int lay_weight(int P, int T, int e, int j) {
    int sum = 0, w = 0;
    for (int k = 0; k <= j; ++k) {
        const int base = (1 << k) > sum + 1 ? (1 << k) : sum + 1;
        w = base + (((lay_bank(P, T, e, k) - base) % 16) + 16) % 16;
        sum += w;
    }
    return w;
}
INC_DEV constexpr int lay(int P, int T, int e, int i) {
    int out = 0;
    for (int j = 0; (1 << j) < P * T; ++j)
        if ((i >> j) & 1) out += lay_weight(P, T, e, j);
    return out;
}
// written index of the lane-dependent part j of a pass with span ns, radix R
INC_DEV constexpr int spread(int j, int ns, int R) { return (j / ns) * ns * R + j % ns; }
INC_DEV constexpr int num_exchanges(int P, int T) { return num_later_passes(P, T); }
template <int P, int T>
INC_DEV constexpr int buf_len() {
    int len = P * T;  // buffer a doubles as the mirror scratch
    for (int e = 0; e < num_exchanges(P, T); ++e) {
        const int l = lay(P, T, e, P * T - 1) + 1;
        len = l > len ? l : len;
    }
    return len;
}
// per-group shared size rounded so that groups of one half-warp land on distinct bank bits
template <int T>
INC_DEV constexpr int group_stride(int size) {
    const int r = T >= 16 ? 0 : (1 << ilog2(T)) % 16;
    int s = size;
    while (s % 16 != r) ++s;
    return s;
}

template <int T>
INC_DEV void group_sync() {
    if constexpr (T <= 32) __syncwarp();
    else __syncthreads();
}

// A group's two exchange buffers and this lane's bases in them: w[e] where
// the pass writing exchange e stores, r[e] where the next pass loads.
template <int P, int T>
struct Buf {
    static constexpr int NE = num_exchanges(P, T) > 0 ? num_exchanges(P, T) : 1;
    float2* a;
    float2* b;
    float2* w[NE];
    const float2* r[NE];
};

template <int P, int T, int E>
INC_DEV int lay_rt(int i) {
    int out = 0;
    static_for<ilog2(P * T)>([&](auto jc) {
        constexpr int j = decltype(jc)::value;
        constexpr int w = lay_weight(P, T, E, j);
        out += ((i >> j) & 1) * w;
    });
    return out;
}

template <int P, int T, int E>
INC_DEV void set_lane_bases(Buf<P, T>& b, int t) {
    if constexpr (E < num_exchanges(P, T)) {
        float2* base = (E % 2) ? b.b : b.a;
        b.w[E] = base + lay_rt<P, T, E>(spread(t, ex_span(P, T, E), ex_radix(P, T, E)));
        b.r[E] = base + lay_rt<P, T, E>(t);
        set_lane_bases<P, T, E + 1>(b, t);
    }
}

// Twiddles of the later passes: in registers (reg) or in the shared table (sm).
template <int P, int T>
struct Twiddles {
    float2 reg[reg_twiddles<P, T>()];
    const float2* sm;
};

template <int P, int T>
INC_DEV void load_lane_twiddles(Twiddles<P, T>& tw, const float2* table, int t) {
    constexpr int N = P * T;
    if constexpr (twiddles_in_registers<P, T>()) {
        int i = 0;
#pragma unroll
        for (int ns = P; ns < N; ns *= pass_radix(P, T, ns)) {
            const int R = pass_radix(P, T, ns), Q = P / R, pi = pass_index(P, T, ns);
#pragma unroll
            for (int q = 0; q < Q; ++q)
#pragma unroll
                for (int r = 1; r < R; ++r) tw.reg[i++] = __ldg(table + pi * N + (q * R + r) * T + t);
        }
    }
}

// The same lane twiddles computed in FP64 on the device (kernels without a plan).
template <int P, int T>
INC_DEV void compute_lane_twiddles(Twiddles<P, T>& tw, int t) {
    static_assert(twiddles_in_registers<P, T>(), "shapes with lane twiddles in registers");
    constexpr int N = P * T;
    int i = 0;
#pragma unroll
    for (int ns = P; ns < N; ns *= pass_radix(P, T, ns)) {
        const int R = pass_radix(P, T, ns), Q = P / R;
#pragma unroll
        for (int q = 0; q < Q; ++q)
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const int k = (t + T * q) % ns;
                double sn, cs;
                sincospi(-2.0 * (double)(r * k) / (double)(ns * R), &sn, &cs);
                tw.reg[i++] = make_float2((float)cs, (float)sn);
            }
    }
}

// The later passes' twiddle table (entry pi*N + (q*R + r)*T + t =
// exp(-2 pi i r k / (NS R)), k = (t + T q) % NS) computed in FP64 by the block
// into shared memory, for kernels without a plan whose shape does not keep
// the lane twiddles in registers.  The caller synchronises before use.
template <int P, int T>
INC_DEV void fill_twiddle_table(float2* table) {
    constexpr int N = P * T;
    int pi = 0;
    for (int ns = P; ns < N; ns *= pass_radix(P, T, ns), ++pi) {
        const int R = pass_radix(P, T, ns), Q = P / R;
        for (int i = threadIdx.x; i < Q * R * T; i += blockDim.x) {
            const int t = i % T, r = (i / T) % R, q = i / (T * R);
            const int k = (t + T * q) % ns;
            double sn, cs;
            sincospi(-2.0 * (double)(r * k) / (double)(ns * R), &sn, &cs);
            table[pi * N + i] = make_float2((float)cs, (float)sn);
        }
    }
}

template <int P, int T, int NS>
INC_DEV void fft_later(float2 (&v)[P], const Buf<P, T>& buf, const Twiddles<P, T>& tw, int t) {
    constexpr int N = P * T;
    if constexpr (NS < N) {
        constexpr int R = pass_radix(P, T, NS);
        constexpr int Q = P / R;
        constexpr bool LAST = NS * R == N;
        constexpr int TOFF = lane_twiddle_offset(P, T, NS);
        constexpr int E = pass_index(P, T, NS);  // the exchange this pass reads
        const float2* twp = tw.sm + E * N;
        group_sync<T>();
        static_for<Q>([&](auto qc) {
            constexpr int q = decltype(qc)::value;
            float2 w[R], twv[R];
            static_for<R>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                constexpr int off = lay(P, T, E, T * q + r * (N / R));
                w[r] = buf.r[E][off];
                if constexpr (r > 0) {
                    if constexpr (twiddles_in_registers<P, T>()) twv[r] = tw.reg[TOFF + q * (R - 1) + r - 1];
                    else twv[r] = twp[(q * R + r) * T + t];
                } else {
                    twv[r] = make_float2(1.f, 0.f);
                }
            });
            if constexpr (P >= 8) {
                dft_tw<R>(w, twv);
            } else {  // four values per lane: separate twiddle products keep the chains short
#pragma unroll
                for (int r = 1; r < R; ++r) w[r] = cmul(w[r], twv[r]);
                dft_reg<R, false>(w);
            }
            if constexpr (LAST) {
#pragma unroll
                for (int r = 0; r < R; ++r) v[q + Q * r] = w[r];
            } else {
                static_for<R>([&](auto rc) {
                    constexpr int r = decltype(rc)::value;
                    constexpr int off = lay(P, T, E + 1, spread(T * q, NS, R) + r * NS);
                    buf.w[E + 1][off] = w[r];
                });
            }
        });
        if constexpr (!LAST) fft_later<P, T, NS * R>(v, buf, tw, t);
    }
}

// Unnormalised forward DFT of the group's row pair, natural order in and out.
template <int P, int T>
INC_DEV void fft_fwd(float2 (&v)[P], const Buf<P, T>& buf, const Twiddles<P, T>& tw, int t) {
    dft_reg<P, false>(v);
    // With an odd number of exchanges the previous transform's last pass read
    // buffer a, which this one writes first; with an even number a was last
    // read before that pass's barrier.
    if constexpr (num_exchanges(P, T) % 2 == 1 || num_exchanges(P, T) == 0) group_sync<T>();
    if constexpr (num_exchanges(P, T) > 0) {
        static_for<P>([&](auto rc) {
            constexpr int r = decltype(rc)::value;
            constexpr int off = lay(P, T, 0, r);
            buf.w[0][off] = v[r];
        });
        fft_later<P, T, P>(v, buf, tw, t);
    }
}

// (re, im) -> (im, re): the unnormalised inverse DFT is swap(FFT(swap(v))).
INC_DEV float2 cswap(float2 z) { return make_float2(z.y, z.x); }

template <int P, int T>
INC_DEV void fft_inv(float2 (&v)[P], const Buf<P, T>& buf, const Twiddles<P, T>& tw, int t) {
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);
    fft_fwd<P, T>(v, buf, tw, t);
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);
}

// ---- mirror exchange: slot k <-> slot N-k --------------------------------------
// Slot k = t + T*m.  Its mirror lives in lane (T-t)%T, register P-1-m (t != 0)
// or in lane 0, register (P-m)%P (t == 0).
// A group wider than a warp exchanges through `scratch` (N float2 of the
// group's shared memory, free between transforms).
template <int P, int T>
INC_DEV void mirror(const float2 (&v)[P], float2 (&mv)[P], int t, float2* scratch) {
    if constexpr (T <= 32) {
        float2 recv[P];
        const int partner = (T - t) & (T - 1);
#pragma unroll
        for (int m = 0; m < P; ++m) {
            recv[m].x = shfl<T>(v[m].x, partner);
            recv[m].y = shfl<T>(v[m].y, partner);
        }
#pragma unroll
        for (int m = 0; m < P; ++m) mv[m] = (t != 0) ? recv[P - 1 - m] : v[(P - m) % P];
    } else {
        constexpr int N = P * T;
        group_sync<T>();
#pragma unroll
        for (int m = 0; m < P; ++m) scratch[t + T * m] = v[m];
        group_sync<T>();
#pragma unroll
        for (int m = 0; m < P; ++m) mv[m] = scratch[(N - (t + T * m)) & (N - 1)];
        group_sync<T>();  // the scratch is exchange buffer a, which the next transform may write first
    }
}

// packed Z = FFT(a + i b)  ->  split (A in the lower half, B in the upper half)
template <int P, int T>
INC_DEV void to_split(float2 (&v)[P], int t, float2* scratch) {
    constexpr int N = P * T;
    float2 mv[P];
    mirror<P, T>(v, mv, t, scratch);
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int k = t + T * m;
        const float2 z = v[m], zm = mv[m];
        if (k == 0 || k == N / 2) continue;
        if (k < N / 2) v[m] = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
        else v[m] = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
    }
}

template <int P, int T>
INC_DEV void to_packed(float2 (&v)[P], int t, float2* scratch) {
    constexpr int N = P * T;
    float2 mv[P];
    mirror<P, T>(v, mv, t, scratch);
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int k = t + T * m;
        const float2 s = v[m], sm = mv[m];
        if (k == 0 || k == N / 2) continue;
        if (k < N / 2) v[m] = make_float2(s.x + sm.y, s.y + sm.x);
        else v[m] = make_float2(sm.x - s.y, s.x - sm.y);
    }
}

// ---- arguments ---------------------------------------------------------------
struct Args {
    const float* u;
    const float* s;
    const float* cu;
    float* out;
    const float* g_out;
    float* g_u;
    float* g_s;
    float* frames;
    float* ckpts;
    const float* g_frames;
    const float* g_final;
    const int* pairs;     // [npairs][2], second = -1 for a lone row
    const float* dR;      // [rows] pi / L
    const float* coef;    // [rows][3][nhp]: exp(L dt), phi1, phi2
    const float2* tw;     // [N] FFT twiddles (layout of fft())
    float2* stage;        // rollout backward scratch: per launched group [ckpt_every][3][N] (or null)
    float2* tape;         // rollout tape: per row pair [steps][4][N], lane layout (or null)
    int rows, n, npairs, scheme, split, dealias, steps, ckpt_every, nhp;
    int substeps;         // k_step / k_step_bwd: 1 = one substep (etd1_step / etrk2_step), else a step()
    float invN;
};

// Per-lane context of one row pair.
struct Ctx {
    int ra, rb;      // rows (rb = -1: lone row)
    int rbc;         // row whose coefficients the upper half uses
    int t;
    bool valid;
    float dRa, dRb;  // pi / L of each row
};

INC_DEV void make_ctx(const Args& a, int pair, int t, bool valid, Ctx& c) {
    c.t = t;
    c.valid = valid;
    const int p = valid ? pair : 0;
    c.ra = __ldg(a.pairs + 2 * p);
    c.rb = valid ? __ldg(a.pairs + 2 * p + 1) : -1;
    c.rbc = c.rb >= 0 ? c.rb : c.ra;
    c.dRa = __ldg(a.dR + c.ra);
    c.dRb = __ldg(a.dR + c.rbc);
}

// Multipliers of slot k = t + T*m.  `sp` marks slots 0 and N/2 in split
// storage, whose .x belongs to row a and .y to row b (real multipliers there).
struct Slot {
    float E, p1, p2, d;  // d: derivative multiplier is -i*d (unscaled)
    float dn;            // d / N
    float Eb, p1b, p2b;
    bool sp;
};

template <int P, int T>
INC_DEV Slot slot(const Args& a, const Ctx& c, int m, bool need_p2) {
    constexpr int N = P * T;
    const int k = c.t + T * m;
    const bool up = k > N / 2;
    const int kk = up ? N - k : k;
    const int row = (a.split && up) ? c.rbc : c.ra;
    const float* cr = a.coef + (int64_t)row * 3 * a.nhp;
    Slot s;
    s.E = __ldg(cr + kk);
    s.p1 = __ldg(cr + a.nhp + kk);
    s.p2 = need_p2 ? __ldg(cr + 2 * a.nhp + kk) : 0.f;
    int f = (k < N / 2) ? k : (k == N / 2 ? 0 : k - N);
    if (a.dealias && 3 * abs(f) > N) f = 0;
    s.d = (float)f * ((a.split && up) ? c.dRb : c.dRa);
    s.dn = s.d * a.invN;
    s.sp = a.split && (k == 0 || k == N / 2);
    if (s.sp) {
        const float* cb = a.coef + (int64_t)c.rbc * 3 * a.nhp;
        s.Eb = __ldg(cb + kk);
        s.p1b = __ldg(cb + a.nhp + kk);
        s.p2b = need_p2 ? __ldg(cb + 2 * a.nhp + kk) : 0.f;
    } else {
        s.Eb = s.E; s.p1b = s.p1; s.p2b = s.p2;
    }
    return s;
}

// The multipliers of this lane's P slots, read once per launch and kept in
// registers (P <= 8); larger lanes re-read them (L1-resident) per stage.
template <int P, int T>
struct SlotCache {
    static constexpr bool ON = P <= 8;
    static constexpr int M = ON ? P : 1;
    float E[M], p1[M], p2[M], d[M], dn[M];
    float Eb[2], p1b[2], p2b[2];  // row b at slots 0 and N/2 (split storage)

    INC_DEV void load(const Args& a, const Ctx& c) {
        if constexpr (ON) {
#pragma unroll
            for (int m = 0; m < P; ++m) {
                const Slot s = slot<P, T>(a, c, m, a.scheme == INC_KS_ETRK2);  // phi2 = 0 for ETD1
                E[m] = s.E; p1[m] = s.p1; p2[m] = s.p2; d[m] = s.d; dn[m] = s.dn;
                if (m == 0 || m == P / 2) {
                    const int i = m == 0 ? 0 : 1;
                    Eb[i] = s.Eb; p1b[i] = s.p1b; p2b[i] = s.p2b;
                }
            }
        }
    }

    INC_DEV Slot get(const Args& a, const Ctx& c, int m, bool need_p2) const {
        if constexpr (ON) {
            Slot s;
            s.E = E[m]; s.p1 = p1[m]; s.p2 = p2[m]; s.d = d[m]; s.dn = dn[m];
            if (m == 0 || m == P / 2) {
                const int i = m == 0 ? 0 : 1;
                s.Eb = Eb[i]; s.p1b = p1b[i]; s.p2b = p2b[i];
            } else {
                s.Eb = s.E; s.p1b = s.p1; s.p2b = s.p2;
            }
            s.sp = false;
            return s;
        } else {
            return slot<P, T>(a, c, m, need_p2);
        }
    }
};

// real multiplier (row a on .x, row b on .y at the special slots)
INC_DEV float2 rmul(float2 z, float ma, float mb) { return make_float2(ma * z.x, mb * z.y); }
// -i * d * z
INC_DEV float2 dmul(float2 z, float d) { return make_float2(d * z.y, -d * z.x); }

// ---- loads / stores of a row pair in the lane layout ----------------------------
template <int P, int T>
INC_DEV void load_pair(float2 (&x)[P], const float* __restrict__ src, const Ctx& c, int n) {
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int i = c.t + T * m;
        x[m].x = c.valid ? __ldg(src + (int64_t)c.ra * n + i) : 0.f;
        x[m].y = (c.valid && c.rb >= 0) ? __ldg(src + (int64_t)c.rb * n + i) : 0.f;
    }
}

template <int P, int T>
INC_DEV void add_pair(float2 (&x)[P], const float* __restrict__ src, const Ctx& c, int n) {
    float2 y[P];
    load_pair<P, T>(y, src, c, n);
#pragma unroll
    for (int m = 0; m < P; ++m) x[m] = cadd(x[m], y[m]);
}

template <int P, int T>
INC_DEV void store_pair(float* __restrict__ dst, const float2 (&x)[P], const Ctx& c, int n) {
    if (!c.valid) return;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int i = c.t + T * m;
        dst[(int64_t)c.ra * n + i] = x[m].x;
        if (c.rb >= 0) dst[(int64_t)c.rb * n + i] = x[m].y;
    }
}

// Row-strided variant for [rows][steps][n] frames / [rows][nseg][n] checkpoints.
template <int P, int T>
INC_DEV void store_pair_strided(float* __restrict__ dst, const float2 (&x)[P], const Ctx& c, int n,
                                int64_t row_stride, int64_t off) {
    if (!c.valid) return;
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int i = c.t + T * m;
        __stcs(dst + (int64_t)c.ra * row_stride + off + i, x[m].x);
        if (c.rb >= 0) __stcs(dst + (int64_t)c.rb * row_stride + off + i, x[m].y);
    }
}

template <int P, int T>
INC_DEV void load_pair_strided(float2 (&x)[P], const float* __restrict__ src, const Ctx& c, int n,
                               int64_t row_stride, int64_t off) {
#pragma unroll
    for (int m = 0; m < P; ++m) {
        const int i = c.t + T * m;
        x[m].x = c.valid ? __ldg(src + (int64_t)c.ra * row_stride + off + i) : 0.f;
        x[m].y = (c.valid && c.rb >= 0) ? __ldg(src + (int64_t)c.rb * row_stride + off + i) : 0.f;
    }
}

INC_DEV float2 sq2(float2 x) { return make_float2(x.x * x.x, x.y * x.y); }

// ---- shared memory ----------------------------------------------------------------
// Per CTA: the twiddle table of the later passes ((passes-1) * N float2), then
// per group its two exchange buffers and, for the backward kernels, state slots.
template <int P, int T>
INC_DEV constexpr int tw_size() { return twiddles_in_registers<P, T>() ? 0 : num_later_passes(P, T) * P * T; }
// Per group: the two exchange buffers, then (backward kernels) state slots.
template <int P, int T>
INC_DEV constexpr int fwd_group_smem() { return group_stride<T>(2 * buf_len<P, T>()); }
template <int P, int T>
INC_DEV constexpr int bwd_group_smem(int K) { return group_stride<T>(2 * buf_len<P, T>() + (5 + K) * P * T); }

template <int P, int T>
INC_DEV float2* group_smem(float2* sm, int per_group) {
    return sm + tw_size<P, T>() + (threadIdx.x / T) * per_group;
}

template <int P, int T>
INC_DEV Buf<P, T> group_buf(float2* g, int t) {
    Buf<P, T> b;
    b.a = g;
    b.b = g + buf_len<P, T>();
    set_lane_bases<P, T, 0>(b, t);
    return b;
}

// The block's shared twiddle table (when lanes do not hold them in registers)
// and this lane's register twiddles.
template <int P, int T>
INC_DEV Twiddles<P, T> setup_twiddles(const Args& a, float2* sm, int t) {
    for (int i = threadIdx.x; i < tw_size<P, T>(); i += blockDim.x) sm[i] = a.tw[i];
    __syncthreads();
    Twiddles<P, T> tw;
    tw.sm = sm;
    load_lane_twiddles<P, T>(tw, a.tw, t);
    return tw;
}

// ---- the forward program ------------------------------------------------------------
// A rollout is a prologue ([FFT(s)], FFT(u)) and then a loop of half-substeps,
// each FFT(x^2) -> stage multiplier -> IFFT -> x: stage 1 then stage 2 per
// ETRK2 substep (stage 1 alone for ETD1), two substeps per step() call.  The
// loop body holds the two transforms of one half-substep, so the phase of the
// program is one bit (the stage) and a step counter.
template <int P, int T>
INC_DEV void st_put(float2* st, const float2 (&v)[P], int t) {
#pragma unroll
    for (int m = 0; m < P; ++m) st[m * T + t] = v[m];
}
template <int P, int T>
INC_DEV void st_get(float2 (&v)[P], const float2* st, int t) {
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = st[m * T + t];
}

// seg (optional): shared memory receiving the state at the start of every step,
// in lane layout [step][m][t] (the backward replay).  ckpt_on: store checkpoints.
// stg (optional, the backward replay): receives the physical states after a
// step's first three half-substeps (ETRK2: xi1, x1, xi2; ETD1: x1 after the
// first), in lane layout [step][3][m][t]; tail_skip half-substeps are left out
// at the end (the last step's states are needed, its result is not).
// tape (optional, the tape rollout): receives per step [4][m][t] the step's start
// state and its states after the first three half-substeps (ETD1: start state and
// the state between its substeps), by streaming stores.
template <int P, int T>
INC_DEV void tape_put(float2* dst, const float2 (&v)[P], int t) {
#pragma unroll
    for (int m = 0; m < P; ++m) __stcs(dst + m * T + t, v[m]);
}

// FAST = 1: the common case compiled alone (ETRK2, both rows of every pair with one
// domain size, so packed spectra): no scheme or storage branches in the loop body,
// which is then smaller (instruction cache) and straight-line.
template <int P, int T, int FAST = 0>
INC_DEV void forward_program(const Args& a, const Ctx& c, float2 (&x)[P], int steps, const Buf<P, T>& buf,
                             const Twiddles<P, T>& tw, bool frames_on, int nseg, bool ckpt_on = true,
                             float2* seg = nullptr, float2* stg = nullptr, int tail_skip = 0,
                             float2* tape = nullptr) {
    constexpr int N = P * T;
    const int t = c.t;
    const bool rk2 = FAST ? true : a.scheme == INC_KS_ETRK2;
    const bool split = FAST ? false : a.split != 0;
    float2 X[P], SS[P];
    SlotCache<P, T> cc;
    cc.load(a, c);
#pragma unroll
    for (int m = 0; m < P; ++m) SS[m] = make_float2(0.f, 0.f);
    // prologue: SS = phi1 FFT(s)/N, X = FFT(u)/N
#pragma unroll 1
    for (int k = a.s ? 0 : 1; k < 2; ++k) {
        float2 v[P];
        if (k == 0) {
            load_pair<P, T>(v, a.s, c, N);
        } else {
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = x[m];
        }
        fft_fwd<P, T>(v, buf, tw, t);
        if (split) to_split<P, T>(v, t, buf.a);
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const float2 z = cscale(v[m], a.invN);
            if (k == 0) {
                const Slot sl = cc.get(a, c, m, false);
                SS[m] = rmul(z, sl.p1, sl.p1b);
            } else {
                X[m] = z;
            }
        }
    }
    const int per_step = rk2 ? 4 : 2;  // half-substeps per step() call
    const int64_t frame_stride = (int64_t)a.steps * N;
    int h = 0, step = 0, ck_left = 0, ck_idx = 0;
    bool stage2 = false;
#pragma unroll 1
    for (int it = steps * per_step - tail_skip; it > 0; --it) {
        if (h == 0) {
            if (ckpt_on && a.ckpts) {
                if (ck_left == 0) {
                    store_pair_strided<P, T>(a.ckpts, x, c, N, (int64_t)nseg * N, (int64_t)ck_idx * N);
                    ++ck_idx;
                    ck_left = a.ckpt_every;
                }
                --ck_left;
            }
            if (seg) st_put<P, T>(seg + step * N, x, t);
            if (tape) tape_put<P, T>(tape + (int64_t)step * 4 * N, x, t);
        }
        float2 v[P];
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = sq2(x[m]);
        fft_fwd<P, T>(v, buf, tw, t);
        if (split) to_split<P, T>(v, t, buf.a);
        if (!stage2) {  // Zi = E X + phi1 (D V + S);  ETRK2 carries Y = Zi - phi2 D V
#pragma unroll
            for (int m = 0; m < P; ++m) {
                const Slot sl = cc.get(a, c, m, rk2);
                const float2 DV = dmul(v[m], sl.dn);
                const float2 Zi = cadd(cadd(rmul(X[m], sl.E, sl.Eb), cscale(DV, sl.p1)), SS[m]);
                X[m] = csub(Zi, cscale(DV, sl.p2));  // phi2 = 0 for ETD1
                v[m] = Zi;
            }
        } else {  // X' = Y + phi2 D V2
#pragma unroll
            for (int m = 0; m < P; ++m) {
                const Slot sl = cc.get(a, c, m, true);
                X[m] = cadd(X[m], cscale(dmul(v[m], sl.dn), sl.p2));
                v[m] = X[m];
            }
        }
        if (split) to_packed<P, T>(v, t, buf.a);
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);  // inverse transform by swapping
        fft_fwd<P, T>(v, buf, tw, t);
#pragma unroll
        for (int m = 0; m < P; ++m) x[m] = cswap(v[m]);
        if (stg && h < per_step - 1) st_put<P, T>(stg + (step * 3 + h) * N, x, t);
        if (tape && h < per_step - 1) tape_put<P, T>(tape + ((int64_t)step * 4 + 1 + h) * N, x, t);
        if (rk2) stage2 = !stage2;
        if (++h == per_step) {
            if (frames_on) store_pair_strided<P, T>(a.frames, x, c, N, frame_stride, (int64_t)step * N);
            h = 0;
            ++step;
        }
    }
}

template <int P, int T, int FAST = 0>
__global__ void __launch_bounds__(128) k_step(Args a) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    const Twiddles<P, T> tw = setup_twiddles<P, T>(a, sm, t);
    const Buf<P, T> buf = group_buf<P, T>(group_smem<P, T>(sm, fwd_group_smem<P, T>()), t);
    const int pair = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    Ctx c;
    make_ctx(a, pair, t, pair < a.npairs, c);
    float2 x[P];
    load_pair<P, T>(x, a.u, c, N);
    if (a.cu) add_pair<P, T>(x, a.cu, c, N);  // u + correction_u, solver_1d.py:281/286
    // a single substep runs the first half of the step's half-substeps
    const int skip = a.substeps == 1 ? (a.scheme == INC_KS_ETRK2 ? 2 : 1) : 0;
    forward_program<P, T, FAST>(a, c, x, 1, buf, tw, false, 0, true, nullptr, nullptr, skip);
    store_pair<P, T>(a.out, x, c, N);
}

// Fused rollout of `steps` step() calls with s held constant.
template <int P, int T, int FAST = 0>
__global__ void __launch_bounds__(128) k_rollout(Args a) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    const Twiddles<P, T> tw = setup_twiddles<P, T>(a, sm, t);
    const Buf<P, T> buf = group_buf<P, T>(group_smem<P, T>(sm, fwd_group_smem<P, T>()), t);
    const int pair = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    Ctx c;
    make_ctx(a, pair, t, pair < a.npairs, c);
    float2 x[P];
    load_pair<P, T>(x, a.u, c, N);
    const int nseg = a.ckpt_every > 0 ? (a.steps + a.ckpt_every - 1) / a.ckpt_every : 0;
    // the tape holds a slot for every launched group (its size is rounded up), so
    // groups past the last row pair write padding
    float2* tape = a.tape ? a.tape + (int64_t)pair * a.steps * 4 * N : nullptr;
    forward_program<P, T, FAST>(a, c, x, a.steps, buf, tw, a.frames != nullptr, nseg, true, nullptr, nullptr, 0,
                                tape);
    if (a.out) store_pair<P, T>(a.out, x, c, N);
}

// ---- adjoint ------------------------------------------------------------------
// Per-group shared memory of the backward kernels, in lane layout [m][t]:
// st[0..3] = x1, xi1, xi2, w2 of the step being differentiated (x0 is read
// where the caller keeps it).  The adjoint of one step() (the maths of the
// forward run backwards, substep by substep):
//   w2 = IFFT(d phi2 G);  Gi = G - FFT(2 xi w2)/N
//   w1 = IFFT(d phi1 Gi); Sacc += phi1 Gi
//   G  = E Gi + FFT(2 x (w2 - w1))/N      (ETD1: w2 = 0, Gi = G)
// with x, xi the substep's start and intermediate states, replayed first.
template <int P, int T>
INC_DEV void pair_mul2(float2 (&v)[P], const float2 (&x)[P], float s) {
#pragma unroll
    for (int m = 0; m < P; ++m) v[m] = make_float2(s * x[m].x * v[m].x, s * x[m].y * v[m].y);
}

// Backward of one step() whose input state x0 (correction_u included) is at
// x0s.  G: scaled adjoint spectrum w.r.t. the step output (in) and input
// (out); Sacc accumulates phi1-weighted adjoints (IFFT(Sacc) = dL/ds).  If
// gframe != nullptr the adjoint of this step's output frame is added first.
//
// After the prologue transforms (frame adjoint, FFT(x0)) the program is a
// loop of two-transform units: replay units (FFT(x^2) -> stage -> IFFT,
// storing xi1, x1, xi2; ETD1 stores x1 only), then per substep, second first,
// the adjoint units  w2 = IFFT(d phi2 G) -> G -= FFT(2 xi w2)/N  and
// Sacc += phi1 G, w1 = IFFT(d phi1 G) -> G = E G + FFT(2 x (w2 - w1))/N
// (ETD1: the second unit alone with w2 = 0).
//
// STG: stg holds the step's states xi1, x1, xi2 (ETD1: x1) kept by the segment
// replay in lane layout [3][m][t]; the replay units and FFT(x0) are skipped.
template <int P, int T, bool STG = false, int FAST = 0>
INC_DEV void step_bwd_program(const Args& a, const Ctx& c, const SlotCache<P, T>& cc, const float2 (&SS)[P],
                              float2 (&G)[P], float2 (&Sacc)[P], const float* gframe, int64_t gf_row_stride,
                              int64_t gf_off, const float2* x0s, float2* st, const Buf<P, T>& buf, const Twiddles<P, T>& tw,
                              const float2* stg = nullptr) {
    constexpr int N = P * T;
    const int t = c.t;
    const bool rk2 = FAST ? true : a.scheme == INC_KS_ETRK2;
    const bool split = FAST ? false : a.split != 0;
    const bool single = !STG && a.substeps == 1;  // one substep: its states are x0 (and xi1)
    const float2* x1s = STG ? stg + (rk2 ? N : 0) : st;
    const float2* xi1s = STG ? stg : st + N;
    const float2* xi2s = STG ? stg + 2 * N : st + 2 * N;
    float2* w2s = st + 3 * N;
    float2 X[P];
#pragma unroll 1
    for (int k = gframe ? 0 : 1; k < (STG ? 1 : 2); ++k) {
        float2 v[P];
        if (k == 0) load_pair_strided<P, T>(v, gframe, c, N, gf_row_stride, gf_off);
        else st_get<P, T>(v, x0s, t);
        fft_fwd<P, T>(v, buf, tw, t);
        if (split) to_split<P, T>(v, t, buf.a);
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const float2 z = cscale(v[m], a.invN);
            if (k == 0) G[m] = cadd(G[m], z);
            else X[m] = z;
        }
    }
    const int nrec = single ? (rk2 ? 1 : 0) : (rk2 ? 3 : 1);
    const int nunits = nrec + (rk2 ? 2 : 1) * (single ? 1 : 2);
#pragma unroll 1
    for (int k = STG ? nrec : 0; k < nunits; ++k) {
        const bool rec = !STG && k < nrec;
        const int j = k - nrec;                        // adjoint unit
        const bool unit_w2 = rk2 && !rec && !(j & 1);  // w2 unit (ETRK2 only)
        const bool sub1 = !single && (rk2 ? j < 2 : j < 1);  // second substep first
        float2 v[P];
        // STG: the adjoint unit's state is loaded from scratch before its first
        // transform, so the load overlaps the transform
        float2 u[P];
        if (STG)
            st_get<P, T>(u, unit_w2 ? (sub1 ? xi2s : xi1s) : (sub1 ? x1s : x0s), t);
        // ---- operand of the first transform
        if (rec) {
            st_get<P, T>(v, k == 0 ? x0s : (k == 1 ? xi1s : x1s), t);
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = sq2(v[m]);
        } else {
#pragma unroll
            for (int m = 0; m < P; ++m) {
                const Slot sl = cc.get(a, c, m, unit_w2);
                v[m] = cscale(dmul(G[m], sl.d), unit_w2 ? sl.p2 : sl.p1);
                if (!unit_w2) Sacc[m] = cadd(Sacc[m], rmul(G[m], sl.p1, sl.p1b));
            }
            if (split) to_packed<P, T>(v, t, buf.a);
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);
        }
        fft_fwd<P, T>(v, buf, tw, t);
        // ---- operand of the second transform
        if (rec) {
            if (split) to_split<P, T>(v, t, buf.a);
            if (rk2 && k == 1) {  // stage 2
#pragma unroll
                for (int m = 0; m < P; ++m) {
                    const Slot sl = cc.get(a, c, m, true);
                    X[m] = cadd(X[m], cscale(dmul(v[m], sl.dn), sl.p2));
                    v[m] = X[m];
                }
            } else {  // stage 1
#pragma unroll
                for (int m = 0; m < P; ++m) {
                    const Slot sl = cc.get(a, c, m, rk2);
                    const float2 DV = dmul(v[m], sl.dn);
                    const float2 Zi = cadd(cadd(rmul(X[m], sl.E, sl.Eb), cscale(DV, sl.p1)), SS[m]);
                    X[m] = csub(Zi, cscale(DV, sl.p2));  // phi2 = 0 for ETD1
                    v[m] = Zi;
                }
            }
            if (split) to_packed<P, T>(v, t, buf.a);
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);
        } else {
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);  // w2 or w1
            if (unit_w2) {
                st_put<P, T>(w2s, v, t);
                if (!STG) st_get<P, T>(u, sub1 ? xi2s : xi1s, t);
                pair_mul2<P, T>(v, u, 2.f);
            } else {
                if (!STG) st_get<P, T>(u, sub1 ? x1s : x0s, t);
                if (rk2) {
                    float2 w2[P];
                    st_get<P, T>(w2, w2s, t);
#pragma unroll
                    for (int m = 0; m < P; ++m) v[m] = csub(w2[m], v[m]);
                    pair_mul2<P, T>(v, u, 2.f);
                } else {
                    pair_mul2<P, T>(v, u, -2.f);
                }
            }
        }
        fft_fwd<P, T>(v, buf, tw, t);
        // ---- result
        if (rec) {
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = cswap(v[m]);
            st_put<P, T>(rk2 ? (k == 0 ? st + N : (k == 1 ? st : st + 2 * N)) : st, v, t);
        } else {
            if (split) to_split<P, T>(v, t, buf.a);
            if (unit_w2) {
#pragma unroll
                for (int m = 0; m < P; ++m) G[m] = csub(G[m], cscale(v[m], a.invN));
            } else {
#pragma unroll
                for (int m = 0; m < P; ++m) {
                    const Slot sl = cc.get(a, c, m, false);
                    G[m] = cadd(rmul(G[m], sl.E, sl.Eb), cscale(v[m], a.invN));
                }
            }
        }
    }
}

// Spectra entering the adjoint: SS = phi1 FFT(s)/N and G = FFT(g)/N of an
// adjoint field g (null: zero), as one loop around one transform.
template <int P, int T>
INC_DEV void adjoint_prologue(const Args& a, const Ctx& c, const SlotCache<P, T>& cc, const float* g,
                              float2 (&SS)[P], float2 (&G)[P], const Buf<P, T>& buf, const Twiddles<P, T>& tw) {
    constexpr int N = P * T;
#pragma unroll
    for (int m = 0; m < P; ++m) { SS[m] = make_float2(0.f, 0.f); G[m] = make_float2(0.f, 0.f); }
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        const float* src = k == 0 ? a.s : g;
        if (!src) continue;
        float2 v[P];
        load_pair<P, T>(v, src, c, N);
        fft_fwd<P, T>(v, buf, tw, c.t);
        if (a.split) to_split<P, T>(v, c.t, buf.a);
#pragma unroll
        for (int m = 0; m < P; ++m) {
            const float2 z = cscale(v[m], a.invN);
            if (k == 0) {
                const Slot sl = cc.get(a, c, m, false);
                SS[m] = rmul(z, sl.p1, sl.p1b);
            } else {
                G[m] = z;
            }
        }
    }
}

// dL/du = IFFT(G) and dL/ds = IFFT(Sacc) stored to the caller's arrays.
template <int P, int T>
INC_DEV void adjoint_epilogue(const Args& a, const Ctx& c, const float2 (&G)[P], const float2 (&Sacc)[P], const Buf<P, T>& buf,
                              const Twiddles<P, T>& tw) {
    constexpr int N = P * T;
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        float* dst = k == 0 ? a.g_u : a.g_s;
        if (!dst) continue;
        float2 v[P];
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = k == 0 ? G[m] : Sacc[m];
        if (a.split) to_packed<P, T>(v, c.t, buf.a);
        fft_inv<P, T>(v, buf, tw, c.t);
        store_pair<P, T>(dst, v, c, N);
    }
}


template <int P, int T, int FAST = 0>
__global__ void __launch_bounds__(128) k_step_bwd(Args a) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    const Twiddles<P, T> tw = setup_twiddles<P, T>(a, sm, t);
    float2* g = group_smem<P, T>(sm, bwd_group_smem<P, T>(0));
    const Buf<P, T> buf = group_buf<P, T>(g, t);
    float2* st = g + 2 * buf_len<P, T>();
    const int pair = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    Ctx c;
    make_ctx(a, pair, t, pair < a.npairs, c);
    SlotCache<P, T> cc;
    cc.load(a, c);
    float2 G[P], Sacc[P], SS[P];
    adjoint_prologue<P, T>(a, c, cc, a.g_out, SS, G, buf, tw);
    {
        float2 x0[P];
        load_pair<P, T>(x0, a.u, c, N);
        if (a.cu) add_pair<P, T>(x0, a.cu, c, N);
        st_put<P, T>(st + 4 * N, x0, t);
    }
#pragma unroll
    for (int m = 0; m < P; ++m) Sacc[m] = make_float2(0.f, 0.f);
    step_bwd_program<P, T, false, FAST>(a, c, cc, SS, G, Sacc, nullptr, 0, 0, st + 4 * N, st, buf, tw);
    adjoint_epilogue<P, T>(a, c, G, Sacc, buf, tw);
}

// Backward of the fused rollout: each ckpt_every-step segment is replayed from
// its checkpoint (states kept in shared memory), then differentiated step by step.
template <int P, int T, bool STG, int FAST = 0>
__global__ void __launch_bounds__(128) k_rollout_bwd(Args a) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    const Twiddles<P, T> tw = setup_twiddles<P, T>(a, sm, t);
    const int K = a.ckpt_every;
    float2* g = group_smem<P, T>(sm, bwd_group_smem<P, T>(K));
    const Buf<P, T> buf = group_buf<P, T>(g, t);
    float2* st = g + 2 * buf_len<P, T>();
    float2* seg = st + 5 * N;
    const int pair = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    Ctx c;
    make_ctx(a, pair, t, pair < a.npairs, c);
    SlotCache<P, T> cc;
    cc.load(a, c);
    float2 G[P], Sacc[P], SS[P];
    adjoint_prologue<P, T>(a, c, cc, a.g_final, SS, G, buf, tw);
#pragma unroll
    for (int m = 0; m < P; ++m) Sacc[m] = make_float2(0.f, 0.f);
    const int nseg = (a.steps + K - 1) / K;
    // STG: this group's scratch for the replayed substep states (every launched group has one)
    float2* stg = STG ? a.stage + (size_t)pair * 3 * K * N : nullptr;
    // STG with up to 8 values per lane: each step's frame adjoint is loaded one step
    // ahead (it comes from HBM; wider lanes have no registers to spare for it)
    constexpr bool GPRE = STG && P <= 8;
    const bool split = FAST ? false : a.split != 0;
    const int64_t gf_stride = (int64_t)a.steps * N;
    float2 gf[P];
    if (GPRE && a.g_frames) load_pair_strided<P, T>(gf, a.g_frames, c, N, gf_stride, (int64_t)(a.steps - 1) * N);
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        {
            float2 x[P];
            load_pair_strided<P, T>(x, a.ckpts, c, N, (int64_t)nseg * N, (int64_t)sidx * N);
            if (STG) {  // every step's start state and its substep states, the last step's result left out
                forward_program<P, T, FAST>(a, c, x, len, buf, tw, false, nseg, false, seg, stg, 1);
            } else {
                forward_program<P, T, FAST>(a, c, x, len - 1, buf, tw, false, nseg, false, seg);
                st_put<P, T>(seg + (len - 1) * N, x, t);
            }
        }
        for (int j = len - 1; j >= 0; --j) {
            const int k = k0 + j;
            if (GPRE && a.g_frames) {  // G += FFT(dL/dframe_k)/N, the next step's frame adjoint loaded meanwhile
                float2 v[P];
#pragma unroll
                for (int m = 0; m < P; ++m) v[m] = gf[m];
                if (k > 0) load_pair_strided<P, T>(gf, a.g_frames, c, N, gf_stride, (int64_t)(k - 1) * N);
                fft_fwd<P, T>(v, buf, tw, t);
                if (split) to_split<P, T>(v, t, buf.a);
#pragma unroll
                for (int m = 0; m < P; ++m) G[m] = cadd(G[m], cscale(v[m], a.invN));
            }
            step_bwd_program<P, T, STG, FAST>(a, c, cc, SS, G, Sacc, GPRE ? nullptr : a.g_frames, gf_stride,
                                              (int64_t)k * N, seg + j * N, st, buf, tw,
                                              STG ? stg + (size_t)j * 3 * N : nullptr);
        }
    }
    adjoint_epilogue<P, T>(a, c, G, Sacc, buf, tw);
}

// The same backward with the segment replay on a second warp: one row pair per
// CTA of 2 T threads (T = 32, P <= 8, the common case).  Warp 0 replays segment s - 1 from
// its checkpoint into one half of a double buffer (every step's start state in
// shared memory, its substep states in the global scratch, which holds two
// segments per pair) while warp 1 differentiates segment s from the other half, so
// only the adjoint's transforms stay on the critical path.  The two warps meet at
// one block barrier per segment, which also orders the replay's scratch stores
// before the adjoint's loads.
template <int P, int T, int FAST>
__global__ void __launch_bounds__(2 * T) k_rollout_bwd_ws(Args a) {
    static_assert(T == 32, "one warp per role");
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    const bool rep = threadIdx.x < T;
    const Twiddles<P, T> tw = setup_twiddles<P, T>(a, sm, t);
    const int K = a.ckpt_every;
    constexpr int GS = group_stride<T>(2 * buf_len<P, T>());
    float2* base = sm + tw_size<P, T>();
    const Buf<P, T> buf = group_buf<P, T>(base + (rep ? 0 : GS), t);
    float2* st = base + 2 * GS;  // the adjoint's state slots
    float2* segb = st + 5 * N;   // [2][K][N] step start states
    const int pair = blockIdx.x;
    Ctx c;
    make_ctx(a, pair, t, pair < a.npairs, c);
    SlotCache<P, T> cc;
    cc.load(a, c);
    const int nseg = (a.steps + K - 1) / K;
    float2* stgb = a.stage + (size_t)pair * 2 * 3 * K * N;  // [2][3K][N] substep states
    auto replay = [&](int sidx) {
        float2 x[P];
        load_pair_strided<P, T>(x, a.ckpts, c, N, (int64_t)nseg * N, (int64_t)sidx * N);
        forward_program<P, T, FAST>(a, c, x, min(K, a.steps - sidx * K), buf, tw, false, nseg, false,
                                    segb + (sidx & 1) * K * N, stgb + (size_t)(sidx & 1) * 3 * K * N, 1);
    };
    float2 G[P], Sacc[P], SS[P], gf[P];
    const int64_t gf_stride = (int64_t)a.steps * N;
    if (!rep) {
        adjoint_prologue<P, T>(a, c, cc, a.g_final, SS, G, buf, tw);
#pragma unroll
        for (int m = 0; m < P; ++m) Sacc[m] = make_float2(0.f, 0.f);
        if (a.g_frames) load_pair_strided<P, T>(gf, a.g_frames, c, N, gf_stride, (int64_t)(a.steps - 1) * N);
    }
    if (rep) replay(nseg - 1);
    __syncthreads();
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        if (rep) {
            if (sidx > 0) replay(sidx - 1);
        } else {
            const float2* seg = segb + (sidx & 1) * K * N;
            const float2* stg = stgb + (size_t)(sidx & 1) * 3 * K * N;
            const int k0 = sidx * K;
            const int len = min(K, a.steps - k0);
            for (int j = len - 1; j >= 0; --j) {
                const int k = k0 + j;
                if (a.g_frames) {  // G += FFT(dL/dframe_k)/N, the next step's frame adjoint loaded meanwhile
                    float2 v[P];
#pragma unroll
                    for (int m = 0; m < P; ++m) v[m] = gf[m];
                    if (k > 0) load_pair_strided<P, T>(gf, a.g_frames, c, N, gf_stride, (int64_t)(k - 1) * N);
                    fft_fwd<P, T>(v, buf, tw, t);
#pragma unroll
                    for (int m = 0; m < P; ++m) G[m] = cadd(G[m], cscale(v[m], a.invN));
                }
                step_bwd_program<P, T, true, FAST>(a, c, cc, SS, G, Sacc, nullptr, gf_stride, (int64_t)k * N,
                                                   seg + j * N, st, buf, tw, stg + (size_t)j * 3 * N);
            }
        }
        __syncthreads();  // segment sidx - 1 replayed, segment sidx's half free
    }
    if (!rep) adjoint_epilogue<P, T>(a, c, G, Sacc, buf, tw);
}

// Asynchronous 8-byte copies global -> shared (cp.async), in commit groups.
INC_DEV void cp_async8(float2* smem_dst, const float2* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
INC_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPENDING>
INC_DEV void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPENDING) : "memory"); }

// This lane's share of one step's tape slot ([4][m][t]) copied into shared memory.
template <int P, int T>
INC_DEV void tape_prefetch(float2* dst, const float2* src, int t) {
#pragma unroll
    for (int q = 0; q < 4 * P; ++q) cp_async8(dst + q * T + t, src + q * T + t);
    cp_async_commit();
}

// Backward of a tape rollout: every step's start and substep states come from the
// tape the forward wrote, so no segment is replayed: per step() the frame
// adjoint's transform and the adjoint units' eight (ETRK2) against 17 with the
// replay.  The tape lives in HBM (it outgrows L2), so each step's states are
// copied into shared memory (cp.async) while the step before them is
// differentiated, and each frame adjoint is loaded a step ahead.
template <int P, int T, int FAST = 0>
__global__ void __launch_bounds__(128) k_rollout_bwd_tape(Args a) {
    extern __shared__ float2 sm[];
    constexpr int N = P * T;
    const int t = threadIdx.x % T;
    const Twiddles<P, T> tw = setup_twiddles<P, T>(a, sm, t);
    float2* g = group_smem<P, T>(sm, bwd_group_smem<P, T>(8));
    const Buf<P, T> buf = group_buf<P, T>(g, t);
    float2* st = g + 2 * buf_len<P, T>();
    float2* stage = st + 5 * N;  // two [4][m][t] slots
    const int pair = blockIdx.x * (blockDim.x / T) + threadIdx.x / T;
    Ctx c;
    make_ctx(a, pair, t, pair < a.npairs, c);
    SlotCache<P, T> cc;
    cc.load(a, c);
    const bool split = FAST ? false : a.split != 0;
    float2 G[P], Sacc[P], SS[P];
    adjoint_prologue<P, T>(a, c, cc, a.g_final, SS, G, buf, tw);
#pragma unroll
    for (int m = 0; m < P; ++m) Sacc[m] = make_float2(0.f, 0.f);
    const float2* tape = a.tape + (int64_t)pair * a.steps * 4 * N;
    const int64_t gf_stride = (int64_t)a.steps * N;
    tape_prefetch<P, T>(stage + ((a.steps - 1) & 1) * 4 * N, tape + (int64_t)(a.steps - 1) * 4 * N, t);
    float2 gf[P];
    if (a.g_frames) load_pair_strided<P, T>(gf, a.g_frames, c, N, gf_stride, (int64_t)(a.steps - 1) * N);
    for (int k = a.steps - 1; k >= 0; --k) {
        if (k > 0) {
            tape_prefetch<P, T>(stage + ((k - 1) & 1) * 4 * N, tape + (int64_t)(k - 1) * 4 * N, t);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        if (a.g_frames) {  // G += FFT(dL/dframe_k)/N, the next step's frame adjoint loaded meanwhile
            float2 v[P];
#pragma unroll
            for (int m = 0; m < P; ++m) v[m] = gf[m];
            if (k > 0) load_pair_strided<P, T>(gf, a.g_frames, c, N, gf_stride, (int64_t)(k - 1) * N);
            fft_fwd<P, T>(v, buf, tw, t);
            if (split) to_split<P, T>(v, t, buf.a);
#pragma unroll
            for (int m = 0; m < P; ++m) G[m] = cadd(G[m], cscale(v[m], a.invN));
        }
        const float2* ts = stage + (k & 1) * 4 * N;
        step_bwd_program<P, T, true, FAST>(a, c, cc, SS, G, Sacc, nullptr, 0, 0, ts, st, buf, tw, ts + N);
    }
    adjoint_epilogue<P, T>(a, c, G, Sacc, buf, tw);
}

// ---- launchers (instantiated per shape in ks_{fwd,bwd}_*.cu) ---------------------
enum class Kind { Step, Rollout, StepBwd, RolloutBwd, TapeBwd };

template <int P, int T>
int launch_fwd(Kind kind, const Args& a, cudaStream_t st, int block);
template <int P, int T>
int launch_bwd(Kind kind, const Args& a, cudaStream_t st, int block);

template <int P, int T>
size_t smem_bytes(Kind kind, int block, int K) {
    const int groups = block / T;
    size_t per = (kind == Kind::Step || kind == Kind::Rollout) ? fwd_group_smem<P, T>()
               : bwd_group_smem<P, T>(kind == Kind::RolloutBwd ? K : (kind == Kind::TapeBwd ? 8 : 0));
    return (tw_size<P, T>() + groups * per) * sizeof(float2);
}

// The kernels compiled for the common case alone (see forward_program).
inline bool fast_case(const Args& a) { return a.scheme == INC_KS_ETRK2 && !a.split; }

template <typename F>
int launch_with_smem(F kernel, int grid, int block, size_t smem, cudaStream_t st, const Args& a) {
    if (smem > 227 * 1024) {
        set_error("ks: %zu bytes of shared memory needed (max 227 KB); lower ckpt_every", smem);
        return INC_E_INVALID;
    }
    if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    kernel<<<grid, block, smem, st>>>(a);
    return check_launch("ks");
}

template <int P, int T>
int launch_fwd_impl(Kind kind, const Args& a, cudaStream_t st, int block) {
    const int gpb = block / T;
    const int grid = (a.npairs + gpb - 1) / gpb;
    const size_t smem = smem_bytes<P, T>(kind, block, a.ckpt_every);
    if (fast_case(a)) {
        if (kind == Kind::Step) return launch_with_smem(k_step<P, T, 1>, grid, block, smem, st, a);
        return launch_with_smem(k_rollout<P, T, 1>, grid, block, smem, st, a);
    }
    if (kind == Kind::Step) return launch_with_smem(k_step<P, T>, grid, block, smem, st, a);
    return launch_with_smem(k_rollout<P, T>, grid, block, smem, st, a);
}

// Shared memory of k_rollout_bwd_ws (one row pair per CTA).
template <int P, int T>
size_t ws_smem_bytes(int K) {
    return (tw_size<P, T>() + 2 * group_stride<T>(2 * buf_len<P, T>()) + (size_t)(5 + 2 * K) * P * T) *
           sizeof(float2);
}

template <int P, int T>
int launch_bwd_impl(Kind kind, const Args& a, cudaStream_t st, int block) {
    const int gpb = block / T;
    const int grid = (a.npairs + gpb - 1) / gpb;
    const size_t smem = smem_bytes<P, T>(kind, block, a.ckpt_every);
    if constexpr (T == 32 && P <= 8) {  // the scratch then holds two segments per pair (inc_ks_rollout_bwd_work_size)
        if (kind == Kind::RolloutBwd && a.stage && fast_case(a) && ws_smem_bytes<P, T>(a.ckpt_every) <= 227 * 1024)
            return launch_with_smem(k_rollout_bwd_ws<P, T, 1>, a.npairs, 2 * T, ws_smem_bytes<P, T>(a.ckpt_every),
                                    st, a);
    }
    if (fast_case(a)) {
        if (kind == Kind::StepBwd) return launch_with_smem(k_step_bwd<P, T, 1>, grid, block, smem, st, a);
        if (kind == Kind::TapeBwd) return launch_with_smem(k_rollout_bwd_tape<P, T, 1>, grid, block, smem, st, a);
        if (a.stage) return launch_with_smem(k_rollout_bwd<P, T, true, 1>, grid, block, smem, st, a);
        return launch_with_smem(k_rollout_bwd<P, T, false, 1>, grid, block, smem, st, a);
    }
    if (kind == Kind::StepBwd) return launch_with_smem(k_step_bwd<P, T>, grid, block, smem, st, a);
    if (kind == Kind::TapeBwd) return launch_with_smem(k_rollout_bwd_tape<P, T>, grid, block, smem, st, a);
    if (a.stage) return launch_with_smem(k_rollout_bwd<P, T, true>, grid, block, smem, st, a);
    return launch_with_smem(k_rollout_bwd<P, T, false>, grid, block, smem, st, a);
}


// (P, T) shapes: N = P*T, T <= 32 lanes per row pair, P <= 32 values per lane.
#define INC_KS_SHAPES(X) \
    X(4, 4) X(4, 8) X(4, 16) X(8, 8) X(4, 32) X(8, 16) X(8, 32) X(16, 16) X(16, 32) X(32, 16) X(4, 64) X(8, 64)

}  // namespace ks
}  // namespace inc
