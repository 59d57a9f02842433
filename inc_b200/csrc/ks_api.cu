// KS C ABI: plan construction (row pairing, FP64 coefficients, twiddles) and
// shape dispatch.  Kernels live in ks_kernels.cuh.
#include <algorithm>
#include <numeric>
#include <vector>

#include "ks_kernels.cuh"

namespace inc {
namespace ks {

// ---- plan kernels (FP64) -------------------------------------------------------
// exp(L dt), phi1, phi2 per row and wavenumber (solver_1d.py:235-267), L = k^2 - k^4,
// k = 2 pi f / domain_size.  Computed in FP64, stored FP32.
__global__ void k_coef(const float* __restrict__ dsz, float* __restrict__ coef, float* __restrict__ dR,
                       int rows, int n, int nhp, double dt, int scheme) {
    const int nh = n / 2 + 1;
    const int64_t total = (int64_t)rows * nh;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(i / nh), kk = (int)(i % nh);
        const double L = (double)dsz[row];
        const double kap = 2.0 * M_PI * (double)kk / L;
        const double lop = kap * kap - kap * kap * kap * kap;
        const double e = exp(lop * dt);
        double p1, p2;
        if (scheme == INC_KS_ETD1) {
            p1 = (lop == 0.0) ? dt : (e - 1.0) / lop;
            p2 = 0.0;
        } else {
            const bool small = fabs(lop) < 1e-6;
            p1 = small ? dt : (e - 1.0) / lop;
            p2 = small ? dt / 2 : (e - 1.0 - lop * dt) / (lop * lop * dt);
        }
        float* cr = coef + (int64_t)row * 3 * nhp;
        cr[kk] = (float)e;
        cr[nhp + kk] = (float)p1;
        cr[2 * nhp + kk] = (float)p2;
        if (kk == 0) dR[row] = (float)(M_PI / L);
    }
}

// FFT twiddles of the later Stockham passes in the layout of fft_later():
// entry pi*N + (q*R + r)*T + t = exp(-2 pi i r k / (NS R)), k = (t + T q) % NS,
// for the pass with index pi, span NS and radix R.  FP64, stored FP32.
__global__ void k_twiddle(float2* tw, int n, int T) {
    const int P = n / T;
    int pi = 0;
    for (int ns = P; ns < n; ns *= (P < n / ns ? P : n / ns), ++pi) {
        const int R = P < n / ns ? P : n / ns;
        const int Q = P / R;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Q * R * T; i += gridDim.x * blockDim.x) {
            const int t = i % T, r = (i / T) % R, q = i / (T * R);
            const int k = (t + T * q) % ns;
            double s, c;
            sincospi(-2.0 * (double)r * (double)k / ((double)ns * (double)R), &s, &c);
            tw[pi * n + i] = make_float2((float)c, (float)s);
        }
    }
}

inline int64_t align256(int64_t v) { return (v + 255) & ~int64_t(255); }
inline int nhp_of(int n) { return ((n / 2 + 1) + 3) & ~3; }

struct Layout {
    int64_t dR, pairs, tw, coef, L, total;
};

inline Layout layout(int rows, int n) {
    Layout l;
    int64_t off = 0;
    l.dR = off; off = align256(off + (int64_t)rows * 4);
    l.pairs = off; off = align256(off + (int64_t)((rows + 1) / 2) * 2 * 4);
    l.tw = off; off = align256(off + (int64_t)4 * n * 8);  // <= 4 later FFT passes
    l.coef = off; off = align256(off + (int64_t)rows * 3 * nhp_of(n) * 4);
    l.L = off; off = align256(off + (int64_t)rows * 4);
    l.total = off;
    return l;
}

// Lanes per row pair: as many as the n allows (<= 32), for latency.
inline int default_tpp(int n) {
    switch (n) {
        case 16: return 4;
        case 32: return 8;
        case 64: return 16;
        case 128: return 32;
        default: return 64;
    }
}

// The (P, T) shapes that have kernels (INC_KS_SHAPES).
inline bool valid_shape(int n, int T) {
    if (!is_pow2(n) || n < 16 || n > 512 || T <= 0 || n % T) return false;
    const int P = n / T;
#define INC_HAS(PP, TT) if (P == PP && T == TT) return true;
    INC_KS_SHAPES(INC_HAS)
#undef INC_HAS
    return false;
}

int fill_args(const inc_ks_plan* p, Args& a) {
    memset(&a, 0, sizeof(a));
    if (!p || !p->dev) { set_error("ks: null plan"); return INC_E_INVALID; }
    if (p->npairs <= 0) { set_error("ks: plan not initialised (call inc_ks_plan_init)"); return INC_E_INVALID; }
    const Layout l = layout(p->rows, p->n);
    const char* base = static_cast<const char*>(p->dev);
    a.rows = p->rows; a.n = p->n; a.npairs = p->npairs; a.scheme = p->scheme; a.split = p->split;
    a.dealias = p->dealias; a.nhp = nhp_of(p->n); a.invN = 1.f / (float)p->n;
    a.dR = reinterpret_cast<const float*>(base + l.dR);
    a.pairs = reinterpret_cast<const int*>(base + l.pairs);
    a.tw = reinterpret_cast<const float2*>(base + l.tw);
    a.coef = reinterpret_cast<const float*>(base + l.coef);
    return INC_OK;
}

int pick_block(Kind kind, int npairs, int T, int n, int K) {
    if (T > 32) return T;  // a wide pair is the whole CTA
    int block = 128;
    // keep >= 2 blocks per SM when the batch allows it
    while (block > 32 && (int64_t)npairs * T / block < 2 * 148) block >>= 1;
    auto smem = [&](int b) {
        const int groups = b / T;
        int64_t per = 2 * (n + n / 4 + 64) + 16;  // bound on the exchange buffers' padded layouts
        if (kind == Kind::StepBwd || kind == Kind::RolloutBwd || kind == Kind::TapeBwd) per += 5 * n;
        if (kind == Kind::RolloutBwd) per += (int64_t)K * n;
        if (kind == Kind::TapeBwd) per += (int64_t)8 * n;  // two staged tape slots
        return (int64_t)(4 * n + groups * per) * 8;
    };
    while (block > 32 && smem(block) > 100 * 1024) block >>= 1;
    return block;
}

int dispatch(Kind kind, const inc_ks_plan* p, const Args& a, cudaStream_t st) {
    const int n = p->n;
    const int T = p->threads_per_pair ? p->threads_per_pair : default_tpp(n);
    if (!valid_shape(n, T)) {
        set_error("ks: unsupported n=%d threads_per_pair=%d", n, T);
        return INC_E_UNSUPPORTED;
    }
    const int P = n / T;
    const int block = pick_block(kind, a.npairs, T, n, a.ckpt_every);
    const bool bwd = kind == Kind::StepBwd || kind == Kind::RolloutBwd || kind == Kind::TapeBwd;
#define INC_CASE(PP, TT) \
    if (P == PP && T == TT) return bwd ? launch_bwd<PP, TT>(kind, a, st, block) : launch_fwd<PP, TT>(kind, a, st, block);
    INC_KS_SHAPES(INC_CASE)
#undef INC_CASE
    set_error("ks: no kernel for n=%d threads_per_pair=%d", n, T);
    return INC_E_UNSUPPORTED;
}

}  // namespace ks
}  // namespace inc

using namespace inc;
using namespace inc::ks;

extern "C" int64_t inc_ks_plan_size(int32_t rows, int32_t n) {
    if (rows <= 0 || !is_pow2(n) || n < 16 || n > 512) return -1;
    return layout(rows, n).total;
}

extern "C" int inc_ks_plan_init(inc_ks_plan* p, const float* dsz_host, void* stream) {
    if (!p || !p->dev || !dsz_host) { set_error("ks_plan_init: null argument"); return INC_E_INVALID; }
    if (p->rows <= 0) { set_error("ks_plan_init: rows must be positive"); return INC_E_INVALID; }
    if (!is_pow2(p->n) || p->n < 16 || p->n > 512) {
        set_error("ks_plan_init: resolution must be a power of two in [16, 512] (got %d)", p->n);
        return INC_E_UNSUPPORTED;
    }
    if (p->scheme != INC_KS_ETRK2 && p->scheme != INC_KS_ETD1) { set_error("ks_plan_init: unknown time scheme %d", p->scheme); return INC_E_INVALID; }
    if (!(p->dt > 0)) { set_error("ks_plan_init: dt must be positive"); return INC_E_INVALID; }
    const int T = p->threads_per_pair ? p->threads_per_pair : default_tpp(p->n);
    if (!valid_shape(p->n, T)) { set_error("ks_plan_init: threads_per_pair=%d invalid for n=%d", T, p->n); return INC_E_UNSUPPORTED; }
    for (int r = 0; r < p->rows; ++r)
        if (!(dsz_host[r] > 0.f)) { set_error("ks_plan_init: domain_size[%d] must be positive", r); return INC_E_INVALID; }
    p->threads_per_pair = T;
    // Pair rows: sort by domain size so equal sizes share a complex FFT.
    std::vector<int> idx(p->rows);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return dsz_host[x] < dsz_host[y]; });
    const int npairs = (p->rows + 1) / 2;
    std::vector<int> pairs(2 * npairs);
    int split = 0;
    for (int q = 0; q < npairs; ++q) {
        pairs[2 * q] = idx[2 * q];
        pairs[2 * q + 1] = (2 * q + 1 < p->rows) ? idx[2 * q + 1] : -1;
        if (pairs[2 * q + 1] >= 0 && dsz_host[pairs[2 * q]] != dsz_host[pairs[2 * q + 1]]) split = 1;
    }
    const Layout l = layout(p->rows, p->n);
    char* base = static_cast<char*>(p->dev);
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemcpyAsync(base + l.pairs, pairs.data(), pairs.size() * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + l.L, dsz_host, (size_t)p->rows * 4, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) { set_error("ks_plan_init: upload failed: %s", cudaGetErrorString(e)); return INC_E_LAUNCH; }
    const int nh = p->n / 2 + 1;
    const int64_t total = (int64_t)p->rows * nh;
    const int grid = (int)std::min<int64_t>((total + 255) / 256, 4096);
    k_coef<<<grid, 256, 0, st>>>(reinterpret_cast<const float*>(base + l.L), reinterpret_cast<float*>(base + l.coef),
                                 reinterpret_cast<float*>(base + l.dR), p->rows, p->n, nhp_of(p->n), p->dt, p->scheme);
    int rc = check_launch("ks_coef");
    if (rc) return rc;
    k_twiddle<<<(p->n + 255) / 256, 256, 0, st>>>(reinterpret_cast<float2*>(base + l.tw), p->n, T);
    rc = check_launch("ks_twiddle");
    if (rc) return rc;
    // The host vectors die with this call: finish the pageable uploads first.
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { set_error("ks_plan_init: %s", cudaGetErrorString(e)); return INC_E_LAUNCH; }
    p->npairs = npairs;
    p->split = split;
    return INC_OK;
}

static inline bool ok_ptr(const void* q) { return q && (reinterpret_cast<uintptr_t>(q) & 3u) == 0; }

extern "C" int inc_ks_step(const inc_ks_plan* p, const float* u, const float* s, const float* cu, float* u_out,
                           void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(u) || !ok_ptr(u_out)) { set_error("ks_step: bad u/u_out"); return INC_E_INVALID; }
    a.u = u; a.s = s; a.cu = cu; a.out = u_out;
    return dispatch(Kind::Step, p, a, as_stream(stream));
}

extern "C" int inc_ks_step_bwd(const inc_ks_plan* p, const float* u, const float* s, const float* cu,
                               const float* g_out, float* g_u, float* g_s, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(u) || !ok_ptr(g_out) || !ok_ptr(g_u)) { set_error("ks_step_bwd: bad pointer"); return INC_E_INVALID; }
    a.u = u; a.s = s; a.cu = cu; a.g_out = g_out; a.g_u = g_u; a.g_s = g_s;
    return dispatch(Kind::StepBwd, p, a, as_stream(stream));
}

extern "C" int inc_ks_substep(const inc_ks_plan* p, const float* u, const float* s, float* u_out, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(u) || !ok_ptr(u_out)) { set_error("ks_substep: bad u/u_out"); return INC_E_INVALID; }
    a.u = u; a.s = s; a.out = u_out; a.substeps = 1;
    return dispatch(Kind::Step, p, a, as_stream(stream));
}

extern "C" int inc_ks_substep_bwd(const inc_ks_plan* p, const float* u, const float* s, const float* g_out,
                                  float* g_u, float* g_s, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(u) || !ok_ptr(g_out) || !ok_ptr(g_u)) { set_error("ks_substep_bwd: bad pointer"); return INC_E_INVALID; }
    a.u = u; a.s = s; a.g_out = g_out; a.g_u = g_u; a.g_s = g_s; a.substeps = 1;
    return dispatch(Kind::StepBwd, p, a, as_stream(stream));
}

extern "C" int inc_ks_rollout(const inc_ks_plan* p, const float* u0, const float* s, int32_t steps, float* frames,
                              float* u_final, int32_t ckpt_every, float* ckpts, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(u0) || steps < 0) { set_error("ks_rollout: bad arguments"); return INC_E_INVALID; }
    if (ckpts && ckpt_every <= 0) { set_error("ks_rollout: ckpt_every must be positive with ckpts"); return INC_E_INVALID; }
    a.u = u0; a.s = s; a.steps = steps; a.frames = frames; a.out = u_final; a.ckpt_every = ckpt_every; a.ckpts = ckpts;
    return dispatch(Kind::Rollout, p, a, as_stream(stream));
}

extern "C" int64_t inc_ks_rollout_bwd_work_size(const inc_ks_plan* p, int32_t ckpt_every) {
    if (!p || p->npairs <= 0 || ckpt_every <= 0) return -1;
    const int n = p->n;
    const int T = p->threads_per_pair ? p->threads_per_pair : default_tpp(n);
    if (!valid_shape(n, T)) return -1;
    // one [ckpt_every][3][n] float2 slot per launched group (the launch's grid x groups per block)
    const int gpb = pick_block(Kind::RolloutBwd, p->npairs, T, n, ckpt_every) / T;
    const int64_t groups = (int64_t)((p->npairs + gpb - 1) / gpb) * gpb;
    // 32 lanes and up to 8 values per lane in the common case (ETRK2, one domain size
    // per pair): the warp-specialised backward keeps two segments per pair
    const int64_t segs = (T == 32 && n / T <= 8 && p->scheme == INC_KS_ETRK2 && !p->split) ? 2 : 1;
    return segs * groups * 3 * ckpt_every * n * (int64_t)sizeof(float2);
}

static int ks_rollout_bwd(const inc_ks_plan* p, const float* ckpts, const float* s, int32_t steps,
                          int32_t ckpt_every, const float* g_frames, const float* g_final, float* g_u0, float* g_s,
                          void* work, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(ckpts) || !ok_ptr(g_u0) || steps <= 0 || ckpt_every <= 0) { set_error("ks_rollout_bwd: bad arguments"); return INC_E_INVALID; }
    a.s = s; a.steps = steps; a.ckpt_every = ckpt_every; a.ckpts = const_cast<float*>(ckpts);
    a.g_frames = g_frames; a.g_final = g_final; a.g_u = g_u0; a.g_s = g_s;
    a.stage = static_cast<float2*>(work);
    return dispatch(Kind::RolloutBwd, p, a, as_stream(stream));
}

extern "C" int inc_ks_rollout_bwd(const inc_ks_plan* p, const float* ckpts, const float* s, int32_t steps,
                                  int32_t ckpt_every, const float* g_frames, const float* g_final, float* g_u0,
                                  float* g_s, void* stream) {
    return ks_rollout_bwd(p, ckpts, s, steps, ckpt_every, g_frames, g_final, g_u0, g_s, nullptr, stream);
}

extern "C" int inc_ks_rollout_bwd_ws(const inc_ks_plan* p, const float* ckpts, const float* s, int32_t steps,
                                     int32_t ckpt_every, const float* g_frames, const float* g_final, float* g_u0,
                                     float* g_s, void* work, int64_t work_bytes, void* stream) {
    const int64_t need = inc_ks_rollout_bwd_work_size(p, ckpt_every);
    if (need < 0) { set_error("ks_rollout_bwd_ws: bad plan or ckpt_every"); return INC_E_INVALID; }
    if (!work || work_bytes < need || (reinterpret_cast<uintptr_t>(work) & 15u) != 0) {
        set_error("ks_rollout_bwd_ws: work needs %lld bytes, 16-byte aligned (got %lld)", (long long)need,
                  (long long)work_bytes);
        return INC_E_INVALID;
    }
    return ks_rollout_bwd(p, ckpts, s, steps, ckpt_every, g_frames, g_final, g_u0, g_s, work, stream);
}

// ---- tape rollouts: the forward records every step's states, the backward reads them
// Row pairs rounded up to 32: the padding absorbs the writes of launched groups past the
// last pair (at most 32 groups per block for the narrowest layout).
extern "C" int64_t inc_ks_tape_size(const inc_ks_plan* p, int32_t steps) {
    if (!p || p->npairs <= 0 || steps <= 0) return -1;
    const int64_t pairs = ((int64_t)p->npairs + 31) / 32 * 32;
    return pairs * steps * 4 * p->n * (int64_t)sizeof(float2);
}

static int check_tape(const inc_ks_plan* p, int32_t steps, const void* tape, int64_t tape_bytes, const char* who) {
    const int64_t need = inc_ks_tape_size(p, steps);
    if (need < 0) { set_error("%s: bad plan or steps", who); return INC_E_INVALID; }
    if (!tape || tape_bytes < need || (reinterpret_cast<uintptr_t>(tape) & 15u)) {
        set_error("%s: tape needs %lld bytes, 16-byte aligned (got %lld)", who, (long long)need, (long long)tape_bytes);
        return INC_E_INVALID;
    }
    return INC_OK;
}

extern "C" int inc_ks_rollout_tape(const inc_ks_plan* p, const float* u0, const float* s, int32_t steps,
                                   float* frames, float* u_final, void* tape, int64_t tape_bytes, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(u0) || steps <= 0) { set_error("ks_rollout_tape: bad arguments"); return INC_E_INVALID; }
    rc = check_tape(p, steps, tape, tape_bytes, "ks_rollout_tape");
    if (rc) return rc;
    a.u = u0; a.s = s; a.steps = steps; a.frames = frames; a.out = u_final; a.tape = static_cast<float2*>(tape);
    return dispatch(Kind::Rollout, p, a, as_stream(stream));
}

extern "C" int inc_ks_rollout_bwd_tape(const inc_ks_plan* p, const void* tape, int64_t tape_bytes, const float* s,
                                       int32_t steps, const float* g_frames, const float* g_final, float* g_u0,
                                       float* g_s, void* stream) {
    Args a;
    int rc = fill_args(p, a);
    if (rc) return rc;
    if (!ok_ptr(g_u0) || steps <= 0) { set_error("ks_rollout_bwd_tape: bad arguments"); return INC_E_INVALID; }
    rc = check_tape(p, steps, tape, tape_bytes, "ks_rollout_bwd_tape");
    if (rc) return rc;
    a.s = s; a.steps = steps; a.tape = const_cast<float2*>(static_cast<const float2*>(tape));
    a.g_frames = g_frames; a.g_final = g_final; a.g_u = g_u0; a.g_s = g_s;
    return dispatch(Kind::TapeBwd, p, a, as_stream(stream));
}
