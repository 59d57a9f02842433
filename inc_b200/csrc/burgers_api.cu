// Burgers C ABI: argument checks and shape dispatch (kernels in burgers_kernels.cuh).
#include <string.h>

#include "burgers_kernels.cuh"

namespace inc {
namespace burgers {

// Default cells-per-lane for a row of n cells.
inline int default_cpt(int n) {
    if (n <= 128) return 4;
    if (n <= 256) return 8;
    return 16;
}

inline bool valid_shape(int n, int cpt) {
    if (!is_pow2(n) || n < 8 || n > 512) return false;
    if (cpt != 4 && cpt != 8 && cpt != 16) return false;
    const int tpr = n / cpt;
    return tpr >= 2 && tpr <= 32;
}

// Threads per block: as many rows per block as keep >= ~2 blocks per SM busy.
inline int pick_block(int rows, int tpr, Kind kind, int n, int K) {
    int block = 256;
    while (block > 32 && (int64_t)rows * tpr / block < 2 * 148) block >>= 1;
    if (block < tpr) block = tpr < 32 ? 32 : tpr;
    if (kind == Kind::RolloutBwd) {
        while (block > 32 && (size_t)(block / tpr) * K * n * 4 > 96 * 1024) block >>= 1;
    }
    return block;
}

int dispatch(Kind kind, const Args& a, int cpt, cudaStream_t st) {
    const int n = a.n;
    const bool fwd = kind == Kind::Step || kind == Kind::Rollout;
    // Small batches: spread each row over a whole CTA (1-2 cells per lane).
    const bool small = a.rows <= 148 && n >= 64;
    if (cpt == 0 && fwd && small) cpt = n >= 256 ? 2 : 1;
    if (!fwd && (cpt == 1 || cpt == 2 || (cpt == 0 && small))) {
        // the adjoints' wide layout has one cell per thread; where it does not
        // apply (n, or a segment too large for shared memory) the warp layouts do
        const int K = kind == Kind::StepBwd ? 1 : a.ckpt_every;
        const size_t seg = (size_t)3 * K * n * sizeof(float);
        if (is_pow2(n) && n >= 64 && n <= 512 && K >= 1) {
#define INC_BW(T) \
            if (n == T && seg + bwd_wide_static_smem<T>() <= 227 * 1024) return launch_bwd_wide<T>(kind, a, st);
            INC_BURGERS_BWD_WIDE_SHAPES(INC_BW)
#undef INC_BW
        }
        cpt = 0;
    }
    if (cpt == 1 || cpt == 2) {
        if (!is_pow2(n) || n < 64 || n / cpt > 512) {
            set_error("burgers: cells_per_thread=%d needs n a power of two with 64 <= n/%d <= 512", cpt, cpt);
            return INC_E_UNSUPPORTED;
        }
        const int tpr = n / cpt;
#define INC_WIDE(C, T) \
        if (cpt == C && tpr == T) return launch_wide<C, T>(kind, a, st);
        INC_BURGERS_WIDE_SHAPES(INC_WIDE)
#undef INC_WIDE
        set_error("burgers: no wide kernel for n=%d cells_per_thread=%d", n, cpt);
        return INC_E_UNSUPPORTED;
    }
    if (cpt == 0) cpt = default_cpt(n);
    if (!valid_shape(n, cpt)) {
        set_error("burgers: unsupported n=%d / cells_per_thread=%d (n must be a power of two in [8,512])", n, cpt);
        return INC_E_UNSUPPORTED;
    }
    const int tpr = n / cpt;
    const int block = pick_block(a.rows, tpr, kind, n, a.ckpt_every);
    const bool bwd = kind == Kind::StepBwd || kind == Kind::RolloutBwd;
#define INC_CASE(C, T) \
    if (cpt == C && tpr == T) return bwd ? launch_bwd<C, T>(kind, a, st, block) : launch_fwd<C, T>(kind, a, st, block);
    INC_BURGERS_SHAPES(INC_CASE)
#undef INC_CASE
    set_error("burgers: no kernel built for n=%d cells_per_thread=%d", n, cpt);
    return INC_E_UNSUPPORTED;
}

int fill_args(const inc_burgers_desc* d, Args& a) {
    memset(&a, 0, sizeof(a));
    if (!d) { set_error("null descriptor"); return INC_E_INVALID; }
    if (d->rows <= 0) { set_error("rows must be positive (got %d)", d->rows); return INC_E_INVALID; }
    if (d->scheme != INC_TS_EULER && d->scheme != INC_TS_SSPRK3) { set_error("unknown time scheme %d", d->scheme); return INC_E_INVALID; }
    if (d->convection != INC_CONV_WENO && d->convection != INC_CONV_FDM) { set_error("Convection scheme not recognized (%d)", d->convection); return INC_E_INVALID; }
    if (d->source < INC_SRC_NONE || d->source > INC_SRC_FORCING) { set_error("Unknown equation type (%d)", d->source); return INC_E_INVALID; }
    if (d->source == INC_SRC_FORCING && (d->forcing == nullptr || d->x == nullptr || d->forcing_terms < 0)) {
        set_error("forcing source needs forcing[rows][4][J] and x[n]"); return INC_E_INVALID;
    }
    if (!(d->dx > 0.f)) { set_error("dx must be positive"); return INC_E_INVALID; }
    a.rows = d->rows; a.n = d->n; a.scheme = d->scheme; a.conv = d->convection; a.src = d->source;
    a.J = d->forcing_terms; a.dx = d->dx; a.inv_dx = 1.f / d->dx; a.inv_dx2 = (float)(1.0 / ((double)d->dx * d->dx));
    a.inv_2dx = (float)(1.0 / (2.0 * d->dx)); a.dt = d->dt; a.nu = d->nu; a.beta = d->beta;
    a.nu_rows = d->nu_rows; a.dt_rows = d->dt_rows; a.beta_rows = d->beta_rows; a.forcing = d->forcing; a.x = d->x;
    return INC_OK;
}

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

extern "C" int inc_weno_reconstruct(const float* f, float* out, int32_t rows, int32_t n, int32_t direction,
                                    void* stream) {
    if (!f || !out || rows <= 0) { set_error("weno: bad arguments"); return INC_E_INVALID; }
    if (direction != 0 && direction != 1) { set_error("Direction must be 'left' or 'right'."); return INC_E_INVALID; }
    if (!aligned16(f) || !aligned16(out)) { set_error("weno: pointers must be 16-byte aligned"); return INC_E_INVALID; }
    const int cpt = default_cpt(n);
    if (!valid_shape(n, cpt)) { set_error("weno: unsupported n=%d (power of two in [8,512])", n); return INC_E_UNSUPPORTED; }
    const int tpr = n / cpt;
    const int block = pick_block(rows, tpr, Kind::Step, n, 0);
    cudaStream_t st = as_stream(stream);
#define INC_W(C, T) \
    if (cpt == C && tpr == T) return launch_weno<C, T>(f, out, rows, n, direction, st, block);
    INC_BURGERS_SHAPES(INC_W)
#undef INC_W
    set_error("weno: no kernel for n=%d", n);
    return INC_E_UNSUPPORTED;
}

extern "C" int inc_burgers_step(const inc_burgers_desc* d, const float* u, const float* s, const float* t_rows,
                                double t0, float* u_out, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!u || !u_out) { set_error("step: null u/u_out"); return INC_E_INVALID; }
    if (!aligned16(u) || !aligned16(u_out) || (s && !aligned16(s))) { set_error("step: pointers must be 16-byte aligned"); return INC_E_INVALID; }
    a.u = u; a.s = s; a.t_rows = t_rows; a.t0 = (float)t0; a.out = u_out;
    return dispatch(Kind::Step, a, d->cells_per_thread, as_stream(stream));
}

extern "C" int inc_burgers_step_bwd(const inc_burgers_desc* d, const float* u, const float* s, const float* t_rows,
                                    double t0, const float* g_out, float* g_u, float* g_s, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!u || !g_out || !g_u) { set_error("step_bwd: null pointer"); return INC_E_INVALID; }
    if (!aligned16(u) || !aligned16(g_out) || !aligned16(g_u) || (g_s && !aligned16(g_s))) { set_error("step_bwd: pointers must be 16-byte aligned"); return INC_E_INVALID; }
    if (s && !aligned16(s)) { set_error("step_bwd: pointers must be 16-byte aligned"); return INC_E_INVALID; }
    a.u = u; a.s = s; a.t_rows = t_rows; a.t0 = (float)t0; a.g_out = g_out; a.g_u = g_u; a.g_s = g_s;
    return dispatch(Kind::StepBwd, a, d->cells_per_thread, as_stream(stream));
}

extern "C" int inc_burgers_rollout(const inc_burgers_desc* d, const float* u0, const float* s, const float* t_rows,
                                   double t0, int32_t steps, float* frames, float* u_final, int32_t ckpt_every,
                                   float* ckpts, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!u0 || steps < 0) { set_error("rollout: bad arguments"); return INC_E_INVALID; }
    if (ckpts && ckpt_every <= 0) { set_error("rollout: ckpt_every must be positive with ckpts"); return INC_E_INVALID; }
    a.u = u0; a.s = s; a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.frames = frames; a.out = u_final;
    a.ckpt_every = ckpt_every; a.ckpts = ckpts;
    return dispatch(Kind::Rollout, a, d->cells_per_thread, as_stream(stream));
}

extern "C" int inc_burgers_rollout_bwd(const inc_burgers_desc* d, const float* ckpts, const float* s,
                                       const float* t_rows, double t0, int32_t steps, int32_t ckpt_every,
                                       const float* g_frames, const float* g_final, float* g_u0, float* g_s,
                                       void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!ckpts || !g_u0 || steps <= 0 || ckpt_every <= 0) { set_error("rollout_bwd: bad arguments"); return INC_E_INVALID; }
    a.u = nullptr; a.s = s; a.t_rows = t_rows; a.t0 = (float)t0; a.steps = steps; a.ckpt_every = ckpt_every;
    a.ckpts = const_cast<float*>(ckpts); a.g_frames = g_frames; a.g_final = g_final; a.g_u = g_u0; a.g_s = g_s;
    return dispatch(Kind::RolloutBwd, a, d->cells_per_thread, as_stream(stream));
}
