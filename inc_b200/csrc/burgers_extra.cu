// Burgers: ragged persistent batch and the reference's term methods.
//
// Ragged batch: rows of different n / nu / dt / dx packed back to back.  A
// persistent grid of warps pulls row indices from one atomic counter
// (fetch-and-add only, no waiting) in the caller's longest-first order; each
// warp advances its row (or, for rows narrower than 128, 32 / (n/4) rows of one
// width, one per lane group) through all steps with the state in registers.
#include "burgers_kernels.cuh"

// The ragged batch evaluates each interface's two WENO reconstructions in packed
// FP32 pairs (weno5_pair); it is issue-bound, not FMA-pipe bound.
#ifndef INC_RAGGED_PACKED
#define INC_RAGGED_PACKED true
#endif

namespace inc {
namespace burgers {

struct RaggedArgs {
    const float* u0;
    float* out;
    const int64_t* offsets;
    const int* n_rows;
    const float* nu_rows;
    const float* dt_rows;
    const float* dx_rows;
    const int* order;
    int* queue;
    int rows, steps, scheme, conv;
};

// Advance this lane's row (row < 0: the lane's group is idle).  Groups of TPR
// lanes are independent: a warp holds 32 / TPR rows of one width at a time.
template <int CPT, int TPR>
INC_DEV void ragged_rows(const RaggedArgs& ra, int row, int lane) {
    const int g = lane % TPR;
    const bool valid = row >= 0;
    const int r = valid ? row : 0;
    const int left = (g + TPR - 1) & (TPR - 1), right = (g + 1) & (TPR - 1);
    Args a;
    memset(&a, 0, sizeof(a));
    a.rows = 1; a.n = CPT * TPR; a.scheme = ra.scheme; a.conv = ra.conv; a.src = INC_SRC_NONE;
    const float dx = __ldg(ra.dx_rows + r);
    a.dx = dx; a.inv_dx = 1.f / dx; a.inv_dx2 = 1.f / (dx * dx); a.inv_2dx = 0.5f / dx;
    Ctx<CPT> cx;
    cx.nu = __ldg(ra.nu_rows + r);
    cx.dt = __ldg(ra.dt_rows + r);
    cx.beta = 0.f; cx.t = 0.f; cx.has_s = false; cx.cell0 = g * CPT; cx.row = r; cx.valid = valid;
#pragma unroll
    for (int c = 0; c < CPT; ++c) cx.s[c] = 0.f;
    const int64_t base = __ldg(ra.offsets + r) + g * CPT;
    float u[CPT], cmp[CPT];  // cmp: compensation carried from step to step (see advance)
    load_row_chunk<CPT>(u, ra.u0 + base, valid);
#pragma unroll
    for (int c = 0; c < CPT; ++c) cmp[c] = 0.f;
    for (int k = 0; k < ra.steps; ++k) advance<CPT, TPR, INC_RAGGED_PACKED>(a, cx, u, cmp, 0.f, left, right);
    store_row_chunk<CPT>(ra.out + base, u, valid);
}

// Rows of width n: one per warp from n = 128 on (4, 8, 16 cells per lane);
// narrower rows (4 cells per lane, n/4 lanes each) fill the warp, one row per
// group of lanes.  `row` is this lane's row (or -1).
INC_DEV void ragged_dispatch(const RaggedArgs& ra, int n, int row, int lane) {
    switch (n) {
        case 8: ragged_rows<4, 2>(ra, row, lane); break;
        case 16: ragged_rows<4, 4>(ra, row, lane); break;
        case 32: ragged_rows<4, 8>(ra, row, lane); break;
        case 64: ragged_rows<4, 16>(ra, row, lane); break;
        case 128: ragged_rows<4, 32>(ra, row, lane); break;
        case 256: ragged_rows<8, 32>(ra, row, lane); break;
        default: ragged_rows<16, 32>(ra, row, lane); break;  // 512 (checked on the host)
    }
}

// Registers uncapped (up to 255 a thread: two blocks of four warps per SM): the rows
// of 512 cells keep 16 cells, their compensation, increments and interface fluxes
// per lane in registers.
__global__ void __launch_bounds__(256, 1) k_ragged(RaggedArgs ra) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(ra.queue, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= ra.rows) break;
        const int row = __ldg(ra.order + item);
        const int n = __ldg(ra.n_rows + row);
        if (n >= 128) {
            ragged_dispatch(ra, n, row, lane);
            continue;
        }
        // Narrow rows: claim per - 1 more items for the other lane groups.  The
        // order is longest first, so they are usually of the same width; any
        // that are not run afterwards, one per warp.
        const int tpr = n / 4, per = 32 / tpr;
        int first = 0;
        if (lane == 0) first = atomicAdd(ra.queue, per - 1);
        first = __shfl_sync(0xffffffffu, first, 0);
        const int j = lane / tpr;
        int mine = -1;
        if (j == 0) {
            mine = row;
        } else if (first + j - 1 < ra.rows) {
            const int r = __ldg(ra.order + first + j - 1);
            if (__ldg(ra.n_rows + r) == n) mine = r;
        }
        ragged_dispatch(ra, n, mine, lane);
        for (int jj = 1; jj < per; ++jj) {
            const int it = first + jj - 1;
            if (it >= ra.rows) break;
            const int r = __ldg(ra.order + it);
            const int nn = __ldg(ra.n_rows + r);
            if (nn == n) continue;
            ragged_dispatch(ra, nn, (lane < (nn >= 128 ? 32 : nn / 4)) ? r : -1, lane);
        }
    }
}

// ---- right-hand-side terms of one state -----------------------------------------
// The reference solver's term methods, each to its own array: calc_nonlinear_weno
// / calc_nonlinear_FDM (solver_1d.py:125-142), calc_linear (:144-146) and
// _compute_source (:104-114, without correction_s).  One CTA per row, one cell
// per thread (n <= 512), the row in shared memory.  The same device functions as
// the step kernels evaluate the fluxes, so the terms agree with what a step adds.
__global__ void __launch_bounds__(512) k_terms(Args a, float* __restrict__ nl_out, float* __restrict__ lin_out,
                                               float* __restrict__ src_out) {
    __shared__ float su[512];
    __shared__ float sh[512];
    __shared__ unsigned smax;
    const int n = a.n, i = threadIdx.x, row = blockIdx.x;
    const int64_t off = (int64_t)row * n + i;
    const float ui = __ldg(a.u + off);
    su[i] = ui;
    if (i == 0) smax = 0u;
    __syncthreads();
    // per-row max |u| (solver_1d.py:133) on the bit patterns: NaN wins, as in torch.max
    atomicMax(&smax, __float_as_uint(fabsf(ui)));
    const int im1 = (i + n - 1) % n, ip1 = (i + 1) % n;
    const float um1 = su[im1], up1 = su[ip1];
    __syncthreads();
    if (nl_out) {
        if (a.conv == INC_CONV_WENO) {
            const float ha = 0.5f * __uint_as_float(smax);
            float fp[7], fm[7];  // cells i-3 .. i+3
#pragma unroll
            for (int k = 0; k < 7; ++k) flux_split(su[(i + k - 3 + 2 * n) % n], ha, fp[k], fm[k]);
            const float h = weno5<false>(fp[1], fp[2], fp[3], fp[4], fp[5]) +
                            weno5<true>(fm[2], fm[3], fm[4], fm[5], fm[6]);
            sh[i] = h;
            __syncthreads();
            nl_out[off] = a.inv_dx * (sh[im1] - h);
        } else {
            nl_out[off] = -ui * ((up1 - um1) * a.inv_2dx);
        }
    }
    const float nu = a.nu_rows ? __ldg(a.nu_rows + row) : a.nu;
    if (lin_out) lin_out[off] = (nu * a.inv_dx2) * fmaf(-2.f, ui, um1 + up1);
    if (src_out) {
        float r = 0.f;
        if (a.src == INC_SRC_LINEAR) {
            r = (a.beta_rows ? __ldg(a.beta_rows + row) : a.beta) * ui;
        } else if (a.src == INC_SRC_FORCING) {
            const float t = a.t_rows ? __ldg(a.t_rows + row) : a.t0;
            const float* fp = a.forcing + (int64_t)row * 4 * a.J;
            const float x = __ldg(a.x + i);
            for (int j = 0; j < a.J; ++j) {
                const float A = __ldg(fp + j), om = __ldg(fp + a.J + j), ph = __ldg(fp + 2 * a.J + j),
                            kx = __ldg(fp + 3 * a.J + j);
                r = fmaf(A, sinf((om * t + kx * x) + ph), r);
            }
        }
        src_out[off] = r;
    }
}

}  // namespace burgers
}  // namespace inc

using namespace inc;
using namespace inc::burgers;

namespace inc {
namespace burgers {
int fill_args(const inc_burgers_desc* d, Args& a);
}
}  // namespace inc

extern "C" int inc_burgers_terms(const inc_burgers_desc* d, const float* u, const float* t_rows, double t0,
                                 float* nonlinear, float* linear, float* source, void* stream) {
    Args a;
    int rc = fill_args(d, a);
    if (rc) return rc;
    if (!u) { set_error("burgers_terms: null u"); return INC_E_INVALID; }
    if (!is_pow2(d->n) || d->n < 8 || d->n > 512) {
        set_error("burgers_terms: n must be a power of two in [8, 512] (got %d)", d->n);
        return INC_E_UNSUPPORTED;
    }
    a.u = u; a.t_rows = t_rows; a.t0 = (float)t0;
    if (!nonlinear && !linear && !source) return INC_OK;
    k_terms<<<d->rows, d->n, 0, as_stream(stream)>>>(a, nonlinear, linear, source);
    return check_launch("burgers_terms");
}

extern "C" int inc_burgers_ragged_rollout(const inc_burgers_ragged_desc* d, const float* u0, int32_t steps,
                                          float* u_final, int32_t* queue, int32_t grid_blocks, void* stream) {
    if (!d || !u0 || !u_final || !queue || !d->offsets || !d->n_rows || !d->nu_rows || !d->dt_rows ||
        !d->dx_rows || !d->order || d->rows <= 0 || steps < 0) {
        set_error("ragged_rollout: bad arguments");
        return INC_E_INVALID;
    }
    if (d->scheme != INC_TS_EULER && d->scheme != INC_TS_SSPRK3) { set_error("unknown time scheme %d", d->scheme); return INC_E_INVALID; }
    if (d->convection != INC_CONV_WENO && d->convection != INC_CONV_FDM) { set_error("Convection scheme not recognized"); return INC_E_INVALID; }
    RaggedArgs ra;
    ra.u0 = u0; ra.out = u_final; ra.offsets = d->offsets; ra.n_rows = d->n_rows; ra.nu_rows = d->nu_rows;
    ra.dt_rows = d->dt_rows; ra.dx_rows = d->dx_rows; ra.order = d->order; ra.queue = queue;
    ra.rows = d->rows; ra.steps = steps; ra.scheme = d->scheme; ra.conv = d->convection;
    const int wpb = d->warps_per_block > 0 ? d->warps_per_block : 4;
    if (wpb > 8) { set_error("ragged_rollout: warps_per_block must be <= 8"); return INC_E_INVALID; }
    const int block = 32 * wpb;
    int grid = grid_blocks;
    if (grid <= 0) {
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ragged, block, 0);
        grid = sms * (per_sm > 0 ? per_sm : 1);
    }
    cudaStream_t st = as_stream(stream);
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int32_t), st);
    if (e != cudaSuccess) { set_error("ragged_rollout: %s", cudaGetErrorString(e)); return INC_E_LAUNCH; }
    k_ragged<<<grid, block, 0, st>>>(ra);
    return check_launch("ragged_rollout");
}
