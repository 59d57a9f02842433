// Burgers WENO5-LF / FDM time stepper for sm_100a: device code and kernels.
//
// Layout: u is [rows][n] FP32.  A row is owned by a group of TPR consecutive
// lanes of one warp (TPR <= 32); lane g of the group holds the CPT contiguous
// cells [g*CPT, g*CPT+CPT) in registers (n = TPR*CPT).  Periodic halos (3 cells
// each side) and the per-row Lax-Friedrichs alpha = max|u| move by warp
// shuffles, so the forward path uses no shared memory and no block barrier.
//
// Reference (tum-pbs/INC solvers/solver_1d.py):
//   weno_reconstruction :4-42, calc_nonlinear_weno :129-142,
//   calc_nonlinear_FDM :125-127, calc_linear :144-146, _compute_delta :74-85,
//   _compute_source :104-114, _apply_corrections :116-123, step :181-195.
#pragma once
#include <string.h>

#include <cooperative_groups.h>

#include "common.cuh"

namespace inc {
namespace burgers {

constexpr float kEps = 1e-6f;  // solver_1d.py:5

// ---------------------------------------------------------------------------
// WENO5 reconstruction on a 5-point window g0..g4.
// 'left' (RIGHT=false): f+ at i+1/2 from f[i-2..i+2]   (solver_1d.py:14-22).
// 'right' (RIGHT=true): f- from f[i-1..i+3]            (solver_1d.py:24-33).
// The two share q0..q2, beta0 and beta1 on the window; they differ only in the
// second term of beta2: (3g2 - 4g3 + g4) for left, (g2 - 4g3 + 3g4) for right.
// ---------------------------------------------------------------------------
// The evaluation uses scaled quantities that need fewer products; the scale
// factors cancel in the normalised weights w_k = alpha_k / sum(alpha):
//   beta'_k = (12/13) beta_k = d_k^2 + (3/13) e_k^2,
//   s'_k    = (12/13) (eps + beta_k) = (12/13) eps + beta'_k,
//   r_k     = 1 / s'_k^2  (= (13/12)^2 / (eps + beta_k)^2),
//   h       = g2 + sum_k (gamma_k dq_k) r_k / sum_k gamma_k r_k,  dq_k = q_k - g2
// (the weights sum to one), with gamma_k folded into the candidates' coefficients
// (qg_k) and everything formed from the first differences D_j = g_{j+1} - g_j.
struct Weno {
    float qg0, qg1, qg2;  // gamma_k (q_k - g2)
    float s0, s1, s2;     // s'_k
    float r0, r1, r2;     // 1 / s'_k^2
    float inv_den, dh;    // dh = h - g2
    float d0, e0, d1, e1, d2, e2;
};

constexpr float kEpsScaled = kEps * (12.f / 13.f);

// 1/x by the hardware reciprocal (PTX rcp.approx.ftz.f32, at most 1 ulp off).
// The WENO denominators are >= (1e-6)^2, far from the subnormal range the
// ftz form flushes; 1/inf = 0 as for a division.
INC_DEV float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <bool RIGHT>
INC_DEV void weno5_eval(float g0, float g1, float g2, float g3, float g4, Weno& w) {
    const float D0 = g1 - g0, D1 = g2 - g1, D2 = g3 - g2, D3 = g4 - g3;
    // gamma = (0.1, 0.6, 0.3); q0 - g2 = -D0/3 + 5 D1/6, q1 - g2 = D1/6 + D2/3,
    // q2 - g2 = 2 D2/3 - D3/6
    w.qg0 = fmaf(-1.f / 30.f, D0, (1.f / 12.f) * D1);
    w.qg1 = fmaf(0.1f, D1, 0.2f * D2);
    w.qg2 = fmaf(0.2f, D2, -0.05f * D3);
    w.d0 = D1 - D0;
    w.d1 = D2 - D1;
    w.d2 = D3 - D2;
    // e0 = g0 - 4 g1 + 3 g2, e1 = g1 - g3, e2 = 3 g2 - 4 g3 + g4 (left) or
    // g2 - 4 g3 + 3 g4 (right), with their signs (the adjoint differentiates them)
    w.e0 = fmaf(3.f, D1, -D0);
    w.e1 = -D1 - D2;
    w.e2 = RIGHT ? fmaf(3.f, D3, -D2) : fmaf(-3.f, D2, D3);
    // s'_k = eps' + d^2 + (3/13) e^2 (beta_k scaled by 12/13), eps folded into the FMA chain
    w.s0 = fmaf(w.d0, w.d0, fmaf((3.f / 13.f) * w.e0, w.e0, kEpsScaled));
    w.s1 = fmaf(w.d1, w.d1, fmaf((3.f / 13.f) * w.e1, w.e1, kEpsScaled));
    w.s2 = fmaf(w.d2, w.d2, fmaf((3.f / 13.f) * w.e2, w.e2, kEpsScaled));
    w.r0 = rcp_approx(w.s0 * w.s0);
    w.r1 = rcp_approx(w.s1 * w.s1);
    w.r2 = rcp_approx(w.s2 * w.s2);
    w.inv_den = rcp_approx(fmaf(0.1f, w.r0, fmaf(0.6f, w.r1, 0.3f * w.r2)));
    w.dh = fmaf(w.qg0, w.r0, fmaf(w.qg1, w.r1, w.qg2 * w.r2)) * w.inv_den;
}

// The reconstruction alone (the forward kernels), in the first differences
// D_j = g_{j+1} - g_j: the candidates as q_k = g2 + dq_k (the weights sum to one,
// so h = g2 + sum w_k dq_k), the smoothness indicators from d_k, e_k of the D's
// (e_k enters squared, so its sign is free).  weno5_eval forms the same
// quantities for the adjoint (weno5_vjp) and keeps them; the two agree up to
// FP32 rounding.
template <bool RIGHT>
INC_DEV float weno5(float g0, float g1, float g2, float g3, float g4) {
    const float D0 = g1 - g0, D1 = g2 - g1, D2 = g3 - g2, D3 = g4 - g3;
    // gamma_k (q_k - g2): gamma = (0.1, 0.6, 0.3); q0 - g2 = -D0/3 + 5 D1/6,
    // q1 - g2 = D1/6 + D2/3, q2 - g2 = 2 D2/3 - D3/6
    const float qg0 = fmaf(-1.f / 30.f, D0, (1.f / 12.f) * D1);
    const float qg1 = fmaf(0.1f, D1, 0.2f * D2);
    const float qg2 = fmaf(0.2f, D2, -0.05f * D3);
    // d_k = second differences; e0 = -(g0 - 4 g1 + 3 g2), e1 = -(g1 - g3); e2: left
    // 3 g2 - 4 g3 + g4 = D3 - 3 D2, right -(g2 - 4 g3 + 3 g4) = D2 - 3 D3
    const float d0 = D1 - D0, d1 = D2 - D1, d2 = D3 - D2;
    const float e0 = fmaf(-3.f, D1, D0);
    const float e1 = D1 + D2;
    const float e2 = RIGHT ? fmaf(1.f, D2, -3.f * D3) : fmaf(-3.f, D2, D3);
    const float s0 = fmaf(d0, d0, fmaf((3.f / 13.f) * e0, e0, kEpsScaled));
    const float s1 = fmaf(d1, d1, fmaf((3.f / 13.f) * e1, e1, kEpsScaled));
    const float s2 = fmaf(d2, d2, fmaf((3.f / 13.f) * e2, e2, kEpsScaled));
    const float r0 = rcp_approx(s0 * s0), r1 = rcp_approx(s1 * s1), r2 = rcp_approx(s2 * s2);
    const float inv = rcp_approx(fmaf(0.1f, r0, fmaf(0.6f, r1, 0.3f * r2)));
    return fmaf(fmaf(qg0, r0, fmaf(qg1, r1, qg2 * r2)), inv, g2);
}

// weno5<false>(g0..g4) + weno5<true>(h0..h4), the two reconstructions of one
// interface evaluated together in the two lanes of Blackwell's packed FP32 pairs
// (fma/add/mul.f32x2: half the issue slots; the reciprocals stay scalar): 36
// packed operations per interface.  Same operations per lane as weno5, so the
// same values.
INC_DEV float2 f2(float a, float b) { return make_float2(a, b); }
INC_DEV float2 f2s(float a) { return make_float2(a, a); }
INC_DEV float2 sub2(float2 a, float2 b) { return __ffma2_rn(f2s(-1.f), b, a); }  // a - b, exactly rounded
INC_DEV float weno5_pair(float g0, float g1, float g2, float g3, float g4, float h0, float h1, float h2, float h3,
                         float h4) {
    const float2 G0 = f2(g0, h0), G1 = f2(g1, h1), G2 = f2(g2, h2), G3 = f2(g3, h3), G4 = f2(g4, h4);
    const float2 D0 = sub2(G1, G0), D1 = sub2(G2, G1), D2 = sub2(G3, G2), D3 = sub2(G4, G3);
    // gamma_k (q_k - g2): gamma = (0.1, 0.6, 0.3); q0 - g2 = -D0/3 + 5 D1/6,
    // q1 - g2 = D1/6 + D2/3, q2 - g2 = 2 D2/3 - D3/6
    const float2 qg0 = __ffma2_rn(f2s(-1.f / 30.f), D0, __fmul2_rn(f2s(1.f / 12.f), D1));
    const float2 qg1 = __ffma2_rn(f2s(0.1f), D1, __fmul2_rn(f2s(0.2f), D2));
    const float2 qg2 = __ffma2_rn(f2s(0.2f), D2, __fmul2_rn(f2s(-0.05f), D3));
    // d_k = second differences; e0 = -(g0 - 4 g1 + 3 g2), e1 = -(g1 - g3); e2: left
    // 3 g2 - 4 g3 + g4 = D3 - 3 D2, right -(g2 - 4 g3 + 3 g4) = D2 - 3 D3
    const float2 d0 = sub2(D1, D0), d1 = sub2(D2, D1), d2 = sub2(D3, D2);
    const float2 e0 = __ffma2_rn(f2s(-3.f), D1, D0);
    const float2 e1 = __fadd2_rn(D1, D2);
    const float2 e2 = __ffma2_rn(f2(-3.f, 1.f), D2, __fmul2_rn(f2(1.f, -3.f), D3));
    const float2 c313 = f2s(3.f / 13.f), eps = f2s(kEpsScaled);
    const float2 s0 = __ffma2_rn(d0, d0, __ffma2_rn(__fmul2_rn(c313, e0), e0, eps));
    const float2 s1 = __ffma2_rn(d1, d1, __ffma2_rn(__fmul2_rn(c313, e1), e1, eps));
    const float2 s2 = __ffma2_rn(d2, d2, __ffma2_rn(__fmul2_rn(c313, e2), e2, eps));
    const float2 q0 = __fmul2_rn(s0, s0), q1 = __fmul2_rn(s1, s1), q2 = __fmul2_rn(s2, s2);
    const float2 r0 = f2(rcp_approx(q0.x), rcp_approx(q0.y)), r1 = f2(rcp_approx(q1.x), rcp_approx(q1.y)),
                 r2 = f2(rcp_approx(q2.x), rcp_approx(q2.y));
    const float2 den = __ffma2_rn(f2s(0.1f), r0, __ffma2_rn(f2s(0.6f), r1, __fmul2_rn(f2s(0.3f), r2)));
    const float2 inv = f2(rcp_approx(den.x), rcp_approx(den.y));
    const float2 h = __ffma2_rn(__ffma2_rn(qg0, r0, __ffma2_rn(qg1, r1, __fmul2_rn(qg2, r2))), inv, G2);
    return h.x + h.y;
}

// Adds hb * d h / d g_m to acc[0..4] (the vector-Jacobian product of weno5), given
// the reconstruction's quantities w (weno5_eval of the same g0..g4).
// With w_k = alpha_k / S:  dh/dq_k = w_k,  dh/dbeta_k = -2 w_k (q_k - h) / (eps + beta_k).
template <bool RIGHT>
INC_DEV void weno5_vjp_tail(const Weno& w, float hb, float& c0, float& c1, float& c2, float& c3, float& c4) {
    const float w0 = 0.1f * w.r0 * w.inv_den, w1 = 0.6f * w.r1 * w.inv_den, w2 = 0.3f * w.r2 * w.inv_den;
    // q_k - h = dq_k - dh
    const float q0 = 10.f * w.qg0, q1 = w.qg1 * (1.f / 0.6f), q2 = w.qg2 * (1.f / 0.3f);
    const float qb0 = hb * w0, qb1 = hb * w1, qb2 = hb * w2;
    // 1 / (eps + beta_k) = (12/13) / s'_k
    const float bb0 = (-24.f / 13.f) * qb0 * (q0 - w.dh) * rcp_approx(w.s0);
    const float bb1 = (-24.f / 13.f) * qb1 * (q1 - w.dh) * rcp_approx(w.s1);
    const float bb2 = (-24.f / 13.f) * qb2 * (q2 - w.dh) * rcp_approx(w.s2);
    // beta_k = 13/12 d^2 + 1/4 e^2  ->  dbeta = 13/6 d dd + 1/2 e de
    const float A0 = 13.f / 6.f * w.d0 * bb0, E0 = 0.5f * w.e0 * bb0;
    const float A1 = 13.f / 6.f * w.d1 * bb1, E1 = 0.5f * w.e1 * bb1;
    const float A2 = 13.f / 6.f * w.d2 * bb2, E2 = 0.5f * w.e2 * bb2;
    // q0 on (g0,g1,g2): (1/3, -7/6, 11/6); beta0: d (1,-2,1), e (1,-4,3)
    c0 += (1.f / 3.f) * qb0 + A0 + E0;
    c1 += (-7.f / 6.f) * qb0 - 2.f * A0 - 4.f * E0;
    c2 += (11.f / 6.f) * qb0 + A0 + 3.f * E0;
    // q1 on (g1,g2,g3): (-1/6, 5/6, 1/3); beta1: d (1,-2,1), e (1,0,-1)
    c1 += (-1.f / 6.f) * qb1 + A1 + E1;
    c2 += (5.f / 6.f) * qb1 - 2.f * A1;
    c3 += (1.f / 3.f) * qb1 + A1 - E1;
    // q2 on (g2,g3,g4): (1/3, 5/6, -1/6); beta2: d (1,-2,1), e left (3,-4,1) / right (1,-4,3)
    c2 += (1.f / 3.f) * qb2 + A2 + (RIGHT ? 1.f : 3.f) * E2;
    c3 += (5.f / 6.f) * qb2 - 2.f * A2 - 4.f * E2;
    c4 += (-1.f / 6.f) * qb2 + A2 + (RIGHT ? 3.f : 1.f) * E2;
}

template <bool RIGHT>
INC_DEV void weno5_vjp(float g0, float g1, float g2, float g3, float g4, float hb,
                       float& c0, float& c1, float& c2, float& c3, float& c4) {
    Weno w;
    weno5_eval<RIGHT>(g0, g1, g2, g3, g4, w);
    weno5_vjp_tail<RIGHT>(w, hb, c0, c1, c2, c3, c4);
}

// Lax-Friedrichs flux splitting of f = u^2 / 2 (solver_1d.py:134-137):
// f+- = (f +- alpha u) / 2 = u (u / 4 +- alpha / 2);  ha = alpha / 2.
INC_DEV void flux_split(float u, float ha, float& fp, float& fm) {
    fp = u * fmaf(0.25f, u, ha);
    fm = u * fmaf(0.25f, u, -ha);
}

// ---------------------------------------------------------------------------
// Per-row context.
// ---------------------------------------------------------------------------
struct Args {
    const float* u;
    const float* s;
    const float* t_rows;
    float* out;
    const float* g_out;  // backward
    float* g_u;
    float* g_s;
    float* frames;
    float* ckpts;
    const float* g_frames;
    const float* g_final;
    const float* nu_rows;
    const float* dt_rows;
    const float* beta_rows;
    const float* forcing;
    const float* x;
    int rows, n, scheme, conv, src, J, steps, ckpt_every;
    float dx, inv_dx, inv_dx2, inv_2dx, dt, nu, beta, t0;
};

template <int CPT>
struct Ctx {
    float nu, dt, beta, t;
    float s[CPT];
    bool has_s;
    int cell0;  // first cell of this lane
    int row;
    bool valid;
};

template <int CPT, int TPR>
INC_DEV void make_ctx(const Args& a, int row, int g, bool valid, Ctx<CPT>& cx) {
    const int r = valid ? row : 0;
    cx.row = r;
    cx.valid = valid;
    cx.cell0 = g * CPT;
    cx.nu = a.nu_rows ? __ldg(a.nu_rows + r) : a.nu;
    cx.dt = a.dt_rows ? __ldg(a.dt_rows + r) : a.dt;
    cx.beta = a.beta_rows ? __ldg(a.beta_rows + r) : a.beta;
    cx.t = a.t_rows ? __ldg(a.t_rows + r) : a.t0;
    cx.has_s = a.s != nullptr;
    if (cx.has_s && CPT % 4 == 0) load_row_chunk<CPT>(cx.s, a.s + (int64_t)r * a.n + cx.cell0, valid);
    else {
#pragma unroll
        for (int c = 0; c < CPT; ++c) cx.s[c] = 0.f;
    }
}

template <int CPT, int TPR>
INC_DEV void halo_window(const float (&u)[CPT], float (&w)[CPT + 6], int left, int right) {
#pragma unroll
    for (int c = 0; c < CPT; ++c) w[c + 3] = u[c];
    w[0] = shfl<TPR>(u[CPT - 3], left);
    w[1] = shfl<TPR>(u[CPT - 2], left);
    w[2] = shfl<TPR>(u[CPT - 1], left);
    w[CPT + 3] = shfl<TPR>(u[0], right);
    w[CPT + 4] = shfl<TPR>(u[1], right);
    w[CPT + 5] = shfl<TPR>(u[2], right);
}

// h+ + h- at the right interface (i + 1/2) of each of the CPT cells of a window
// w (3 halo cells each side), f+- reconstructed at i+1/2 (solver_1d.py:129-142).
// The right-hand side r[c] = -(Dminus f+ + Dminus f-)/dx + nu D2 u (:129-146; the
// dense D2 matmul is the 3-point stencil) also needs the first cell's left
// interface: the previous thread's last right interface, computed there from the
// same row values by the same operations, so the callers hand it over (a shuffle,
// or a shared slot) instead of reconstructing it again.  The r loop stays inline
// at each caller: as a separate function it made the fused CNN kernel 13% slower.
template <int CPT, bool PK = false>
INC_DEV void weno_right_fluxes(const float (&w)[CPT + 6], float alpha, float (&hs)[CPT]) {
    const float ha = 0.5f * alpha;
    float fp[CPT + 6], fm[CPT + 6];
#pragma unroll
    for (int k = 1; k < CPT + 6; ++k) flux_split(w[k], ha, fp[k], fm[k]);
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        if constexpr (PK)
            hs[c] = weno5_pair(fp[c + 1], fp[c + 2], fp[c + 3], fp[c + 4], fp[c + 5], fm[c + 2], fm[c + 3], fm[c + 4],
                               fm[c + 5], fm[c + 6]);
        else
            hs[c] = weno5<false>(fp[c + 1], fp[c + 2], fp[c + 3], fp[c + 4], fp[c + 5]) +
                    weno5<true>(fm[c + 2], fm[c + 3], fm[c + 4], fm[c + 5], fm[c + 6]);
    }
}

// central-difference convection (calc_nonlinear_FDM, solver_1d.py:125-127) + diffusion
template <int CPT>
INC_DEV void fdm_rhs(const float (&w)[CPT + 6], float nu_dx2, float inv_2dx, float (&r)[CPT]) {
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        const float nl = -w[c + 3] * ((w[c + 4] - w[c + 2]) * inv_2dx);
        r[c] = fmaf(nu_dx2, fmaf(-2.f, w[c + 3], w[c + 2] + w[c + 4]), nl);
    }
}

// r = nonlinear + linear (no source): calc_nonlinear_weno / _FDM + calc_linear.
template <int CPT, int TPR, bool PK = false>
INC_DEV void rhs_core(const float (&u)[CPT], float (&r)[CPT], int conv, float nu,
                      float inv_dx, float inv_dx2, float inv_2dx, int left, int right) {
    float w[CPT + 6];
    halo_window<CPT, TPR>(u, w, left, right);
    if (conv == INC_CONV_WENO) {
        float m = 0.f;
#pragma unroll
        for (int c = 0; c < CPT; ++c) m = fmaxf(m, fabsf(u[c]));
        const float alpha = group_max_nonneg<TPR>(m);  // per-row max |u|, solver_1d.py:133
        const float nu_dx2 = nu * inv_dx2;
        if constexpr (CPT <= 8 || PK) {
            float hs[CPT];
            weno_right_fluxes<CPT, PK>(w, alpha, hs);
            float prev = shfl<TPR>(hs[CPT - 1], left);
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const float lap = fmaf(-2.f, w[c + 3], w[c + 2] + w[c + 4]);
                r[c] = fmaf(inv_dx, prev - hs[c], nu_dx2 * lap);
                prev = hs[c];
            }
        } else {
            // 16 cells per lane in the register-bound backward and adaptive kernels:
            // the left interface is reconstructed here (one reconstruction in 17 more
            // than the handover) and the fluxes are consumed as they are made (two live
            // values).  The ragged forward (PK) keeps the handover at 16 cells too: with
            // its registers uncapped that made its rows of 512 cells 9% faster.
            const float ha = 0.5f * alpha;
            float fp[CPT + 6], fm[CPT + 6];
#pragma unroll
            for (int k = 0; k < CPT + 6; ++k) flux_split(w[k], ha, fp[k], fm[k]);
            float prev = PK ? weno5_pair(fp[0], fp[1], fp[2], fp[3], fp[4], fm[1], fm[2], fm[3], fm[4], fm[5])
                            : weno5<false>(fp[0], fp[1], fp[2], fp[3], fp[4]) +
                                  weno5<true>(fm[1], fm[2], fm[3], fm[4], fm[5]);
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const float hs = PK ? weno5_pair(fp[c + 1], fp[c + 2], fp[c + 3], fp[c + 4], fp[c + 5], fm[c + 2],
                                                 fm[c + 3], fm[c + 4], fm[c + 5], fm[c + 6])
                                    : weno5<false>(fp[c + 1], fp[c + 2], fp[c + 3], fp[c + 4], fp[c + 5]) +
                                          weno5<true>(fm[c + 2], fm[c + 3], fm[c + 4], fm[c + 5], fm[c + 6]);
                const float lap = fmaf(-2.f, w[c + 3], w[c + 2] + w[c + 4]);
                r[c] = fmaf(inv_dx, prev - hs, nu_dx2 * lap);
                prev = hs;
            }
        }
    } else {
        fdm_rhs<CPT>(w, nu * inv_dx2, inv_2dx, r);
    }
}

// r += source(u, t) + correction s (solver_1d.py:104-123).
template <int CPT>
INC_DEV void add_source(const Args& a, const Ctx<CPT>& cx, const float (&u)[CPT], float (&r)[CPT], float t) {
    if (a.src == INC_SRC_LINEAR) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) r[c] = fmaf(cx.beta, u[c], r[c]);
    } else if (a.src == INC_SRC_FORCING) {
        const float* fp = a.forcing + (int64_t)cx.row * 4 * a.J;
        for (int j = 0; j < a.J; ++j) {
            const float A = __ldg(fp + j), om = __ldg(fp + a.J + j), ph = __ldg(fp + 2 * a.J + j),
                        kx = __ldg(fp + 3 * a.J + j);
            const float wt = om * t;
#pragma unroll
            for (int c = 0; c < CPT; ++c) {
                const float x = __ldg(a.x + cx.cell0 + c);
                r[c] = fmaf(A, sinf((wt + kx * x) + ph), r[c]);
            }
        }
    }
    if (cx.has_s) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) r[c] += cx.s[c];
    }
}

template <int CPT, int TPR, bool PK = false>
INC_DEV void full_rhs(const Args& a, const Ctx<CPT>& cx, const float (&u)[CPT], float (&r)[CPT], float t,
                      int left, int right) {
    rhs_core<CPT, TPR, PK>(u, r, a.conv, cx.nu, a.inv_dx, a.inv_dx2, a.inv_2dx, left, right);
    add_source<CPT>(a, cx, u, r, t);
}

// u_new = u0 + d with compensated summation: cmp holds the rounding error of
// earlier updates (zero for a single step) and receives this one's.
INC_DEV void step_update(float u0, float d, float& cmp, float& u_new) {
    const float y = d + cmp;
    u_new = u0 + y;
    cmp = y - (u_new - u0);
}

// Shu-Osher SSP-RK3 as stage coefficients: stage k evaluates the RHS at
// t + kC[k] dt on the current stage value u and sets u = kA[k] u0 + kB[k] (u + dt R).
INC_DEV float rk3_c(int k) { return k == 0 ? 0.f : (k == 1 ? 1.f : 0.5f); }
INC_DEV float rk3_a(int k) { return k == 0 ? 0.f : (k == 1 ? 0.75f : 1.f / 3.f); }
INC_DEV float rk3_b(int k) { return k == 0 ? 1.f : (k == 1 ? 0.25f : 2.f / 3.f); }

// One step (Euler or SSP-RK3) of size cx.dt starting at time t, in increment
// form: d_1 = dt R(u), d_{k+1} = b_k (d_k + dt R(u + d_k)), u_new = u + d_S.
// These are the Shu-Osher stages u_{k+1} = a_k u + b_k (u_k + dt R(u_k)) with
// a_k = 1 - b_k; the increments are small, so they keep their relative
// precision, and the one rounding left is the final u + d.  Fused rollouts
// carry that rounding error to the next step in `cmp` (compensated summation):
// without it, FP32 rounding of the update accumulates over a rollout, by 1.8e-5
// relative L2 after 500 SSP-RK3 steps of the ragged benchmark rows (6e-8 with
// it).  The stages run as a loop around one copy of the right-hand side
// (instruction cache).
template <int CPT, int TPR, bool PK = false>
INC_DEV void advance(const Args& a, const Ctx<CPT>& cx, float (&u)[CPT], float (&cmp)[CPT], float t, int left,
                     int right) {
    float r[CPT], u0[CPT], d[CPT];
    const float dt = cx.dt;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
#pragma unroll
    for (int c = 0; c < CPT; ++c) { u0[c] = u[c]; d[c] = 0.f; }
#pragma unroll 1
    for (int k = 0; k < stages; ++k) {
        full_rhs<CPT, TPR, PK>(a, cx, u, r, t + rk3_c(k) * dt, left, right);
        const float kb = rk3_b(k);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            d[c] = kb * fmaf(dt, r[c], d[c]);
            u[c] = u0[c] + d[c];
        }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) step_update(u0[c], d[c], cmp[c], u[c]);
}

// A step without a carried compensation (single steps, segment replays).
template <int CPT, int TPR>
INC_DEV void advance(const Args& a, const Ctx<CPT>& cx, float (&u)[CPT], float t, int left, int right) {
    float cmp[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) cmp[c] = 0.f;
    advance<CPT, TPR>(a, cx, u, cmp, t, left, right);
}

// out = J(u)^T v for the spatial operator (nonlinear + linear + beta*u source).
template <int CPT, int TPR>
INC_DEV void rhs_vjp(const Args& a, const Ctx<CPT>& cx, const float (&u)[CPT], const float (&v)[CPT],
                     float (&out)[CPT], int g, int left, int right) {
    float w[CPT + 6];
    halo_window<CPT, TPR>(u, w, left, right);
    const float v_r = shfl<TPR>(v[0], right);
    const float v_l = shfl<TPR>(v[CPT - 1], left);
    const float nu = cx.nu;
    if (a.conv == INC_CONV_WENO) {
        float m = 0.f;  // as the forward's fmaxf: NaN cells are passed over
        int mi = g * CPT;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            const float av = fabsf(u[c]);
            if (av > m) { m = av; mi = g * CPT + c; }
        }
        group_argmax_nonneg<TPR>(m, mi);
        const float alpha = m;
        float fp[CPT + 6], fm[CPT + 6];
#pragma unroll
        for (int k = 0; k < CPT + 6; ++k) flux_split(w[k], 0.5f * alpha, fp[k], fm[k]);
        float accp[CPT + 5], accm[CPT + 5];  // index e <-> cell cell0 - 2 + e
#pragma unroll
        for (int e = 0; e < CPT + 5; ++e) { accp[e] = 0.f; accm[e] = 0.f; }
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            const float vn = (c + 1 < CPT) ? v[c + 1] : v_r;
            // hp[i] enters R[i] with -1/dx and R[i+1] with +1/dx (same for hm).
            const float hb = (vn - v[c]) * a.inv_dx;
            weno5_vjp<false>(fp[c + 1], fp[c + 2], fp[c + 3], fp[c + 4], fp[c + 5], hb,
                             accp[c], accp[c + 1], accp[c + 2], accp[c + 3], accp[c + 4]);
            weno5_vjp<true>(fm[c + 2], fm[c + 3], fm[c + 4], fm[c + 5], fm[c + 6], hb,
                            accm[c + 1], accm[c + 2], accm[c + 3], accm[c + 4], accm[c + 5]);
        }
        float ub[CPT + 5];
        float abar = 0.f;
#pragma unroll
        for (int e = 0; e < CPT + 5; ++e) {
            const float uj = w[e + 1];
            ub[e] = accp[e] * (0.5f * (uj + alpha)) + accm[e] * (0.5f * (uj - alpha));
            abar += 0.5f * uj * (accp[e] - accm[e]);
        }
        const float fl0 = shfl<TPR>(ub[CPT + 2], left), fl1 = shfl<TPR>(ub[CPT + 3], left),
                    fl2 = shfl<TPR>(ub[CPT + 4], left);
        const float fr0 = shfl<TPR>(ub[0], right), fr1 = shfl<TPR>(ub[1], right);
#pragma unroll
        for (int c = 0; c < CPT; ++c) out[c] = ub[c + 2];
        out[0] += fl0;
        out[1] += fl1;
        out[2] += fl2;
        out[CPT - 2] += fr0;
        out[CPT - 1] += fr1;
        abar = group_sum<TPR>(abar);
        // alpha = |u[argmax]|: d|u|/du = sign(u) (torch.abs backward, 0 at 0)
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            if (g * CPT + c == mi) {
                const float sg = u[c] > 0.f ? 1.f : (u[c] < 0.f ? -1.f : 0.f);
                out[c] = fmaf(abar, sg, out[c]);
            }
        }
    } else {
        // R_i = -u_i (u_{i+1} - u_{i-1}) / (2 dx)
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            const float vm = c > 0 ? v[c - 1] : v_l;
            const float vp = c + 1 < CPT ? v[c + 1] : v_r;
            out[c] = -v[c] * ((w[c + 4] - w[c + 2]) * a.inv_2dx) - vm * w[c + 2] * a.inv_2dx +
                     vp * w[c + 4] * a.inv_2dx;
        }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) {
        const float vm = c > 0 ? v[c - 1] : v_l;
        const float vp = c + 1 < CPT ? v[c + 1] : v_r;
        out[c] += nu * ((vm - 2.f * v[c] + vp) * a.inv_dx2);
        if (a.src == INC_SRC_LINEAR) out[c] = fmaf(cx.beta, v[c], out[c]);
    }
}

// Backward of `advance`: given gu = dL/du_new (in), returns dL/du in gu and
// accumulates dL/ds into gs.  Stage k maps u_k to
// u_{k+1} = a_k u + b_k (u_k + dt R(u_k)), so in reverse:
//   dL/du_k = b_k (g + dt J(u_k)^T g),  dL/du += a_k g,  dL/ds += b_k dt g.
// The stage inputs u_1, u_2 are replayed from u first.
template <int CPT, int TPR>
INC_DEV void advance_bwd(const Args& a, const Ctx<CPT>& cx, const float (&u)[CPT], float (&gu)[CPT],
                         float (&gs)[CPT], float t, int g, int left, int right) {
    const float dt = cx.dt;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    float u1[CPT], u2[CPT], x[CPT], r[CPT], d[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) { x[c] = u[c]; u1[c] = u[c]; u2[c] = u[c]; d[c] = 0.f; }
#pragma unroll 1
    for (int k = 0; k + 1 < stages; ++k) {  // replay u_1, u_2 (as advance)
        full_rhs<CPT, TPR>(a, cx, x, r, t + rk3_c(k) * dt, left, right);
        const float kb = rk3_b(k);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            d[c] = kb * fmaf(dt, r[c], d[c]);
            x[c] = u[c] + d[c];
            if (k == 0) u1[c] = x[c];
            else u2[c] = x[c];
        }
    }
    float acc[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) acc[c] = 0.f;
#pragma unroll 1
    for (int k = stages - 1; k >= 0; --k) {
#pragma unroll
        for (int c = 0; c < CPT; ++c) x[c] = k == 2 ? u2[c] : (k == 1 ? u1[c] : u[c]);
        rhs_vjp<CPT, TPR>(a, cx, x, gu, r, g, left, right);
        const float ka = rk3_a(k), kb = rk3_b(k);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            gs[c] += kb * dt * gu[c];
            acc[c] += ka * gu[c];
            gu[c] = kb * (gu[c] + dt * r[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) gu[c] += acc[c];
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
template <int CPT, int TPR>
INC_DEV void lane_setup(int& row, int& g, int& left, int& right, bool& valid, int rows) {
    const int rpb = blockDim.x / TPR;
    row = blockIdx.x * rpb + threadIdx.x / TPR;
    g = threadIdx.x % TPR;
    left = (g + TPR - 1) & (TPR - 1);
    right = (g + 1) & (TPR - 1);
    valid = row < rows;
}

template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_step(Args a) {
    int row, g, left, right;
    bool valid;
    lane_setup<CPT, TPR>(row, g, left, right, valid, a.rows);
    Ctx<CPT> cx;
    make_ctx<CPT, TPR>(a, row, g, valid, cx);
    float u[CPT];
    const int64_t base = (int64_t)row * a.n + g * CPT;
    load_row_chunk<CPT>(u, a.u + base, valid);
    advance<CPT, TPR>(a, cx, u, cx.t, left, right);
    store_row_chunk<CPT>(a.out + base, u, valid);
}

template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_step_bwd(Args a) {
    int row, g, left, right;
    bool valid;
    lane_setup<CPT, TPR>(row, g, left, right, valid, a.rows);
    Ctx<CPT> cx;
    make_ctx<CPT, TPR>(a, row, g, valid, cx);
    float u[CPT], gu[CPT], gs[CPT];
    const int64_t base = (int64_t)row * a.n + g * CPT;
    load_row_chunk<CPT>(u, a.u + base, valid);
    load_row_chunk<CPT>(gu, a.g_out + base, valid);
#pragma unroll
    for (int c = 0; c < CPT; ++c) gs[c] = 0.f;
    advance_bwd<CPT, TPR>(a, cx, u, gu, gs, cx.t, g, left, right);
    store_row_chunk<CPT>(a.g_u + base, gu, valid);
    if (a.g_s) store_row_chunk<CPT>(a.g_s + base, gs, valid);
}

// Fused rollout: `steps` steps with the state in registers.
template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_rollout(Args a) {
    int row, g, left, right;
    bool valid;
    lane_setup<CPT, TPR>(row, g, left, right, valid, a.rows);
    Ctx<CPT> cx;
    make_ctx<CPT, TPR>(a, row, g, valid, cx);
    float u[CPT];
    const int64_t base = (int64_t)row * a.n + g * CPT;
    load_row_chunk<CPT>(u, a.u + base, valid);
    float cmp[CPT];  // compensation carried from step to step (see advance)
#pragma unroll
    for (int c = 0; c < CPT; ++c) cmp[c] = 0.f;
    const int nseg = a.ckpt_every > 0 ? (a.steps + a.ckpt_every - 1) / a.ckpt_every : 0;
    for (int k = 0; k < a.steps; ++k) {
        if (a.ckpts && k % a.ckpt_every == 0)
            store_row_chunk<CPT>(a.ckpts + ((int64_t)row * nseg + k / a.ckpt_every) * a.n + g * CPT, u, valid);
        advance<CPT, TPR>(a, cx, u, cmp, cx.t + k * cx.dt, left, right);
        if (a.frames) store_row_chunk_cs<CPT>(a.frames + ((int64_t)row * a.steps + k) * a.n + g * CPT, u, valid);
    }
    if (a.out) store_row_chunk<CPT>(a.out + base, u, valid);
}

// Backward of the fused rollout.  Segments of ckpt_every steps are replayed
// from their checkpoint; the replayed states of one segment live in shared
// memory laid out [state][c][lane] so that lanes access consecutive words.
template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_rollout_bwd(Args a) {
    extern __shared__ float sm[];
    int row, g, left, right;
    bool valid;
    lane_setup<CPT, TPR>(row, g, left, right, valid, a.rows);
    Ctx<CPT> cx;
    make_ctx<CPT, TPR>(a, row, g, valid, cx);
    const int K = a.ckpt_every;
    const int n = a.n;
    float* seg = sm + (threadIdx.x / TPR) * (K * n);
    const int nseg = (a.steps + K - 1) / K;
    float gu[CPT], gs[CPT];
    const int64_t base = (int64_t)row * n + g * CPT;
    if (a.g_final) load_row_chunk<CPT>(gu, a.g_final + base, valid);
    else {
#pragma unroll
        for (int c = 0; c < CPT; ++c) gu[c] = 0.f;
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) gs[c] = 0.f;
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        float u[CPT];
        load_row_chunk<CPT>(u, a.ckpts + ((int64_t)row * nseg + sidx) * n + g * CPT, valid);
        for (int j = 0; j < len; ++j) {
#pragma unroll
            for (int c = 0; c < CPT; ++c) seg[j * n + c * TPR + g] = u[c];
            if (j + 1 < len) advance<CPT, TPR>(a, cx, u, cx.t + (k0 + j) * cx.dt, left, right);
        }
        for (int j = len - 1; j >= 0; --j) {
            const int k = k0 + j;
            if (a.g_frames) {
                float gf[CPT];
                load_row_chunk<CPT>(gf, a.g_frames + ((int64_t)row * a.steps + k) * n + g * CPT, valid);
#pragma unroll
                for (int c = 0; c < CPT; ++c) gu[c] += gf[c];
            }
#pragma unroll
            for (int c = 0; c < CPT; ++c) u[c] = seg[j * n + c * TPR + g];
            advance_bwd<CPT, TPR>(a, cx, u, gu, gs, cx.t + k * cx.dt, g, left, right);
        }
    }
    store_row_chunk<CPT>(a.g_u + base, gu, valid);
    if (a.g_s) store_row_chunk<CPT>(a.g_s + base, gs, valid);
}

// ---------------------------------------------------------------------------
// Wide rows: one CTA per row, TPR = n / CPT lanes (64..512), CPT = 1 or 2
// cells per lane.  For small batches this spreads a row over more lanes so a
// step's dependency chain is shorter.  Halos and the alpha row max go through
// a shared row buffer, double-buffered by RHS evaluation so that one block
// barrier per evaluation suffices.
// ---------------------------------------------------------------------------
template <int CPT, int TPR>
struct WideSmem {
    float row[2][CPT * TPR];
    float wmax[2][TPR / 32];
    int warg[2][TPR / 32];  // (ARG) each warp's first cell of its max |u|
    float flux[2][TPR];  // each thread's last right-interface flux sum, read by its right neighbour
};


// The barrier of the threads that run one row: the whole CTA (BAR = 0), or one of
// the two thread groups of the warp-specialised adjoint (named barrier BAR over NT
// threads).
template <int BAR, int NT>
INC_DEV void row_sync() {
    if constexpr (BAR == 0) __syncthreads();
    else asm volatile("bar.sync %0, %1;\n" ::"n"(BAR), "n"(NT) : "memory");
}

// ARG: also the row's first cell of max |u| (as the adjoint picks it); thread 0
// writes alpha and that cell (as int bits) to arg_out[0], arg_out[1] (WENO only).
template <int CPT, int TPR, int BAR = 0, bool ARG = false>
INC_DEV void rhs_core_wide(const float (&u)[CPT], float (&r)[CPT], int conv, float nu, float inv_dx, float inv_dx2,
                           float inv_2dx, WideSmem<CPT, TPR>& sh, int parity, int g, float* arg_out = nullptr) {
    constexpr int N = CPT * TPR;
    float* row = sh.row[parity];
#pragma unroll
    for (int c = 0; c < CPT; ++c) row[g * CPT + c] = u[c];
    float m = 0.f;
    if constexpr (ARG) {  // as fmaxf: a NaN cell is passed over
        int mi = g * CPT;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            const float av = fabsf(u[c]);
            if (av > m) { m = av; mi = g * CPT + c; }
        }
        group_argmax_nonneg<32>(m, mi);
        if ((g & 31) == 0) {
            sh.wmax[parity][g >> 5] = m;
            sh.warg[parity][g >> 5] = mi;
        }
    } else {
#pragma unroll
        for (int c = 0; c < CPT; ++c) m = fmaxf(m, fabsf(u[c]));
        m = group_max_nonneg<32>(m);
        if ((g & 31) == 0) sh.wmax[parity][g >> 5] = m;
    }
    row_sync<BAR, TPR>();
    float w[CPT + 6];
#pragma unroll
    for (int k = 0; k < CPT + 6; ++k) w[k] = row[(g * CPT - 3 + k + N) & (N - 1)];
    if (conv == INC_CONV_WENO) {
        float alpha = 0.f;
#pragma unroll
        for (int i = 0; i < TPR / 32; ++i) alpha = fmaxf(alpha, sh.wmax[parity][i]);
        if constexpr (ARG) {
            if (g == 0) {
                float best = sh.wmax[parity][0];
                int am = sh.warg[parity][0];
#pragma unroll
                for (int i = 1; i < TPR / 32; ++i)
                    if (sh.wmax[parity][i] > best) {
                        best = sh.wmax[parity][i];
                        am = sh.warg[parity][i];
                    }
                arg_out[0] = alpha;
                arg_out[1] = __int_as_float(am);
            }
        }
        // the first cell's left interface from the previous thread, after one barrier
        float hs[CPT];
        weno_right_fluxes<CPT>(w, alpha, hs);
        sh.flux[parity][g] = hs[CPT - 1];
        row_sync<BAR, TPR>();
        float prev = sh.flux[parity][(g + TPR - 1) % TPR];
        const float nu_dx2 = nu * inv_dx2;
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            const float lap = fmaf(-2.f, w[c + 3], w[c + 2] + w[c + 4]);
            r[c] = fmaf(inv_dx, prev - hs[c], nu_dx2 * lap);
            prev = hs[c];
        }
    } else {
        fdm_rhs<CPT>(w, nu * inv_dx2, inv_2dx, r);
    }
}

template <int CPT, int TPR, int BAR = 0, bool ARG = false>
INC_DEV void full_rhs_wide(const Args& a, const Ctx<CPT>& cx, const float (&x)[CPT], float (&r)[CPT], float t,
                           WideSmem<CPT, TPR>& sh, int& parity, int g, float* arg_out = nullptr) {
    rhs_core_wide<CPT, TPR, BAR, ARG>(x, r, a.conv, cx.nu, a.inv_dx, a.inv_dx2, a.inv_2dx, sh, parity, g, arg_out);
    parity ^= 1;
    add_source<CPT>(a, cx, x, r, t);
}

// The wide layout serves small, latency-bound batches: its stages stay
// unrolled (straight-line code schedules better; one row per CTA keeps the
// code footprint per SM small).  Increment form and carried compensation as
// in advance.
template <int CPT, int TPR>
INC_DEV void advance_wide(const Args& a, const Ctx<CPT>& cx, float (&u)[CPT], float (&cmp)[CPT], float t,
                          WideSmem<CPT, TPR>& sh, int& parity, int g) {
    float r[CPT], u0[CPT], d[CPT];
    const float dt = cx.dt;
#pragma unroll
    for (int c = 0; c < CPT; ++c) u0[c] = u[c];
    if (a.scheme == INC_TS_EULER) {
        full_rhs_wide<CPT, TPR>(a, cx, u, r, t, sh, parity, g);
#pragma unroll
        for (int c = 0; c < CPT; ++c) step_update(u0[c], dt * r[c], cmp[c], u[c]);
        return;
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) d[c] = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        full_rhs_wide<CPT, TPR>(a, cx, u, r, t + rk3_c(k) * dt, sh, parity, g);
        const float kb = rk3_b(k);
#pragma unroll
        for (int c = 0; c < CPT; ++c) {
            d[c] = kb * fmaf(dt, r[c], d[c]);
            u[c] = u0[c] + d[c];
        }
    }
#pragma unroll
    for (int c = 0; c < CPT; ++c) step_update(u0[c], d[c], cmp[c], u[c]);
}

template <int CPT, int TPR>
INC_DEV void advance_wide(const Args& a, const Ctx<CPT>& cx, float (&u)[CPT], float t, WideSmem<CPT, TPR>& sh,
                          int& parity, int g) {
    float cmp[CPT];
#pragma unroll
    for (int c = 0; c < CPT; ++c) cmp[c] = 0.f;
    advance_wide<CPT, TPR>(a, cx, u, cmp, t, sh, parity, g);
}

// ---- wide-row adjoint (one cell per thread, TPR threads per row) -----------------
// Shared scratch: the forward's row buffers (stage replays) and the adjoint's
// rows, contributions and per-warp reductions.
template <int TPR>
struct WideAdjSmem {
    WideSmem<1, TPR> fw;
    float urow[TPR];   // u of the stage being differentiated
    float vrow[TPR];   // the adjoint vector v
    float ub[6][TPR];  // ub[e][i]: cell i's contribution to cell i - 2 + e
    float wmax[TPR / 32];
    int warg[TPR / 32];
    float wsum[TPR / 32];
};

// out = J(u)^T v at this thread's cell: rhs_vjp for one cell per thread, the
// halos, the row max |u| with its first argmax (alpha's gradient) and the
// neighbours' contributions through shared memory (two block barriers).
template <int TPR, int BAR = 0>
INC_DEV void rhs_vjp_wide(const Args& a, const Ctx<1>& cx, float u, float v, float& out, WideAdjSmem<TPR>& sh,
                          int g) {
    constexpr int N = TPR, NW = TPR / 32;
    const int lane = g & 31, warp = g >> 5;
    sh.urow[g] = u;
    sh.vrow[g] = v;
    const bool weno = a.conv == INC_CONV_WENO;
    if (weno) {  // as the forward's fmaxf: a NaN cell is passed over
        const float au = fabsf(u);
        float m = au > 0.f ? au : 0.f;
        int mi = g;
        group_argmax_nonneg<32>(m, mi);
        if (lane == 0) {
            sh.wmax[warp] = m;
            sh.warg[warp] = mi;
        }
    }
    row_sync<BAR, TPR>();
    float w[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) w[k] = sh.urow[(g - 3 + k + N) & (N - 1)];
    const float v_r = sh.vrow[(g + 1) & (N - 1)], v_l = sh.vrow[(g + N - 1) & (N - 1)];
    float alpha = 0.f;
    int am = 0;
    if (weno) {
        alpha = sh.wmax[0];
        am = sh.warg[0];
#pragma unroll
        for (int i = 1; i < NW; ++i)
            if (sh.wmax[i] > alpha) {
                alpha = sh.wmax[i];
                am = sh.warg[i];
            }
        float fp[7], fm[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) flux_split(w[k], 0.5f * alpha, fp[k], fm[k]);
        float accp[6], accm[6];  // index e <-> cell g - 2 + e
#pragma unroll
        for (int e = 0; e < 6; ++e) { accp[e] = 0.f; accm[e] = 0.f; }
        // hp at g + 1/2 enters R[g] with -1/dx and R[g+1] with +1/dx (same for hm)
        const float hb = (v_r - v) * a.inv_dx;
        weno5_vjp<false>(fp[1], fp[2], fp[3], fp[4], fp[5], hb, accp[0], accp[1], accp[2], accp[3], accp[4]);
        weno5_vjp<true>(fm[2], fm[3], fm[4], fm[5], fm[6], hb, accm[1], accm[2], accm[3], accm[4], accm[5]);
        float abar = 0.f;
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const float uj = w[e + 1];
            sh.ub[e][g] = accp[e] * (0.5f * (uj + alpha)) + accm[e] * (0.5f * (uj - alpha));
            abar += 0.5f * uj * (accp[e] - accm[e]);
        }
        abar = group_sum<32>(abar);
        if (lane == 0) sh.wsum[warp] = abar;
    }
    row_sync<BAR, TPR>();
    if (weno) {
        out = sh.ub[0][(g + 2) & (N - 1)] + sh.ub[1][(g + 1) & (N - 1)] + sh.ub[2][g] +
              sh.ub[3][(g + N - 1) & (N - 1)] + sh.ub[4][(g + N - 2) & (N - 1)] + sh.ub[5][(g + N - 3) & (N - 1)];
        if (g == am) {  // alpha = |u[argmax]|: d|u|/du = sign(u) (torch.abs backward, 0 at 0)
            float abar = 0.f;
#pragma unroll
            for (int i = 0; i < NW; ++i) abar += sh.wsum[i];
            const float sg = u > 0.f ? 1.f : (u < 0.f ? -1.f : 0.f);
            out = fmaf(abar, sg, out);
        }
    } else {  // R_i = -u_i (u_{i+1} - u_{i-1}) / (2 dx)
        out = -v * ((w[4] - w[2]) * a.inv_2dx) - v_l * w[2] * a.inv_2dx + v_r * w[4] * a.inv_2dx;
    }
    out += cx.nu * ((v_l - 2.f * v + v_r) * a.inv_dx2);
    if (a.src == INC_SRC_LINEAR) out = fmaf(cx.beta, v, out);
}

// rhs_vjp_wide with its v-independent part done ahead.  At one cell the WENO part
// of J(u)^T v is linear in hb = (v[g+1] - v[g]) / dx, the adjoint of the
// interface flux g + 1/2 this cell owns: the contributions to cells g-2 .. g+3
// are hb * m[e] and to alpha hb * pa.  vjp_pre forms m, pa from the stage input's
// window and its alpha / first argmax (recorded by the segment replay); the
// stage then scales and scatters them.
struct VjpPre {
    float m[6];  // d(hp + hm)/du at cells g-2 .. g+3 through the flux split
    float pa;    // d(hp + hm)/dalpha
    float u_l, u, u_r;  // the stage input at cells g-1, g, g+1
    int am;
};

// stage input row `row` (in shared memory, read with the row's period) and its
// recorded alpha / argmax al[0], al[1]
template <int TPR>
INC_DEV void vjp_pre(const Args& a, const float* row, const float* al, int g, VjpPre& p) {
    constexpr int N = TPR;
    float w[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) w[k] = row[(g - 3 + k + N) & (N - 1)];
    p.u_l = w[2];
    p.u = w[3];
    p.u_r = w[4];
    if (a.conv == INC_CONV_WENO) {
        const float alpha = al[0];
        p.am = __float_as_int(al[1]);
        float fp[7], fm[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) flux_split(w[k], 0.5f * alpha, fp[k], fm[k]);
        Weno wl, wr;
        weno5_eval<false>(fp[1], fp[2], fp[3], fp[4], fp[5], wl);
        weno5_eval<true>(fm[2], fm[3], fm[4], fm[5], fm[6], wr);
        float kp[6], km[6];  // dh+/df+ and dh-/df- at cells g-2 .. g+3 (hb = 1)
#pragma unroll
        for (int e = 0; e < 6; ++e) { kp[e] = 0.f; km[e] = 0.f; }
        weno5_vjp_tail<false>(wl, 1.f, kp[0], kp[1], kp[2], kp[3], kp[4]);
        weno5_vjp_tail<true>(wr, 1.f, km[1], km[2], km[3], km[4], km[5]);
        float pa = 0.f;
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const float uj = w[e + 1];  // f+- = u (u/4 +- alpha/2)
            p.m[e] = kp[e] * (0.5f * (uj + alpha)) + km[e] * (0.5f * (uj - alpha));
            pa += 0.5f * uj * (kp[e] - km[e]);
        }
        p.pa = pa;
    }
}

// out = J(u)^T v at this thread's cell from the precomputed p (rhs_vjp_wide's
// values up to FP32 rounding).  `ahead` runs between the two barriers, beside
// this stage's arithmetic: the caller's precomputation for the next stage.
template <int TPR, int BAR, typename AHEAD>
INC_DEV void rhs_vjp_wide_pre(const Args& a, const Ctx<1>& cx, const VjpPre& p, float v, float& out,
                              WideAdjSmem<TPR>& sh, int g, AHEAD&& ahead) {
    constexpr int N = TPR, NW = TPR / 32;
    const int lane = g & 31, warp = g >> 5;
    sh.vrow[g] = v;
    row_sync<BAR, TPR>();
    const float v_r = sh.vrow[(g + 1) & (N - 1)], v_l = sh.vrow[(g + N - 1) & (N - 1)];
    const bool weno = a.conv == INC_CONV_WENO;
    if (weno) {
        const float hb = (v_r - v) * a.inv_dx;
#pragma unroll
        for (int e = 0; e < 6; ++e) sh.ub[e][g] = hb * p.m[e];
        const float abar = group_sum<32>(hb * p.pa);
        if (lane == 0) sh.wsum[warp] = abar;
    }
    ahead();
    row_sync<BAR, TPR>();
    if (weno) {
        out = sh.ub[0][(g + 2) & (N - 1)] + sh.ub[1][(g + 1) & (N - 1)] + sh.ub[2][g] +
              sh.ub[3][(g + N - 1) & (N - 1)] + sh.ub[4][(g + N - 2) & (N - 1)] + sh.ub[5][(g + N - 3) & (N - 1)];
        if (g == p.am) {  // alpha = |u[argmax]|: d|u|/du = sign(u)
            float abar = 0.f;
#pragma unroll
            for (int i = 0; i < NW; ++i) abar += sh.wsum[i];
            const float sg = p.u > 0.f ? 1.f : (p.u < 0.f ? -1.f : 0.f);
            out = fmaf(abar, sg, out);
        }
    } else {
        out = -v * ((p.u_r - p.u_l) * a.inv_2dx) - v_l * p.u_l * a.inv_2dx + v_r * p.u_r * a.inv_2dx;
    }
    out += cx.nu * ((v_l - 2.f * v + v_r) * a.inv_dx2);
    if (a.src == INC_SRC_LINEAR) out = fmaf(cx.beta, v, out);
}

// The stages' adjoints in reverse (see advance_bwd) for one cell per thread,
// given the step's stage inputs u, u1, u2 (u1, u2 unused for Euler).
template <int TPR, int BAR = 0>
INC_DEV void stages_bwd_wide(const Args& a, const Ctx<1>& cx, float u, float u1, float u2, float& gu, float& gs,
                             WideAdjSmem<TPR>& sh, int g) {
    const float dt = cx.dt;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    float acc = 0.f;
    for (int k = stages - 1; k >= 0; --k) {
        float rv;
        rhs_vjp_wide<TPR, BAR>(a, cx, k == 2 ? u2 : (k == 1 ? u1 : u), gu, rv, sh, g);
        const float ka = rk3_a(k), kb = rk3_b(k);
        gs += kb * dt * gu;
        acc += ka * gu;
        gu = kb * (gu + dt * rv);
    }
    gu += acc;
}

// advance_bwd for one cell per thread: the stage inputs replayed with the wide
// forward, then the stages' adjoints in reverse.
template <int TPR>
INC_DEV void advance_bwd_wide(const Args& a, const Ctx<1>& cx, float u, float& gu, float& gs, float t,
                              WideAdjSmem<TPR>& sh, int& parity, int g) {
    const float dt = cx.dt;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    float x[1] = {u}, r[1];
    float u1 = u, u2 = u, d = 0.f;
    for (int k = 0; k + 1 < stages; ++k) {  // replay u_1, u_2 (as advance_wide)
        full_rhs_wide<1, TPR>(a, cx, x, r, t + rk3_c(k) * dt, sh.fw, parity, g);
        d = rk3_b(k) * fmaf(dt, r[0], d);
        x[0] = u + d;
        if (k == 0) u1 = x[0];
        else u2 = x[0];
    }
    stages_bwd_wide<TPR>(a, cx, u, u1, u2, gu, gs, sh, g);
}

template <int CPT>
INC_DEV void load_cells(float (&r)[CPT], const float* __restrict__ p) {
#pragma unroll
    for (int c = 0; c < CPT; ++c) r[c] = __ldg(p + c);
}
template <int CPT>
INC_DEV void store_cells(float* __restrict__ p, const float (&r)[CPT]) {
#pragma unroll
    for (int c = 0; c < CPT; ++c) p[c] = r[c];
}

// One step (steps == 1 && frames == nullptr) or a fused rollout, one row per CTA.
template <int CPT, int TPR>
__global__ void __launch_bounds__(TPR, 1) k_rollout_wide(Args a, int single_step) {
    __shared__ WideSmem<CPT, TPR> sh;
    const int row = blockIdx.x, g = threadIdx.x;
    Ctx<CPT> cx;
    make_ctx<CPT, TPR>(a, row, g, true, cx);
    if (cx.has_s) load_cells<CPT>(cx.s, a.s + (int64_t)row * a.n + g * CPT);
    float u[CPT];
    const int64_t base = (int64_t)row * a.n + g * CPT;
    load_cells<CPT>(u, a.u + base);
    int parity = 0;
    const int steps = single_step ? 1 : a.steps;
    const int nseg = a.ckpt_every > 0 ? (a.steps + a.ckpt_every - 1) / a.ckpt_every : 0;
    float cmp[CPT];  // compensation carried from step to step (see advance)
#pragma unroll
    for (int c = 0; c < CPT; ++c) cmp[c] = 0.f;
    for (int k = 0; k < steps; ++k) {
        if (a.ckpts && k % a.ckpt_every == 0)
            store_cells<CPT>(a.ckpts + ((int64_t)row * nseg + k / a.ckpt_every) * a.n + g * CPT, u);
        advance_wide<CPT, TPR>(a, cx, u, cmp, cx.t + k * cx.dt, sh, parity, g);
        if (a.frames) store_cells<CPT>(a.frames + ((int64_t)row * a.steps + k) * a.n + g * CPT, u);
    }
    if (a.out) store_cells<CPT>(a.out + base, u);
}

// Backward of a fused rollout (or of one step: ckpts = u, one one-step segment,
// g_final = dL/du_new), one row per CTA and one cell per thread.  Each segment
// is replayed from its checkpoint with the wide forward, the three stage inputs
// of every step going to this thread's slots of `seg` ([step][stage][cell],
// written and read by the same thread; the segment's last step runs only the
// stages that give its stage inputs), and then differentiated step by step,
// last first.  For small batches, where the warp layout's serial cells per lane
// set the latency of every step.
template <int TPR>
__global__ void __launch_bounds__(TPR, 1) k_rollout_bwd_wide(Args a) {
    __shared__ WideAdjSmem<TPR> sh;
    extern __shared__ float seg[];
    const int row = blockIdx.x, g = threadIdx.x;
    Ctx<1> cx;
    make_ctx<1, TPR>(a, row, g, true, cx);
    if (cx.has_s) cx.s[0] = __ldg(a.s + (int64_t)row * TPR + g);
    const int K = a.ckpt_every;
    const int nseg = (a.steps + K - 1) / K;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    const float dt = cx.dt;
    const int64_t base = (int64_t)row * TPR + g;
    // global loads are issued one step (g_frames) or one segment (ckpts) ahead
    const float* gfr = a.g_frames ? a.g_frames + (int64_t)row * a.steps * TPR + g : nullptr;
    const float* ckr = a.ckpts + (int64_t)row * nseg * TPR + g;
    float gu = a.g_final ? __ldg(a.g_final + base) : 0.f;
    float gf = gfr ? __ldg(gfr + (int64_t)(a.steps - 1) * TPR) : 0.f;
    float ck = __ldg(ckr + (int64_t)(nseg - 1) * TPR);
    float gs = 0.f;
    int parity = 0;
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        float x[1] = {ck}, r[1];
        if (sidx > 0) ck = __ldg(ckr + (int64_t)(sidx - 1) * TPR);
        for (int j = 0; j < len; ++j) {
            const float t = cx.t + (k0 + j) * dt;
            const float u0 = x[0];
            seg[3 * j * TPR + g] = u0;
            const int run = j + 1 < len ? stages : stages - 1;
            float d = 0.f;
            for (int k = 0; k < run; ++k) {  // as advance_wide
                full_rhs_wide<1, TPR>(a, cx, x, r, t + rk3_c(k) * dt, sh.fw, parity, g);
                d = rk3_b(k) * fmaf(dt, r[0], d);
                x[0] = u0 + d;
                if (k + 1 < stages) seg[(3 * j + 1 + k) * TPR + g] = x[0];
            }
        }
        for (int j = len - 1; j >= 0; --j) {
            const int k = k0 + j;
            if (gfr) {
                gu += gf;
                if (k > 0) gf = __ldg(gfr + (int64_t)(k - 1) * TPR);
            }
            stages_bwd_wide<TPR>(a, cx, seg[3 * j * TPR + g], seg[(3 * j + 1) * TPR + g],
                                 seg[(3 * j + 2) * TPR + g], gu, gs, sh, g);
        }
    }
    a.g_u[base] = gu;
    if (a.g_s) a.g_s[base] = gs;
}

// The same backward, warp-specialised: 2 TPR threads per row.  Threads [0, TPR)
// replay segment s - 1 from its checkpoint (every step's three stage inputs, into
// one half of a double buffer) while threads [TPR, 2 TPR) differentiate segment s
// from the other half, so the replay leaves the adjoint's critical path.  Each
// group syncs on its own named barrier (1: replay, 2: adjoint); the two meet at
// one CTA barrier per segment, where the halves change hands.  Rows up to 128
// cells: the replay also records each stage input's alpha and first argmax, and
// the adjoint forms the next stage's reconstruction quantities (vjp_pre) while
// it differentiates this one, between the stage's two barriers.
template <int TPR>
__global__ void __launch_bounds__(2 * TPR, 1) k_rollout_bwd_wide2(Args a) {
    constexpr bool AHEAD = TPR <= 128;  // wider rows keep 128 registers a thread (512 threads)
    __shared__ WideSmem<1, TPR> shr;
    __shared__ WideAdjSmem<TPR> sha;
    extern __shared__ float segbuf[];  // [2][3 ckpt_every][TPR], then (AHEAD) [2][3 ckpt_every][2] alpha, argmax
    const int row = blockIdx.x;
    const bool rep = threadIdx.x < TPR;
    const int g = rep ? threadIdx.x : threadIdx.x - TPR;
    Ctx<1> cx;
    make_ctx<1, TPR>(a, row, g, true, cx);
    if (cx.has_s) cx.s[0] = __ldg(a.s + (int64_t)row * TPR + g);
    const int K = a.ckpt_every;
    const int nseg = (a.steps + K - 1) / K;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    const float dt = cx.dt;
    const int64_t base = (int64_t)row * TPR + g;
    const int half = 3 * K * TPR;
    float* alph = segbuf + 2 * half;
    const float* ckr = a.ckpts + (int64_t)row * nseg * TPR + g;
    int parity = 0;
    // segment sidx replayed into its half of the buffer (replay group)
    auto replay = [&](int sidx) {
        float* seg = segbuf + (sidx & 1) * half;
        float* al = alph + (sidx & 1) * 6 * K;
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        float x[1] = {__ldg(ckr + (int64_t)sidx * TPR)}, r[1];
        for (int j = 0; j < len; ++j) {
            const float t = cx.t + (k0 + j) * dt;
            const float u0 = x[0];
            seg[3 * j * TPR + g] = u0;
            // with AHEAD every stage input's right-hand side runs (its alpha is recorded),
            // the last step's last one included
            const int run = (AHEAD || j + 1 < len) ? stages : stages - 1;
            float d = 0.f;
            for (int k = 0; k < run; ++k) {  // as advance_wide
                if constexpr (AHEAD)
                    full_rhs_wide<1, TPR, 1, true>(a, cx, x, r, t + rk3_c(k) * dt, shr, parity, g,
                                                   al + 2 * (3 * j + k));
                else
                    full_rhs_wide<1, TPR, 1>(a, cx, x, r, t + rk3_c(k) * dt, shr, parity, g);
                d = rk3_b(k) * fmaf(dt, r[0], d);
                x[0] = u0 + d;
                if (k + 1 < stages) seg[(3 * j + 1 + k) * TPR + g] = x[0];
            }
        }
    };
    if (rep) replay(nseg - 1);
    __syncthreads();
    const float* gfr = a.g_frames ? a.g_frames + (int64_t)row * a.steps * TPR + g : nullptr;
    float gu = 0.f, gf = 0.f, gs = 0.f;
    if (!rep) {
        gu = a.g_final ? __ldg(a.g_final + base) : 0.f;
        gf = gfr ? __ldg(gfr + (int64_t)(a.steps - 1) * TPR) : 0.f;
    }
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        if (rep) {
            if (sidx > 0) replay(sidx - 1);
        } else {
            const float* seg = segbuf + (sidx & 1) * half;
            const int k0 = sidx * K;
            const int len = min(K, a.steps - k0);
            if constexpr (AHEAD) {
                const float* al = alph + (sidx & 1) * 6 * K;
                VjpPre cur, nxt;
                vjp_pre<TPR>(a, seg + (3 * (len - 1) + stages - 1) * TPR, al + 2 * (3 * (len - 1) + stages - 1), g,
                             cur);
                for (int j = len - 1; j >= 0; --j) {
                    const int k = k0 + j;
                    if (gfr) {
                        gu += gf;
                        if (k > 0) gf = __ldg(gfr + (int64_t)(k - 1) * TPR);
                    }
                    float acc = 0.f;
                    for (int st = stages - 1; st >= 0; --st) {  // as stages_bwd_wide
                        const int jn = st > 0 ? j : j - 1, sn = st > 0 ? st - 1 : stages - 1;
                        float rv;
                        rhs_vjp_wide_pre<TPR, 2>(a, cx, cur, gu, rv, sha, g, [&] {
                            if (jn >= 0) vjp_pre<TPR>(a, seg + (3 * jn + sn) * TPR, al + 2 * (3 * jn + sn), g, nxt);
                        });
                        const float ka = rk3_a(st), kb = rk3_b(st);
                        gs += kb * dt * gu;
                        acc += ka * gu;
                        gu = kb * (gu + dt * rv);
                        cur = nxt;
                    }
                    gu += acc;
                }
            } else {
                for (int j = len - 1; j >= 0; --j) {
                    const int k = k0 + j;
                    if (gfr) {
                        gu += gf;
                        if (k > 0) gf = __ldg(gfr + (int64_t)(k - 1) * TPR);
                    }
                    stages_bwd_wide<TPR, 2>(a, cx, seg[3 * j * TPR + g], seg[(3 * j + 1) * TPR + g],
                                            seg[(3 * j + 2) * TPR + g], gu, gs, sha, g);
                }
            }
        }
        __syncthreads();  // segment sidx - 1 replayed, segment sidx's half free
    }
    if (!rep) {
        a.g_u[base] = gu;
        if (a.g_s) a.g_s[base] = gs;
    }
}

// The same backward on a cluster of two CTAs per row, for small batches (two
// CTAs per row fit on the GPU's SMs): CTA 0 replays segment s - 1 and writes its
// stage inputs, alphas and argmaxes straight into CTA 1's shared memory
// (distributed shared memory); CTA 1 differentiates segment s with the stage
// quantities formed one stage ahead.  Each CTA has an SM's schedulers to itself;
// they meet at one cluster barrier per segment, where the buffer halves change
// hands (the barrier orders the remote stores before CTA 1's reads).
template <int TPR>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(TPR, 1) k_rollout_bwd_cl(Args a) {
    namespace cg = cooperative_groups;
    __shared__ WideSmem<1, TPR> shr;   // CTA 0
    __shared__ WideAdjSmem<TPR> sha;   // CTA 1
    extern __shared__ float segbuf[];  // (CTA 1) [2][3 ckpt_every][TPR], then [2][3 ckpt_every][2] alpha, argmax
    cg::cluster_group cl = cg::this_cluster();
    const bool rep = cl.block_rank() == 0;
    const int row = blockIdx.x >> 1;
    const int g = threadIdx.x;
    Ctx<1> cx;
    make_ctx<1, TPR>(a, row, g, true, cx);
    if (cx.has_s) cx.s[0] = __ldg(a.s + (int64_t)row * TPR + g);
    const int K = a.ckpt_every;
    const int nseg = (a.steps + K - 1) / K;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    const float dt = cx.dt;
    const int64_t base = (int64_t)row * TPR + g;
    const int half = 3 * K * TPR;
    float* dseg = rep ? cl.map_shared_rank(segbuf, 1) : segbuf;  // CTA 1's buffer
    float* dalph = dseg + 2 * half;
    const float* ckr = a.ckpts + (int64_t)row * nseg * TPR + g;
    int parity = 0;
    auto replay = [&](int sidx) {  // CTA 0: segment sidx into its half of CTA 1's buffer
        float* seg = dseg + (sidx & 1) * half;
        float* al = dalph + (sidx & 1) * 6 * K;
        const int k0 = sidx * K;
        const int len = min(K, a.steps - k0);
        float x[1] = {__ldg(ckr + (int64_t)sidx * TPR)}, r[1];
        for (int j = 0; j < len; ++j) {
            const float t = cx.t + (k0 + j) * dt;
            const float u0 = x[0];
            seg[3 * j * TPR + g] = u0;
            float d = 0.f;
            for (int k = 0; k < stages; ++k) {  // every stage input's alpha is recorded, the last one's too
                full_rhs_wide<1, TPR, 0, true>(a, cx, x, r, t + rk3_c(k) * dt, shr, parity, g, al + 2 * (3 * j + k));
                d = rk3_b(k) * fmaf(dt, r[0], d);
                x[0] = u0 + d;
                if (k + 1 < stages) seg[(3 * j + 1 + k) * TPR + g] = x[0];
            }
        }
    };
    if (rep) replay(nseg - 1);
    cl.sync();
    const float* gfr = a.g_frames ? a.g_frames + (int64_t)row * a.steps * TPR + g : nullptr;
    float gu = 0.f, gf = 0.f, gs = 0.f;
    if (!rep) {
        gu = a.g_final ? __ldg(a.g_final + base) : 0.f;
        gf = gfr ? __ldg(gfr + (int64_t)(a.steps - 1) * TPR) : 0.f;
    }
    for (int sidx = nseg - 1; sidx >= 0; --sidx) {
        if (rep) {
            if (sidx > 0) replay(sidx - 1);
        } else {
            const float* seg = segbuf + (sidx & 1) * half;
            const float* al = dalph + (sidx & 1) * 6 * K;
            const int k0 = sidx * K;
            const int len = min(K, a.steps - k0);
            VjpPre cur, nxt;
            vjp_pre<TPR>(a, seg + (3 * (len - 1) + stages - 1) * TPR, al + 2 * (3 * (len - 1) + stages - 1), g,
                         cur);
            for (int j = len - 1; j >= 0; --j) {
                const int k = k0 + j;
                if (gfr) {
                    gu += gf;
                    if (k > 0) gf = __ldg(gfr + (int64_t)(k - 1) * TPR);
                }
                float acc = 0.f;
                for (int st = stages - 1; st >= 0; --st) {  // as stages_bwd_wide
                    const int jn = st > 0 ? j : j - 1, sn = st > 0 ? st - 1 : stages - 1;
                    float rv;
                    rhs_vjp_wide_pre<TPR, 0>(a, cx, cur, gu, rv, sha, g, [&] {
                        if (jn >= 0) vjp_pre<TPR>(a, seg + (3 * jn + sn) * TPR, al + 2 * (3 * jn + sn), g, nxt);
                    });
                    const float ka = rk3_a(st), kb = rk3_b(st);
                    gs += kb * dt * gu;
                    acc += ka * gu;
                    gu = kb * (gu + dt * rv);
                    cur = nxt;
                }
                gu += acc;
            }
        }
        cl.sync();  // segment sidx - 1 written, segment sidx's half free
    }
    if (!rep) {
        a.g_u[base] = gu;
        if (a.g_s) a.g_s[base] = gs;
    }
}

// Per cell and stage input, what the precompute CTA hands the adjoint CTA:
// m[0..5], pa (VjpPre) and the stage input u.
constexpr int kPreVals = 8;

// The same backward on a cluster of three CTAs per row (3 TPR threads each), a
// pipeline over segments: CTA 0 replays segment s - 2 into CTA 1's shared memory
// (every step's stage inputs); CTA 1's three thread groups take one stage input
// each at a time, find its alpha and first argmax and form its per-cell stage
// quantities (vjp_pre) into CTA 2's shared memory (segment s - 1); CTA 2
// differentiates segment s, each stage only scaling and scattering them.  One
// cluster barrier per pipeline step orders the remote stores before their
// readers and frees the double buffers' halves.
constexpr int kPreGroups = 3;

template <int TPR>
__global__ void __cluster_dims__(3, 1, 1) __launch_bounds__(kPreGroups * TPR, 1) k_rollout_bwd_cl3(Args a) {
    namespace cg = cooperative_groups;
    constexpr int NW = TPR / 32;
    __shared__ WideSmem<1, TPR> shr;   // CTA 0
    __shared__ WideAdjSmem<TPR> sha;   // CTA 2
    __shared__ float rmax[kPreGroups][2][NW];  // CTA 1: each group's per-warp max |u| (double-buffered)
    __shared__ int rarg[kPreGroups][2][NW];    //        and its first cell
    extern __shared__ float dsm[];     // CTA 1: seg [2][3K][TPR];  CTA 2: pre [2][3K][kPreVals][TPR], argmax [2][3K]
    cg::cluster_group cl = cg::this_cluster();
    const int role = (int)cl.block_rank();  // 0 replay, 1 precompute, 2 adjoint
    const int row = blockIdx.x / 3;
    const int t = threadIdx.x;
    const int g = t % TPR, q = t / TPR;
    const bool lead = t < TPR;  // CTAs 0 and 2 run one group of TPR threads
    Ctx<1> cx;
    make_ctx<1, TPR>(a, row, g, true, cx);
    if (cx.has_s) cx.s[0] = __ldg(a.s + (int64_t)row * TPR + g);
    const int K = a.ckpt_every;
    const int nseg = (a.steps + K - 1) / K;
    const int stages = a.scheme == INC_TS_EULER ? 1 : 3;
    const float dt = cx.dt;
    const int64_t base = (int64_t)row * TPR + g;
    const int half_seg = 3 * K * TPR, half_pre = 3 * K * kPreVals * TPR;
    float* seg1 = role == 0 ? cl.map_shared_rank(dsm, 1) : dsm;   // CTA 1's buffer
    float* pre2 = role == 1 ? cl.map_shared_rank(dsm, 2) : dsm;   // CTA 2's buffers
    int* am2 = reinterpret_cast<int*>(pre2 + 2 * half_pre);
    const float* ckr = a.ckpts + (int64_t)row * nseg * TPR + g;
    int parity = 0;
    auto seg_len = [&](int sidx) { return min(K, a.steps - sidx * K); };
    auto replay = [&](int sidx) {  // CTA 0, threads [0, TPR)
        float* seg = seg1 + (sidx & 1) * half_seg;
        const int k0 = sidx * K, len = seg_len(sidx);
        float x[1] = {__ldg(ckr + (int64_t)sidx * TPR)}, r[1];
        for (int j = 0; j < len; ++j) {
            const float tt = cx.t + (k0 + j) * dt;
            const float u0 = x[0];
            seg[3 * j * TPR + g] = u0;
            const int run = j + 1 < len ? stages : stages - 1;
            float d = 0.f;
            for (int k = 0; k < run; ++k) {
                full_rhs_wide<1, TPR, 1>(a, cx, x, r, tt + rk3_c(k) * dt, shr, parity, g);
                d = rk3_b(k) * fmaf(dt, r[0], d);
                x[0] = u0 + d;
                if (k + 1 < stages) seg[(3 * j + 1 + k) * TPR + g] = x[0];
            }
        }
    };
    int rpar = 0;  // CTA 1: which half of the group's max buffers this stage input uses
    auto precompute = [&](int sidx) {  // CTA 1, group q takes every kPreGroups-th stage input
        const float* seg = dsm + (sidx & 1) * half_seg;
        float* out = pre2 + (sidx & 1) * half_pre;
        int* amo = am2 + (sidx & 1) * 3 * K;
        const int len = seg_len(sidx);
        for (int j = 0; j < len; ++j)
            for (int k = 0; k < stages; ++k) {
                if ((j * stages + k) % kPreGroups != q) continue;
                const int i = 3 * j + k;
                const float* rowp = seg + i * TPR;
                // alpha = max |u| and its first cell, as the forward's row max (a NaN cell is passed over)
                float al[2] = {0.f, 0.f};
                if (a.conv == INC_CONV_WENO) {
                    const float au = fabsf(rowp[g]);
                    float m = au > 0.f ? au : 0.f;
                    int mi = g;
                    group_argmax_nonneg<32>(m, mi);
                    if ((g & 31) == 0) {
                        rmax[q][rpar][g >> 5] = m;
                        rarg[q][rpar][g >> 5] = mi;
                    }
                    asm volatile("bar.sync %0, %1;\n" ::"r"(3 + q), "n"(TPR) : "memory");
                    float best = rmax[q][rpar][0];
                    int am = rarg[q][rpar][0];
#pragma unroll
                    for (int w = 1; w < NW; ++w)
                        if (rmax[q][rpar][w] > best) {
                            best = rmax[q][rpar][w];
                            am = rarg[q][rpar][w];
                        }
                    al[0] = best;
                    al[1] = __int_as_float(am);
                    rpar ^= 1;
                }
                VjpPre p;
                vjp_pre<TPR>(a, rowp, al, g, p);
                float* o = out + i * kPreVals * TPR + g;
#pragma unroll
                for (int e = 0; e < 6; ++e) o[e * TPR] = p.m[e];
                o[6 * TPR] = p.pa;
                o[7 * TPR] = p.u;
                if (g == 0) amo[i] = p.am;
            }
    };
    const float* gfr = a.g_frames ? a.g_frames + (int64_t)row * a.steps * TPR + g : nullptr;
    float gu = 0.f, gf = 0.f, gs = 0.f;
    if (role == 2 && lead) {
        gu = a.g_final ? __ldg(a.g_final + base) : 0.f;
        gf = gfr ? __ldg(gfr + (int64_t)(a.steps - 1) * TPR) : 0.f;
    }
    auto adjoint = [&](int sidx) {  // CTA 2, threads [0, TPR)
        const float* pre = dsm + (sidx & 1) * half_pre;
        const int* am = reinterpret_cast<const int*>(dsm + 2 * half_pre) + (sidx & 1) * 3 * K;
        const int k0 = sidx * K, len = seg_len(sidx);
        for (int j = len - 1; j >= 0; --j) {
            const int k = k0 + j;
            if (gfr) {
                gu += gf;
                if (k > 0) gf = __ldg(gfr + (int64_t)(k - 1) * TPR);
            }
            float acc = 0.f;
            for (int st = stages - 1; st >= 0; --st) {  // as stages_bwd_wide
                const int i = 3 * j + st;
                const float* qv = pre + i * kPreVals * TPR;
                VjpPre p;
#pragma unroll
                for (int e = 0; e < 6; ++e) p.m[e] = qv[e * TPR + g];
                p.pa = qv[6 * TPR + g];
                p.u = qv[7 * TPR + g];
                p.u_l = qv[7 * TPR + ((g + TPR - 1) & (TPR - 1))];
                p.u_r = qv[7 * TPR + ((g + 1) & (TPR - 1))];
                p.am = am[i];
                float rv;
                rhs_vjp_wide_pre<TPR, 2>(a, cx, p, gu, rv, sha, g, [] {});
                const float ka = rk3_a(st), kb = rk3_b(st);
                gs += kb * dt * gu;
                acc += ka * gu;
                gu = kb * (gu + dt * rv);
            }
            gu += acc;
        }
    };
    for (int it = 0; it < nseg + 2; ++it) {
        if (role == 0) {
            if (lead && nseg - 1 - it >= 0) replay(nseg - 1 - it);
        } else if (role == 1) {
            if (nseg - it >= 0 && nseg - it < nseg) precompute(nseg - it);
        } else if (lead && nseg + 1 - it >= 0 && nseg + 1 - it < nseg) {
            adjoint(nseg + 1 - it);
        }
        cl.sync();
    }
    if (role == 2 && lead) {
        a.g_u[base] = gu;
        if (a.g_s) a.g_s[base] = gs;
    }
}

// weno_reconstruction(f, direction) as a standalone op (solver_1d.py:4-42).
template <int CPT, int TPR>
__global__ void __launch_bounds__(256) k_weno(const float* __restrict__ f, float* __restrict__ out, int rows,
                                              int n, int right_dir) {
    int row, g, left, right;
    bool valid;
    lane_setup<CPT, TPR>(row, g, left, right, valid, rows);
    float u[CPT], w[CPT + 6], h[CPT];
    const int64_t base = (int64_t)row * n + g * CPT;
    load_row_chunk<CPT>(u, f + base, valid);
    halo_window<CPT, TPR>(u, w, left, right);
#pragma unroll
    for (int c = 0; c < CPT; ++c)
        h[c] = right_dir ? weno5<true>(w[c + 2], w[c + 3], w[c + 4], w[c + 5], w[c + 6])
                         : weno5<false>(w[c + 1], w[c + 2], w[c + 3], w[c + 4], w[c + 5]);
    store_row_chunk<CPT>(out + base, h, valid);
}

// ---------------------------------------------------------------------------
// Launchers (instantiated per shape in burgers_inst_*.cu)
// ---------------------------------------------------------------------------
enum class Kind { Step, StepBwd, Rollout, RolloutBwd };

// Forward (Step, Rollout) and backward (StepBwd, RolloutBwd) launchers.  They
// are declared here and explicitly instantiated per shape in
// burgers_{fwd,bwd}_c*.cu so that the shapes compile in parallel.
template <int CPT, int TPR>
int launch_fwd(Kind kind, const Args& a, cudaStream_t st, int block);
template <int CPT, int TPR>
int launch_bwd(Kind kind, const Args& a, cudaStream_t st, int block);

template <int CPT, int TPR>
int launch_fwd_impl(Kind kind, const Args& a, cudaStream_t st, int block) {
    const int rpb = block / TPR;
    const int grid = (a.rows + rpb - 1) / rpb;
    if (kind == Kind::Step) k_step<CPT, TPR><<<grid, block, 0, st>>>(a);
    else k_rollout<CPT, TPR><<<grid, block, 0, st>>>(a);
    return check_launch("burgers");
}

template <int CPT, int TPR>
int launch_bwd_impl(Kind kind, const Args& a, cudaStream_t st, int block) {
    const int rpb = block / TPR;
    const int grid = (a.rows + rpb - 1) / rpb;
    if (kind == Kind::StepBwd) {
        k_step_bwd<CPT, TPR><<<grid, block, 0, st>>>(a);
    } else {
        const size_t smem = (size_t)rpb * a.ckpt_every * a.n * sizeof(float);
        if (smem > 227 * 1024) {
            set_error("rollout_bwd: ckpt_every*n too large for shared memory (%zu bytes)", smem);
            return INC_E_INVALID;
        }
        if (smem > 48 * 1024)
            cudaFuncSetAttribute(k_rollout_bwd<CPT, TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_rollout_bwd<CPT, TPR><<<grid, block, smem, st>>>(a);
    }
    return check_launch("burgers_bwd");
}

// Wide-row forward launchers (CPT 1 or 2), instantiated in burgers_fwd_wide.cu.
template <int CPT, int TPR>
int launch_wide(Kind kind, const Args& a, cudaStream_t st);

template <int CPT, int TPR>
int launch_wide_impl(Kind kind, const Args& a, cudaStream_t st) {
    k_rollout_wide<CPT, TPR><<<a.rows, TPR, 0, st>>>(a, kind == Kind::Step ? 1 : 0);
    return check_launch("burgers_wide");
}

#define INC_BURGERS_WIDE_SHAPES(X) X(1, 64) X(1, 128) X(1, 256) X(1, 512) X(2, 64) X(2, 128) X(2, 256)

// Wide-row backward launchers (one cell per thread), instantiated in burgers_bwd_wide.cu.
// The dynamic shared memory holds one segment's stage inputs: 3 * ckpt_every * n floats.
template <int TPR>
int launch_bwd_wide(Kind kind, const Args& a, cudaStream_t st);

template <int TPR>
constexpr size_t bwd_wide_static_smem() { return sizeof(WideAdjSmem<TPR>); }
template <int TPR>
constexpr size_t bwd_wide2_static_smem() { return sizeof(WideAdjSmem<TPR>) + sizeof(WideSmem<1, TPR>); }

template <int TPR>
int launch_bwd_wide_impl(Kind kind, const Args& a, cudaStream_t st) {
    Args b = a;
    if (kind == Kind::StepBwd) {  // one step = a one-step rollout from the checkpoint u
        b.ckpts = const_cast<float*>(a.u);
        b.steps = 1;
        b.ckpt_every = 1;
        b.g_final = a.g_out;
        b.g_frames = nullptr;
    }
    const size_t smem = (size_t)3 * b.ckpt_every * TPR * sizeof(float);
    const int nseg = (b.steps + b.ckpt_every - 1) / b.ckpt_every;
    // few rows: three CTAs per row (replay, the stages' precomputation and the
    // adjoint each on an SM of their own), or two (replay, adjoint)
    if constexpr (TPR <= 128) {
        const size_t seg1 = (size_t)2 * 3 * b.ckpt_every * TPR * sizeof(float);
        const size_t pre2 = (size_t)(2 * 3 * b.ckpt_every * kPreVals * TPR + 2 * 3 * b.ckpt_every) * sizeof(float);
        const size_t dyn = seg1 > pre2 ? seg1 : pre2;
        if (3 * b.rows <= sm_count() && dyn + bwd_wide2_static_smem<TPR>() <= 227 * 1024) {
            if (dyn + bwd_wide2_static_smem<TPR>() > 48 * 1024)
                cudaFuncSetAttribute(k_rollout_bwd_cl3<TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            k_rollout_bwd_cl3<TPR><<<3 * b.rows, kPreGroups * TPR, dyn, st>>>(b);
            return check_launch("burgers_bwd_cluster3");
        }
    }
    if constexpr (TPR <= 256) {
        const size_t dyn = 2 * smem + (size_t)2 * 3 * b.ckpt_every * 2 * sizeof(float);
        if (nseg >= 2 && 2 * b.rows <= sm_count() && dyn + bwd_wide2_static_smem<TPR>() <= 227 * 1024) {
            if (dyn + bwd_wide2_static_smem<TPR>() > 48 * 1024)
                cudaFuncSetAttribute(k_rollout_bwd_cl<TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
            k_rollout_bwd_cl<TPR><<<2 * b.rows, TPR, dyn, st>>>(b);
            return check_launch("burgers_bwd_cluster");
        }
    }
    // several segments: the warp-specialised form overlaps each replay with the adjoint
    // before it (two thread groups; rows up to 256 cells keep 128 registers a thread)
    if constexpr (TPR <= 256) {
        const size_t dyn = 2 * smem + (size_t)2 * 3 * b.ckpt_every * 2 * sizeof(float);  // + alpha, argmax
        if (nseg >= 2 && dyn + bwd_wide2_static_smem<TPR>() <= 227 * 1024) {
            if (dyn + bwd_wide2_static_smem<TPR>() > 48 * 1024)
                cudaFuncSetAttribute(k_rollout_bwd_wide2<TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)dyn);
            k_rollout_bwd_wide2<TPR><<<b.rows, 2 * TPR, dyn, st>>>(b);
            return check_launch("burgers_bwd_wide2");
        }
    }
    if (smem + bwd_wide_static_smem<TPR>() > 48 * 1024)  // the 48 KB default covers static + dynamic
        cudaFuncSetAttribute(k_rollout_bwd_wide<TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_rollout_bwd_wide<TPR><<<b.rows, TPR, smem, st>>>(b);
    return check_launch("burgers_bwd_wide");
}

#define INC_BURGERS_BWD_WIDE_SHAPES(X) X(64) X(128) X(256) X(512)

template <int CPT, int TPR>
int launch_weno(const float* f, float* out, int rows, int n, int dir, cudaStream_t st, int block);

template <int CPT, int TPR>
int launch_weno_impl(const float* f, float* out, int rows, int n, int dir, cudaStream_t st, int block) {
    const int grid = (rows + block / TPR - 1) / (block / TPR);
    k_weno<CPT, TPR><<<grid, block, 0, st>>>(f, out, rows, n, dir);
    return check_launch("weno");
}

#define INC_BURGERS_SHAPES_C4(X) X(4, 2) X(4, 4) X(4, 8) X(4, 16) X(4, 32)
#define INC_BURGERS_SHAPES_C8(X) X(8, 4) X(8, 8) X(8, 16) X(8, 32)
#define INC_BURGERS_SHAPES_C16(X) X(16, 8) X(16, 16) X(16, 32)
#define INC_BURGERS_SHAPES(X) INC_BURGERS_SHAPES_C4(X) INC_BURGERS_SHAPES_C8(X) INC_BURGERS_SHAPES_C16(X)

}  // namespace burgers
}  // namespace inc
