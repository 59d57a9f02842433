/*
 * inc_b200.h -- C ABI of the B200 (sm_100a) INC 1D hybrid time-stepper.
 *
 * One shared library, libinc_b200.so, exports these entry points.  They take
 * plain device pointers, sizes and a cudaStream_t passed as `void*`; no torch
 * or C++ types cross the boundary.  All arrays are FP32, row-major [rows][n],
 * contiguous, on the device that is current for the calling thread.  Every
 * call is asynchronous on `stream`, allocates nothing and synchronises
 * nothing, and returns 0 on success or one of the INC_E* codes below; the
 * message for the last failure on the calling thread is inc_last_error_string().
 *
 * Reference interfaces replaced (tum-pbs/INC, solvers/solver_1d.py):
 *   weno_reconstruction(f, direction)             :4-42    -> inc_weno_reconstruct
 *   BurgersSolverTorch.step(u)                    :181-195 -> inc_burgers_step
 *     (calc_nonlinear_weno :129, calc_nonlinear_FDM :125, calc_linear :144,
 *      _compute_source :104, _apply_corrections :116, forward Euler :192;
 *      SSP-RK3 composed on the same right-hand side)
 *   autograd backward through BurgersSolverTorch.step -> inc_burgers_step_bwd
 *   BurgersSolverTorch.step_adaptive(u)           :148-179 -> inc_burgers_step_adaptive (+ _bwd)
 *   calc_nonlinear_weno / _FDM, calc_linear, _compute_source
 *                                   :104-146 -> inc_burgers_terms
 *   simulate_rollout(model=None, BurgersSolverTorch) trainer/trainer_1d.py:154-183
 *                                                  -> inc_burgers_rollout (+ _bwd)
 *   KSSolverTorch.__init__ / calc_linear / etd coefficients :199-212, :235-267
 *                                                  -> inc_ks_plan_size, inc_ks_plan_init
 *   KSSolverTorch.step(u, L) = etrk2 / etd1        :280-288 -> inc_ks_step
 *   KSSolverTorch.etrk2_step / etd1_step          :242-278 -> inc_ks_substep (+ _bwd)
 *   KSSolverTorch.calc_nonlinear's FFT(u^2)       :225-233 -> inc_ks_fft_rows
 *   autograd backward through KSSolverTorch.step   -> inc_ks_step_bwd
 *   simulate_rollout(model=None, KSSolverTorch)    -> inc_ks_rollout (+ _bwd)
 */
#ifndef INC_B200_H
#define INC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define INC_OK              0
#define INC_E_INVALID       1   /* bad argument: size, enum, null pointer    */
#define INC_E_UNSUPPORTED   2   /* valid request the library has no kernel for */
#define INC_E_LAUNCH        3   /* CUDA launch/config error                   */
#define INC_E_NONFINITE     4   /* a kernel saw a non-finite state            */

/* ---- enums ------------------------------------------------------------- */
#define INC_TS_EULER        0   /* forward Euler (reference parity)          */
#define INC_TS_SSPRK3       1   /* Shu-Osher SSP-RK3                          */
#define INC_CONV_WENO       0   /* WENO5 + Lax-Friedrichs splitting          */
#define INC_CONV_FDM        1   /* central 2nd-order  -u * du/dx             */
#define INC_SRC_NONE        0   /* equation_type homogeneous / viscosity     */
#define INC_SRC_LINEAR      1   /* equation_type linear: beta * u            */
#define INC_SRC_FORCING     2   /* equation_type learning: sum_j A sin(...)   */
#define INC_KS_ETRK2        0
#define INC_KS_ETD1         1

/* Burgers problem description (solver_1d.py:45-66 sim_params fields). */
typedef struct inc_burgers_desc {
    int32_t rows;            /* B                                           */
    int32_t n;               /* cells per row, power of two in [8, 512]     */
    int32_t scheme;          /* INC_TS_*                                    */
    int32_t convection;      /* INC_CONV_*                                  */
    int32_t source;          /* INC_SRC_*                                   */
    int32_t forcing_terms;   /* J for INC_SRC_FORCING                       */
    int32_t cells_per_thread;/* 0 = library default, else 4, 8 or 16        */
    int32_t reserved;
    float dx;                /* L / n                                       */
    float dt;                /* used when dt_rows == NULL                   */
    float nu;                /* used when nu_rows == NULL                   */
    float beta;              /* used when beta_rows == NULL                 */
    const float* nu_rows;    /* [rows] or NULL                               */
    const float* dt_rows;    /* [rows] or NULL                               */
    const float* beta_rows;  /* [rows] or NULL                               */
    const float* forcing;    /* [rows][4][J]: A, omega, phi, 2*pi*l/L        */
    const float* x;          /* [n] grid coordinates (forcing), or NULL      */
} inc_burgers_desc;

/* Ragged batch: rows of different n, nu, dt and dx, packed back to back. */
typedef struct inc_burgers_ragged_desc {
    int32_t rows;
    int32_t scheme;          /* INC_TS_*                                    */
    int32_t convection;      /* INC_CONV_*                                  */
    int32_t warps_per_block; /* 0 = library default                          */
    const int64_t* offsets;  /* [rows] first cell of each row in the packing */
    const int32_t* n_rows;   /* [rows] powers of two in [8, 512]            */
    const float* nu_rows;    /* [rows]                                       */
    const float* dt_rows;    /* [rows]                                       */
    const float* dx_rows;    /* [rows]                                       */
    const int32_t* order;    /* [rows] processing order (longest first)      */
} inc_burgers_ragged_desc;

/* KS plan (solver_1d.py:199-212).  The caller fills the inputs, owns `dev`
 * (inc_ks_plan_size() bytes of device memory) and calls inc_ks_plan_init once;
 * the plan is then immutable and may be shared by any number of calls.      */
typedef struct inc_ks_plan {
    int32_t rows;            /* in: B                                        */
    int32_t n;               /* in: power of two in [16, 512]                */
    int32_t scheme;          /* in: INC_KS_*                                 */
    int32_t dealias;         /* in: 0 = reference (no dealiasing), 1 = 2/3   */
    int32_t threads_per_pair;/* in: 0 = library default                       */
    int32_t npairs;          /* out: row pairs sharing one complex FFT        */
    int32_t split;           /* out: 1 if a pair holds two domain sizes       */
    int32_t reserved;
    double dt;               /* in                                           */
    void* dev;               /* in: device buffer                            */
} inc_ks_plan;

/* ---- library ------------------------------------------------------------ */
int32_t     inc_version(void);               /* 10000*major + 100*minor + patch */
const char* inc_last_error_string(void);

/* ---- WENO5 reconstruction (solver_1d.py:4-42); direction 0=left 1=right - */
int inc_weno_reconstruct(const float* f, float* out, int32_t rows, int32_t n,
                         int32_t direction, void* stream);

/* ---- Burgers ------------------------------------------------------------ */
/* One step of size dt per row: u_out = S(u, s).  s (correction_s) may be NULL.
 * t_rows [rows] (or NULL: t0 for every row) is the time at the step start,
 * read only by INC_SRC_FORCING.                                              */
int inc_burgers_step(const inc_burgers_desc* d, const float* u, const float* s,
                     const float* t_rows, double t0, float* u_out, void* stream);

/* Vector-Jacobian product of inc_burgers_step: given g_out = dL/du_out,
 * writes g_u = dL/du and (if g_s != NULL) g_s = dL/ds.  u, s, t as passed to
 * the forward step (SSP-RK3 replays its stages from them).                  */
int inc_burgers_step_bwd(const inc_burgers_desc* d, const float* u, const float* s,
                         const float* t_rows, double t0, const float* g_out,
                         float* g_u, float* g_s, void* stream);

/* `steps` fixed steps in one launch with the state held on chip.  s is held
 * constant.  frames [rows][steps][n] (or NULL) receives every state after a
 * step; u_final [rows][n] the last.  If ckpts != NULL the state at the start of
 * every `ckpt_every`-step segment is stored in ckpts [rows][nseg][n],
 * nseg = ceil(steps / ckpt_every), for inc_burgers_rollout_bwd.             */
int inc_burgers_rollout(const inc_burgers_desc* d, const float* u0, const float* s,
                        const float* t_rows, double t0, int32_t steps,
                        float* frames, float* u_final, int32_t ckpt_every,
                        float* ckpts, void* stream);

/* Backward of inc_burgers_rollout from its checkpoints.  g_frames
 * [rows][steps][n] and g_final [rows][n] may each be NULL (zero).           */
int inc_burgers_rollout_bwd(const inc_burgers_desc* d, const float* ckpts,
                            const float* s, const float* t_rows, double t0,
                            int32_t steps, int32_t ckpt_every,
                            const float* g_frames, const float* g_final,
                            float* g_u0, float* g_s, void* stream);

/* The right-hand side's terms for a state u [rows][n], each to its own array
 * (any of the three may be NULL): nonlinear = calc_nonlinear_weno or
 * calc_nonlinear_FDM (solver_1d.py:125-142, per the descriptor's convection),
 * linear = calc_linear, nu * D2 u (:144-146), source = _compute_source (:104-114;
 * zero for homogeneous / viscosity, beta u for linear, the forcing sum at time
 * t_rows / t0 for learning; correction_s is not added, as in the reference).
 * The same device arithmetic as the step kernels.  n: a power of two in [8, 512]. */
int inc_burgers_terms(const inc_burgers_desc* d, const float* u, const float* t_rows,
                      double t0, float* nonlinear, float* linear, float* source,
                      void* stream);

/* Adaptive-CFL Euler sub-stepping over one dt with the global max |u|
 * (solver_1d.py:148-179), all on the device: no host synchronisation.  One
 * cooperative launch spreads the rows over every SM; a grid barrier between
 * substeps lets all CTAs take dt_local = min(remaining, cfl dx / max|u|) from
 * the same batch maximum; the loop stops as the reference's does (remaining
 * time spent, or ceil(remaining / dt_local) > max_substeps).  t_out [rows] (or
 * NULL) receives t + sum(dt_local); substeps_out (device int32, or NULL) the
 * reference's substep count.  work: inc_burgers_step_adaptive_work_size(
 * max_substeps) bytes of device memory, 256-byte aligned, which receives the
 * run: int32 at byte 20 = error (0 ok; 1 a barrier wait gave up; 2 more than
 * max_substeps + 1 substeps), int32 at byte 24 = substeps run, then the
 * dt_local and time offset of each (read by inc_burgers_step_adaptive_bwd).  */
int64_t inc_burgers_step_adaptive_work_size(int32_t max_substeps);
int inc_burgers_step_adaptive(const inc_burgers_desc* d, float cfl,
                              int32_t max_substeps, const float* u,
                              const float* s, const float* t_rows, double t0,
                              float* u_out, float* t_out, void* work,
                              int32_t* substeps_out, void* stream);
/* Vector-Jacobian product of one inc_burgers_step_adaptive call with its
 * substep sizes held constant (as autograd through the reference, whose
 * dt_local comes from .item()): the run recorded in `work` (same max_substeps;
 * `executed` = its substeps run, read from work by the caller) is replayed from
 * u with its states in `states` ([executed][rows][n] floats of device scratch),
 * then differentiated in reverse.  g_s (dL/d correction_s) may be NULL.       */
int inc_burgers_step_adaptive_bwd(const inc_burgers_desc* d, const float* u,
                                  const float* s, const float* t_rows, double t0,
                                  const void* work, int32_t max_substeps,
                                  int32_t executed, const float* g_out,
                                  float* g_u, float* g_s, float* states,
                                  void* stream);

/* Ragged batch: every row advances `steps` steps in one persistent launch.
 * queue: one device int32 of caller memory, zeroed by this call.            */
int inc_burgers_ragged_rollout(const inc_burgers_ragged_desc* d,
                               const float* u0, int32_t steps, float* u_final,
                               int32_t* queue, int32_t grid_blocks, void* stream);

/* Forward rollout and its backward in one call, for callers that cannot
 * allocate device memory while the op runs: a host framework that owns all
 * device memory and forbids allocation inside a foreign-function call, or an
 * application held to a fixed memory budget.  The checkpoints that the other
 * pair (inc_burgers_rollout + inc_burgers_rollout_bwd) keeps in caller memory
 * live here in a fixed 8 MiB array compiled into the library, of which every
 * GPU that loads the library holds one copy until exit.  The call allocates
 * nothing: the caller passes only inputs (u0, s, t, g_frames, g_final) and
 * outputs (frames and u_final may be NULL; g_u0 required, g_s may be NULL).
 * Limit: rows * ceil(steps / ckpt_every) * n <= INC_NOALLOC_CKPT_FLOATS, else
 * INC_E_INVALID.  A call looks the array's device address up in the current
 * context (cudaGetSymbolAddress) unless its stream is capturing; a capturing
 * call reuses the address the last call on that device found, so make the
 * first call on a device, and the first one after a context reset
 * (cudaDeviceReset) or a switch to another context, before any stream capture
 * there.  All calls share the one array, which keeps
 * the last call's checkpoints; each call writes every checkpoint before it
 * reads it, so nothing needs clearing, but calls that overlap on the GPU (on
 * different streams) race on it.  No counterpart in the reference.          */
#define INC_NOALLOC_CKPT_FLOATS (2 * 1024 * 1024)
int inc_burgers_rollout_grad_noalloc(const inc_burgers_desc* d, const float* u0,
                                     const float* s, const float* t_rows, double t0,
                                     int32_t steps, int32_t ckpt_every,
                                     const float* g_frames, const float* g_final,
                                     float* frames, float* u_final, float* g_u0,
                                     float* g_s, void* stream);

/* Hybrid rollout with the corrector evaluated inside the kernel: per step
 * s = CNN(u), then u = step(u, s) -- simulate_rollout with correction "INC"
 * (trainer/trainer_1d.py:154-183) and the benchmark's periodic CNN corrector
 * (PeriodicCNN1D: Conv1d 1 -> 32 -> 32 -> 32 -> 1, kernel 5, circular padding,
 * erf GELU between layers).  ckpts (with ckpt_every > 0) receives the state at
 * the start of every ckpt_every-th step for the backward below, or is NULL.
 * It replaces the per-step pair
 * `s = model(u); u = solver.step(u)` of the reference loop.  weights: device, INC_CNN_WEIGHT_FLOATS floats, 16-byte aligned,
 * packed as w1[co][k], b1[co], w2[ci][co][k], b2[co], w3[ci][co][k], b3[co],
 * w4[ci][k], b4 (torch's Conv1d weight is [co][ci][k]; the hidden layers are
 * stored input-channel major).  frames, corrections ([rows][steps][n]) and
 * u_final may be NULL.  n: 64, 128, 256 or 512 (else INC_E_UNSUPPORTED);
 * desc->cells_per_thread is ignored.                                        */
#define INC_CNN_WEIGHT_FLOATS 10657
int inc_burgers_cnn_rollout(const inc_burgers_desc* d, const float* weights,
                            const float* u0, const float* t_rows, double t0,
                            int32_t steps, float* frames, float* corrections,
                            float* u_final, int32_t ckpt_every, float* ckpts,
                            void* stream);
/* Backward of inc_burgers_cnn_rollout (the training step of the hybrid
 * rollout): from the forward's checkpoints (ckpts [rows][ceil(steps/k)][n],
 * written with ckpt_every = k) and corrections, and the adjoints of the
 * frames and corrections (either may be NULL), it replays each k-step segment,
 * recomputes the network's activations and returns dL/du0 (g_u0 [rows][n]) and
 * dL/dweights (g_weights, INC_CNN_WEIGHT_FLOATS floats in the packed layout).
 * work: rows * INC_CNN_WEIGHT_FLOATS floats of device scratch (the weight
 * gradients of each CTA's rows, summed in a fixed order, so results are
 * deterministic).  n: 64, 128, 256 or 512 (else INC_E_UNSUPPORTED);
 * ckpt_every <= 32, and <= 26 at n = 512 (else INC_E_INVALID).               */
int inc_burgers_cnn_rollout_bwd(const inc_burgers_desc* d, const float* weights,
                                const float* ckpts, const float* corrections,
                                const float* t_rows, double t0, int32_t steps,
                                int32_t ckpt_every, const float* g_frames,
                                const float* g_corrections, const float* g_final,
                                float* g_u0, float* g_weights, float* work,
                                void* stream);

/* The same pair with the hidden layers' pre-activations recorded: the forward
 * also writes z2 and z3 (the two 32-channel convolutions before their GELU) of
 * every step to acts [rows][steps][2][32][n] floats (16-byte aligned), and the
 * backward reads them there instead of recomputing them, a third of its
 * convolution work.  acts must not be NULL (INC_E_INVALID).                    */
int inc_burgers_cnn_rollout_acts(const inc_burgers_desc* d, const float* weights,
                                 const float* u0, const float* t_rows, double t0,
                                 int32_t steps, float* frames, float* corrections,
                                 float* u_final, int32_t ckpt_every, float* ckpts,
                                 float* acts, void* stream);
int inc_burgers_cnn_rollout_bwd_acts(const inc_burgers_desc* d, const float* weights,
                                     const float* ckpts, const float* corrections,
                                     const float* t_rows, double t0, int32_t steps,
                                     int32_t ckpt_every, const float* g_frames,
                                     const float* g_corrections, const float* g_final,
                                     float* g_u0, float* g_weights, float* work,
                                     const float* acts, void* stream);

/* ---- Kuramoto-Sivashinsky --------------------------------------------- */
/* Bytes of device memory a plan needs.                                       */
int64_t inc_ks_plan_size(int32_t rows, int32_t n);
/* Pairs rows (equal domain sizes first), uploads the pairing, and computes
 * exp(L dt), phi1, phi2 per row in FP64 on the GPU (stored FP32) and the FFT
 * twiddles.  domain_size_host: [rows] on the host.  Synchronises `stream`
 * before returning (set-up call; not for use inside stream capture).       */
int inc_ks_plan_init(inc_ks_plan* plan, const float* domain_size_host, void* stream);

/* One reference step() = two ETRK2 / ETD1 substeps.  s (correction_s) and cu
 * (correction_u) may be NULL.                                                */
int inc_ks_step(const inc_ks_plan* plan, const float* u, const float* s,
                const float* cu, float* u_out, void* stream);
/* Vector-Jacobian product of inc_ks_step (g_s may be NULL).                 */
int inc_ks_step_bwd(const inc_ks_plan* plan, const float* u, const float* s,
                    const float* cu, const float* g_out, float* g_u, float* g_s,
                    void* stream);
/* One substep: etrk2_step / etd1_step (solver_1d.py:242-278) per the plan's
 * scheme, without correction_u (the reference adds it in etrk2 / etd1 only).  */
int inc_ks_substep(const inc_ks_plan* plan, const float* u, const float* s,
                   float* u_out, void* stream);
/* Vector-Jacobian product of inc_ks_substep (g_s may be NULL).              */
int inc_ks_substep_bwd(const inc_ks_plan* plan, const float* u, const float* s,
                       const float* g_out, float* g_u, float* g_s, void* stream);
/* `steps` step() calls in one launch with s held constant; frames, u_final,
 * ckpts as for inc_burgers_rollout.                                          */
int inc_ks_rollout(const inc_ks_plan* plan, const float* u0, const float* s,
                   int32_t steps, float* frames, float* u_final,
                   int32_t ckpt_every, float* ckpts, void* stream);
int inc_ks_rollout_bwd(const inc_ks_plan* plan, const float* ckpts, const float* s,
                       int32_t steps, int32_t ckpt_every, const float* g_frames,
                       const float* g_final, float* g_u0, float* g_s, void* stream);
/* inc_ks_rollout_bwd with a caller-owned device scratch of
 * inc_ks_rollout_bwd_work_size(plan, ckpt_every) bytes (16-byte aligned; -1 for
 * a bad plan or ckpt_every).  The segment replay keeps every step's substep
 * states there, so the adjoint does not rebuild them: 17 instead of 24 row-pair
 * transforms per step() (ETRK2).  With 32 lanes and up to 8 values per lane per
 * row pair, ETRK2 and one domain size per pair, a second warp replays the next
 * segment while the first differentiates this one, and the scratch holds two
 * segments per pair.  Same results to rounding.                                */
int64_t inc_ks_rollout_bwd_work_size(const inc_ks_plan* plan, int32_t ckpt_every);
int inc_ks_rollout_bwd_ws(const inc_ks_plan* plan, const float* ckpts, const float* s,
                          int32_t steps, int32_t ckpt_every, const float* g_frames,
                          const float* g_final, float* g_u0, float* g_s, void* work,
                          int64_t work_bytes, void* stream);

/* Tape rollouts: inc_ks_rollout (ckpt_every = 0) that also records, for every
 * step, its start state and its three intermediate substep states (ETD1: the
 * one between its substeps) in `tape`, inc_ks_tape_size(plan, steps) bytes of
 * device memory (16-byte aligned; -1 for a bad plan or steps); and the
 * backward that reads them instead of replaying segments from checkpoints:
 * 9 row-pair transforms per step() (ETRK2) instead of 17.  For callers with
 * the memory to spare (4 x 8 bytes per row pair, cell and step: 1.3 GB for
 * 1024 rows x 256 cells x 400 steps).  Same results as the checkpointed pair to
 * rounding.  No counterpart in the reference (autograd keeps its whole graph). */
int64_t inc_ks_tape_size(const inc_ks_plan* plan, int32_t steps);
int inc_ks_rollout_tape(const inc_ks_plan* plan, const float* u0, const float* s,
                        int32_t steps, float* frames, float* u_final, void* tape,
                        int64_t tape_bytes, void* stream);
int inc_ks_rollout_bwd_tape(const inc_ks_plan* plan, const void* tape, int64_t tape_bytes,
                            const float* s, int32_t steps, const float* g_frames,
                            const float* g_final, float* g_u0, float* g_s, void* stream);

/* ---- analysis -------------------------------------------------------------- */
/* Energy spectrum of each of `rows` real rows of length n (a power of two in
 * [16, 512]): out[row][k] = |FFT(u)[k]|^2 for k in [0, n/2], bins 1..n/2-1
 * doubled.  Replaces calculate_energy_spectrum (analysis/Plot_KS.py:196-235),
 * which the reference runs on the CPU after a rollout.                        */
int inc_energy_spectrum(const float* u, float* out, int32_t rows, int32_t n, void* stream);

/* Spectra of real rows for KSSolverTorch.calc_nonlinear (solver_1d.py:225-233):
 * mode 0: out = FFT(v), mode 1: out = FFT(v^2), both [rows][n] complex (re, im
 * interleaved; 8-byte aligned), unnormalised as torch.fft.fft; mode 2: v is
 * [rows][n] complex and out [rows][n] real, the real part of the unnormalised
 * inverse DFT (the adjoint of a real row's FFT).  n: power of two in [16, 512]. */
int inc_ks_fft_rows(const float* v, float* out, int32_t rows, int32_t n, int32_t mode,
                    void* stream);

/* ---- corrector: FNO spectral convolution ----------------------------------- */
/* y[b][o] = irfft(sum_c rfft(x[b][c])[k] * (w_re + i w_im)[c][o][k] for
 * k < modes, zero above), n points, plus bias[o] and addend[b][o][n] where
 * those are not NULL.  Replaces SpectralConv1d.forward
 * (models/models_1d/fno.py:26-37: rfft, compl_mul1d einsum, irfft) for
 * in_channels == out_channels == width, and with bias and addend the sum of
 * an FNO layer's two branches (fno.py:86-88: conv(x) + w(x), the 1x1
 * convolution's bias and product passed in).  x, y, addend [batch][width][n];
 * w_re, w_im [width][width][modes]; bias [width].  x_modes receives
 * rfft(x)[..., :modes] as complex pairs [batch][width][modes][2] (the weight
 * gradient's input); work is scratch of 2 * modes * width * (batch + width)
 * floats, 16-byte aligned.  n a power of two in [16, 512]; width even,
 * <= 128; 1 <= modes <= min(32, n/2).  Returns INC_E_UNSUPPORTED outside
 * those.                                                                     */
int inc_spectral_conv1d(const float* x, const float* w_re, const float* w_im, const float* bias,
                        const float* addend, float* y, float* x_modes, float* work, int32_t batch,
                        int32_t width, int32_t n, int32_t modes, void* stream);
/* Adjoint w.r.t. x: g_x = d<g_y, y>/dx (what autograd gives through
 * SpectralConv1d.forward).  g_modes receives the gradient of the mixed modes
 * out_ft[..., :modes] [batch][width][modes][2] (irfft's adjoint: 2/n
 * rfft(g_y), 1/n at k = 0 with the imaginary part dropped); the weight
 * gradient is then sum_b g_modes[b][o][k] * conj(x_modes[b][c][k]), and the
 * bias gradient n * sum_b Re g_modes[b][o][0].  work as for the forward.     */
int inc_spectral_conv1d_bwd(const float* g_y, const float* w_re, const float* w_im, float* g_x,
                            float* g_modes, float* work, int32_t batch, int32_t width, int32_t n,
                            int32_t modes, void* stream);

/* y = gelu(h + bias[r % channels]) for every row r of [rows][n] activations
 * (exact erf GELU, torch.nn.functional.gelu): the FNO projection's bias and
 * activation (models/models_1d/fno.py:101-102, fc1 then F.gelu) in one pass
 * over the channel-major [batch][channels][n] layout.  n a positive multiple
 * of 4, rows a multiple of channels; 16-byte aligned arrays.               */
int inc_bias_gelu(const float* h, const float* bias, float* y, int32_t rows, int32_t n,
                  int32_t channels, void* stream);
/* Its backward: g_h = g_y * gelu'(h + bias[r % channels]), and row_sums[r]
 * = sum over the row of g_h (the bias gradient is their sum over the rows of
 * each channel).                                                             */
int inc_bias_gelu_bwd(const float* g_y, const float* h, const float* bias, float* g_h,
                      float* row_sums, int32_t rows, int32_t n, int32_t channels, void* stream);

/* ---- measurement utility ------------------------------------------------ */
/* FP32 FMA throughput probe used by bench.py for the roofline denominator:
 * `blocks` x 256 threads, each 128 * iters FMAs (2 flops each) in 8
 * independent chains; out [blocks * 256] keeps the results live.  No
 * counterpart in the reference.                                               */
int inc_bench_fma(float* out, int32_t blocks, int32_t iters, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* INC_B200_H */
