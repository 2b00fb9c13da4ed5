/*
 * dqb200.h -- C ABI of the B200 (sm_100a) implementation of dynamiqs' mesolve hot
 * path: the Lindblad right-hand side evaluated inside the Tsit5 / Dopri5 adaptive
 * Runge-Kutta loop, with embedded error norm, step-size controller and tsave saving.
 *
 * Every entry point takes plain pointers and sizes.  Array arguments are DEVICE
 * pointers (complex64 = interleaved float re/im, like numpy / JAX complex64) unless
 * stated otherwise; `stream` is a cudaStream_t passed as void*.  Work is enqueued on
 * `stream` and nothing synchronises the device.  No entry point allocates device
 * memory: scratch space is the caller's `workspace` buffer, sized by the matching
 * *_workspace_size() query.  Errors are returned as a DQB_* status code (0 = OK);
 * per-instance outcomes (max_steps reached, non-finite state, ...) are written to the
 * caller's `status` array.  No C++ exception crosses this boundary and no kernel traps.
 *
 * Reference interfaces replaced (paths relative to the dynamiqs repository):
 *   - DiffraxIntegrator.run / diffeqsolve       dynamiqs/integrators/core/diffrax_integrator.py:101-147
 *   - MESolveDiffraxIntegrator vector fields    dynamiqs/integrators/core/diffrax_integrator.py:312-336
 *   - SolveSaveMixin.save / postprocess_saved   dynamiqs/integrators/core/save_mixin.py:44-68
 *   - AdaptiveStepInfos                         dynamiqs/integrators/core/diffrax_integrator.py:35-50,149-157
 *   - sparse-DIA matmul primitives              dynamiqs/qarrays/sparsedia_primitives.py:199-261
 */
#ifndef DQB200_H
#define DQB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DQB_API __attribute__((visibility("default")))
#else
#define DQB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------------ */
#define DQB_OK 0
#define DQB_ERR_INVALID_ARGUMENT 1
#define DQB_ERR_UNSUPPORTED 2
#define DQB_ERR_WORKSPACE_TOO_SMALL 3
#define DQB_ERR_CUDA 4
#define DQB_ERR_SCRATCH_TOO_SMALL 5 /* problem needs more than DQB_NOALLOC_SCRATCH_BYTES */

/* ---- per-instance status (written to outputs->status[b]) -------------------- */
#define DQB_INST_OK 0
#define DQB_INST_MAX_STEPS 1     /* diffrax "maximum number of method steps" error   */
#define DQB_INST_NONFINITE 2     /* NaN/inf in the state or the error estimate       */
#define DQB_INST_NOT_HERMITIAN 3 /* check_hermitian(rho0) failed (rtol = atol = 1e-5) */
#define DQB_INST_CANCELLED 4     /* stopped by its ragged descriptor's cancel word      */

/* ---- options ----------------------------------------------------------------- */
#define DQB_METHOD_TSIT5 0
#define DQB_METHOD_DOPRI5 1
#define DQB_FORM_HERMITIAN 0 /* tmp = Hnh rho + 1/2 sum L rho L^+ ; out = tmp + tmp^+ */
#define DQB_FORM_STANDARD 1  /* Hnh rho + rho Hnh^+ + sum L rho L^+                 */
/* dqb_lindblad_rhs_dia(_tiled) only: the hermitian form with out[b] defined on the 32 x 32
 * tiles on and above the diagonal alone (every element (i, j) with j >= 32 floor(i / 32);
 * the rest is left as it was, except by stencil shapes that always write the whole
 * matrix): the layout of the stage slots in dqb_mesolve_dia's stage form, which the
 * autotuner times. */
#define DQB_FORM_HERMITIAN_UPPER 2

/* Arithmetic of the complex products.  The tensor-core modes run tcgen05 MMAs with FP32
 * accumulation in tensor memory, on each operand split into hi + lo parts (three products
 * hi*hi + hi*lo + lo*hi).  TF32X3, BF16X3 and TF32 apply to the GEMM path
 * (dqb_mesolve_dense_large and its ragged and right-hand-side entry points), where they
 * need the hermitian form and an even n (else DQB_ERR_UNSUPPORTED).  F16X3 applies to the
 * n <= 64 persistent kernel (dqb_mesolve_dense) for 32 < n <= 64, at most two jump
 * operators and the hermitian form; other problems given F16X3 run on FP32 CUDA cores.
 * The sparse-DIA kernels always use FP32 CUDA cores. */
#define DQB_PREC_FP32 0    /* FP32 FMA on CUDA cores (default)                         */
#define DQB_PREC_TF32X3 1  /* 3 x TF32 tensor-core products, ~2^-21 relative per product */
#define DQB_PREC_BF16X3 2  /* 3 x BF16 tensor-core products, ~2^-17 relative per product */
#define DQB_PREC_TF32 3    /* 1 x TF32 (hi*hi only), ~2^-11: for error studies          */
#define DQB_PREC_F16X3 4   /* 3 x FP16 tensor-core products of operands scaled by powers
                              of two, ~2^-22 relative per product                        */

/* Mirrors dq.method.Tsit5 / Dopri5 (dynamiqs/method.py:121-127,356-476) and the
 * mesolve options that reach the integrator (dynamiqs/options.py:17-77). */
typedef struct dqb_ode_options {
  int32_t method;          /* DQB_METHOD_*                                              */
  int32_t form;            /* DQB_FORM_*                                                */
  double rtol;             /* relative tolerance (default 1e-6)                         */
  double atol;             /* absolute tolerance (default 1e-6)                         */
  double safety;           /* safety factor (default 0.9)                               */
  double factormin;        /* min step factor after a rejection (default 0.2)           */
  double factormax;        /* max step factor (default 5.0)                             */
  int64_t max_steps;       /* attempted steps before DQB_INST_MAX_STEPS (100_000)       */
  double t0;               /* start time: tsave[0] unless options.t0 is set             */
  int32_t save_states;     /* 1: state at every tsave; 0: final state only              */
  int32_t check_hermitian; /* 1: flag rho0 that fails isherm(rtol=atol=1e-5)            */
  int32_t precision;       /* DQB_PREC_* (0 = FP32; see above for the paths of each)   */
  int32_t tile;            /* launch-shape choice of the sparse-DIA stencil: 4, 8 or 16 =
                              tiled kernel with that many rows per thread; 108 or 116 =
                              staged kernel with 8 or 16 rows per CTA; 208 or 216 (4
                              columns per thread), 308 or 316 (2 columns) = wide kernel
                              with 8 or 16 rows per CTA, 408 / 508 = 8 rows with two
                              rows in flight per thread, 708 = 8 rows, 2 columns,
                              registers capped for 6 CTAs per SM;
                              604 / 608 = bulk-staged kernel
                              (rows of X copied into shared memory by the bulk-copy
                              engine, stages of 4 / 8 rows; hermitian form, else 308);
                              0 (default) or 1 = generic
                              kernel; shapes that do not fit the operators fall back to
                              the generic kernel; ignored by other paths                  */
  int32_t stepper;         /* DQB_STEPPER_* (0 = AUTO): how the sparse-DIA and dense GEMM
                              (n > 64) paths form an RK step; the n <= 64 kernel, sesolve
                              and the vectorized form always run STAGES                  */
} dqb_ode_options;

/* Forms of an RK step (dqb_ode_options.stepper), for the sparse-DIA and GEMM paths:
 *   STAGES: stage by stage, as diffrax does (six right-hand sides per attempted step);
 *   KRYLOV: for the linear constant-operator right-hand side every stage, y1, the error
 *           estimate and the dense output are polynomials in hL applied to y: six
 *           right-hand sides build u_q = (tau L)^q y, q <= 7, once per accepted step,
 *           and one streaming pass over u_0..u_7 forms y1, the error and the next first
 *           stage; a rejected step keeps the basis.  Equal to STAGES in exact arithmetic,
 *           22 instead of 54 passes over the state per attempted step; in FP32 the
 *           expanded polynomial rounds worse than the stages' nested evaluation on stiff
 *           problems (up to ~5x the stage form's rounding error, still inside the solve's
 *           tolerance), so it is an opt-in;
 *   AUTO:   STAGES. */
#define DQB_STEPPER_AUTO 0
#define DQB_STEPPER_STAGES 1
#define DQB_STEPPER_KRYLOV 2

/* Outputs of a batched solve.  nsave = n_tsave if save_states else 1. */
typedef struct dqb_outputs {
  void* states;    /* complex64 [batch, nsave, n, n]                      */
  void* expects;   /* complex64 [batch, n_exp, n_tsave], NULL if n_exp==0 */
  int32_t* infos;  /* int32 [batch, 3]: nsteps, naccepted, nrejected      */
  int32_t* status; /* int32 [batch]: DQB_INST_*                           */
} dqb_outputs;

/* ---- dense operators ---------------------------------------------------------- */
/* Instance b solves with H[H_index[b]], jump set L[L_index[b]] (n_jumps matrices)
 * and rho0[rho0_index[b]]; a NULL index array means "item b".  This is how the
 * cartesian / flat batching of _vectorized_mesolve (mesolve.py:307-336) reaches the
 * kernels without materialising broadcast copies. */
typedef struct dqb_dense_problem {
  int32_t n;             /* Hilbert dimension                                  */
  int32_t n_jumps;       /* K                                                  */
  int32_t n_exp;         /* number of exp_ops                                  */
  int32_t n_tsave;       /* >= 1                                               */
  int64_t batch;         /* number of instances                                */
  const void* H;         /* complex64 [*, n, n]                                */
  const void* L;         /* complex64 [*, n_jumps, n, n]                       */
  const void* rho0;      /* complex64 [*, n, n], or [*, n, 1] if rho0_is_ket   */
  int32_t rho0_is_ket;   /* 1: rho0 = psi psi^+ (todm, utils/general.py:821)   */
  const void* E;         /* complex64 [n_exp, n, n]                            */
  const double* tsave;   /* float64 [n_tsave], strictly ascending              */
  const int32_t* H_index;    /* int32 [batch] or NULL */
  const int32_t* L_index;    /* int32 [batch] or NULL */
  const int32_t* rho0_index; /* int32 [batch] or NULL */
  const int32_t* start_order; /* int32 [batch] or NULL: a permutation of 0..batch-1, the
                                 order in which the n <= 64 kernel starts instances (e.g.
                                 stiffest first, so that short solves fill the tail);
                                 entries outside [0, batch) are skipped.  Results do not
                                 depend on it. */
} dqb_dense_problem;

/* Scratch bytes needed by dqb_mesolve_dense on the current device. */
DQB_API size_t dqb_mesolve_dense_workspace_size(int32_t n, int32_t n_jumps, int64_t batch);

/* Batched adaptive solve with dense operators.  Replaces DiffraxIntegrator.run for
 * MESolveDiffraxIntegrator with Tsit5 / Dopri5 (diffrax_integrator.py:135-147,
 * 283-378).  n <= 64: one persistent CTA per in-flight instance, the whole RK loop on
 * the device (operators and the stage input in shared memory, stages in an
 * L2-resident per-CTA scratch slot).  n > 64 returns DQB_ERR_UNSUPPORTED: use
 * dqb_mesolve_dense_large. */
DQB_API int dqb_mesolve_dense(const dqb_dense_problem* problem, const dqb_ode_options* options,
                      const dqb_outputs* outputs, void* workspace,
                      size_t workspace_bytes, void* stream);

/* One Lindblad right-hand-side evaluation per instance, out[b] = f(rho[b]) with
 * operators H[H_index[b]], L[L_index[b]] (vector_field_unvec_hermitian / _standard,
 * diffrax_integrator.py:312-323).  rho, out: complex64 [batch, n, n]. n <= 64. */
DQB_API int dqb_lindblad_rhs_dense(const dqb_dense_problem* problem, int32_t form,
                           const void* rho, void* out, void* stream);

/* Same, with the products in `precision`: DQB_PREC_F16X3 runs the tensor-core
 * right-hand side of dqb_mesolve_dense (32 < n <= 64, n_jumps <= 2, hermitian form; else
 * DQB_ERR_UNSUPPORTED) and needs a `workspace` of batch * 32768 bytes; DQB_PREC_FP32 is
 * dqb_lindblad_rhs_dense (no workspace). */
DQB_API int dqb_lindblad_rhs_dense_prec(const dqb_dense_problem* problem, int32_t form,
                                        int32_t precision, const void* rho, void* out,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* Same solve as dqb_mesolve_dense, for callers that cannot allocate device memory.
 * No counterpart in the reference (it is an addition of this library).  Who needs it:
 * code running in a process whose framework already holds nearly all device memory in
 * its own pool (JAX preallocates 75% of it by default), where a cudaMalloc made for this
 * library fails or takes memory the framework does not track, and deployments whose
 * device footprint is fixed when the library loads.  Scratch comes from a static device
 * array of DQB_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until the
 * process exits; nothing is allocated or freed.  At most
 * (DQB_NOALLOC_SCRATCH_BYTES - 256) / (9 * NP * NP * 8) instances run at once (NP = n
 * rounded up to 16, 32 or 64: 28 at n = 64), so results equal dqb_mesolve_dense's but
 * throughput is lower.  n > 64 returns DQB_ERR_UNSUPPORTED; a problem whose single-instance
 * scratch exceeds the array returns DQB_ERR_SCRATCH_TOO_SMALL.  The first call on each
 * device looks up the array's address (cudaGetSymbolAddress) and should come before any
 * stream capture.  Under CUDA's lazy module loading (the default since CUDA 12.2) the
 * driver reserves the array at that first call, not when the library loads
 * (CUDA_MODULE_LOADING=EAGER reserves it at load): make the first call before a
 * framework preallocates its pool.  The address is cached per device index and assumes
 * the device's context is never reset (after cudaDeviceReset it would be stale).  All
 * calls share the array: each clears its work counter first; calls that overlap on the
 * GPU race and must be serialised by the caller. */
#define DQB_NOALLOC_SCRATCH_BYTES (8u << 20)
DQB_API int dqb_mesolve_dense_noalloc(const dqb_dense_problem* problem, const dqb_ode_options* options,
                                      const dqb_outputs* outputs, void* stream);

/* ---- gradients (n <= 64 kernel, constant operators) ----------------------------------- */
/* Reverse-mode derivatives of a dqb_mesolve_dense solve with respect to H, the jump
 * operators and rho0, through the discrete Runge-Kutta steps the solve took (the step sizes
 * are constants, as in the reference's Direct / BackwardCheckpointed gradients,
 * dynamiqs/gradient.py:10-110, diffrax_integrator.py:88-99).  A first taped solve records
 * every accepted step (its start time, size and starting state); the adjoint pass then runs
 * the steps backwards.  Complex gradients use the convention dLoss = Re tr(G^+ dA) (torch's
 * and JAX's for a real loss).  The stage states are taken hermitian, as every stage of a
 * hermitian rho0 is. */
typedef struct dqb_tape {
  double* t;      /* device float64 [batch, capacity]: start time of each accepted step  */
  double* h;      /* device float64 [batch, capacity]: its size                          */
  void* y;        /* device complex64, dqb_mesolve_dense_tape_bytes(n, capacity, batch):
                     its starting state, padded to 16, 32 or 64                          */
  int32_t capacity; /* accepted steps recorded per instance (steps beyond it are not)  */
} dqb_tape;

typedef struct dqb_cotangents {
  const void* states;   /* complex64 [batch, nsave, n, n] dLoss/dstates, or NULL           */
  const void* expects;  /* complex64 [batch, n_exp, n_tsave] dLoss/dexpects, or NULL      */
} dqb_cotangents;

typedef struct dqb_gradients {
  void* rho0;  /* complex64 [batch, n, n], or [batch, n] when rho0_is_ket (dLoss/dpsi0)    */
  void* H;     /* complex64 [batch, n, n]: each instance's gradient of its own H            */
  void* L;     /* complex64 [batch, n_jumps, n, n]                                         */
} dqb_gradients;

DQB_API size_t dqb_mesolve_dense_tape_bytes(int32_t n, int32_t capacity, int64_t batch);

/* dqb_mesolve_dense (FP32 CUDA cores), recording `tape`; results are bitwise those of
 * dqb_mesolve_dense. */
DQB_API int dqb_mesolve_dense_taped(const dqb_dense_problem* problem, const dqb_ode_options* options,
                                    const dqb_outputs* outputs, const dqb_tape* tape, void* workspace,
                                    size_t workspace_bytes, void* stream);

DQB_API size_t dqb_mesolve_dense_adjoint_workspace_size(int32_t n, int32_t n_jumps, int64_t batch);

/* The adjoint pass: `naccepted` is the device int32 [batch] of accepted steps the taped
 * solve reported (infos[:, 1]); every one of them must be on the tape. */
DQB_API int dqb_mesolve_dense_adjoint(const dqb_dense_problem* problem, const dqb_ode_options* options,
                                      const dqb_tape* tape, const int32_t* naccepted,
                                      const dqb_cotangents* cotangents, const dqb_gradients* gradients,
                                      void* workspace, size_t workspace_bytes, void* stream);

/* ---- bounded waits (diagnostics) ----------------------------------------------------- */
/* Every mbarrier wait of the tensor-core kernels gives up after a time limit (2 s by
 * default) instead of spinning for ever: the instance then ends with DQB_INST_NONFINITE,
 * the kernel waits (2 s at most) for the MMAs it had issued, frees its tensor memory and
 * returns.  dqb_set_tc_wait_limit_ns changes the limit for the n <= 64 tensor-core kernel
 * (F16X3) of later launches in this process (0 restores 2 s; 1 makes every wait give up at
 * once, so that a test drives the failure path deterministically); dqb_probe_bounded_wait runs one wait that nothing ever completes with
 * `limit_ns` (<= 1 s) and writes result[0] = 1 if it gave up, result[1] = microseconds
 * waited (device int32 [2]).  No counterpart in the reference. */
DQB_API void dqb_set_tc_wait_limit_ns(uint64_t ns);
DQB_API int dqb_probe_bounded_wait(uint64_t limit_ns, int32_t* result, void* stream);

/* ---- time-dependent Hamiltonians (n <= 64 kernel) ------------------------------------ */
/* H(t) = H + sum_m c_m(t) ops[m] (the reference's ConstantTimeQArray + PWCTimeQArray /
 * ModulatedTimeQArray sums, dynamiqs/time_qarray.py:497-754), with prefactors the device
 * evaluates at every stage time: */
#define DQB_TD_PWC 0  /* c(t) = values[v][k] for times[k] <= t < times[k+1]; 0 outside
                         [times[0], times[n_times-1]) (PWCTimeQArray._prefactor, :631-641) */
#define DQB_TD_WAVE 1 /* c(t) = (amp_re + i amp_im) cos(omega t + phase) env(t) for
                         t_start <= t < t_end, else 0; env(t) = exp(-(t - t_center)^2 /
                         (2 sigma^2)) when sigma > 0, else 1 (a ModulatedTimeQArray whose
                         prefactor is one of these closed forms) */
#define DQB_TD_CONST 2 /* c(t) = 1 (a jump operator without time dependence)                */
#define DQB_TD_MAX_TERMS 4

typedef struct dqb_td_term {
  int32_t kind;                /* DQB_TD_*                                                 */
  int32_t n_times;             /* PWC: number of time points (n_times - 1 values per set)  */
  const double* times;         /* PWC: device float64 [n_times], ascending                 */
  const void* values;          /* PWC: device complex128 [n_sets, n_times - 1]             */
  const int32_t* value_index;  /* PWC: device int32 [batch]: instance b uses set
                                  value_index[b]; NULL: set 0 for every instance          */
  double amp_re, amp_im, omega, phase, t_center, sigma, t_start, t_end; /* WAVE           */
} dqb_td_term;

typedef struct dqb_td_hamiltonian {
  int32_t n_terms;             /* M <= DQB_TD_MAX_TERMS                                    */
  const void* ops;             /* device complex64 [M, n, n]                               */
  const dqb_td_term* terms;    /* host array [M]                                           */
  int32_t n_jump_ts;           /* discontinuity times handed to the controller            */
  const double* jump_ts;       /* device float64 [n_jump_ts], ascending (PIDController
                                  jump_ts, diffrax_integrator.py:59-72): a step never
                                  crosses one; it ends just before it, the next starts on
                                  it with its first stage re-evaluated, and the next step
                                  size scales the proposal, not the clipped step          */
  const dqb_td_term* jump_terms; /* host array [n_jumps] or NULL: jump operator k is
                                    c_k(t) L_k with c_k of jump_terms[k] (DQB_TD_CONST: 1);
                                    dqb_mesolve_dia_td and dqb_mesolve_dense_large_td only
                                    (the others return DQB_ERR_UNSUPPORTED when it is set) */
} dqb_td_hamiltonian;

/* dqb_mesolve_dense with a time-dependent Hamiltonian: problem->H is the constant part;
 * jump operators stay constant.  n <= 64 on CUDA cores (the workspace of
 * dqb_mesolve_dense_workspace_size(n, n_jumps + 1, batch) suffices). */
DQB_API int dqb_mesolve_dense_td(const dqb_dense_problem* problem, const dqb_td_hamiltonian* td,
                                 const dqb_ode_options* options, const dqb_outputs* outputs,
                                 void* workspace, size_t workspace_bytes, void* stream);

/* ---- Schroedinger equation on the same Runge-Kutta engine ---------------------------- */
/* Scratch bytes of dqb_sesolve_dense (a work counter). */
DQB_API size_t dqb_sesolve_dense_workspace_size(void);

/* Batched adaptive solve of d psi/dt = -i H psi with dense H, n <= 128.  Replaces
 * DiffraxIntegrator.run for SESolveDiffraxIntegrator with Tsit5 / Dopri5
 * (dynamiqs/integrators/core/diffrax_integrator.py:221-228,265-280; sesolve.py:240-330):
 * the same tableaux, starting step, controller, error norm (RMS over the n entries of
 * psi) and dense output as dqb_mesolve_dense.  The problem is a dqb_dense_problem with
 * n_jumps = 0 and rho0 = psi0 as kets [*, n, 1] (rho0_is_ket and L are ignored); states
 * are kets: complex64 [batch, nsave, n, 1]; expects[b, m, s] = <psi|E_m|psi>
 * (utils/general.py:467-474).  One warp per in-flight instance, H in shared memory, psi
 * and the stages in registers.  n > 128 returns DQB_ERR_UNSUPPORTED. */
DQB_API int dqb_sesolve_dense(const dqb_dense_problem* problem, const dqb_ode_options* options,
                              const dqb_outputs* outputs, void* workspace, size_t workspace_bytes,
                              void* stream);

/* Scratch bytes of dqb_sesolve_dense_large and dqb_sesolve_dia (controller state, FP64
 * expectation sums and ten n-vectors per instance); 0 for n > 8192. */
DQB_API size_t dqb_sesolve_large_workspace_size(int32_t n, int32_t n_exp, int32_t n_tsave, int64_t batch);

/* dqb_sesolve_dense beyond n = 128 (1 <= n <= 8192): the same solve (tableaux, starting
 * step, controller, RMS error norm over psi, dense output, expectation values) on the
 * batched large-problem stepper of dqb_mesolve_dense_large / dqb_mesolve_dia, whose slots
 * hold n-vectors here; the right-hand side -i H x is one batched matrix-vector product per
 * stage (one warp per row of H, x in shared memory), and <psi|E|psi> is summed in FP64 by
 * the save pass.  Same problem and output conventions as dqb_sesolve_dense; the whole
 * solve is one CUDA-graph launch (sesolve.py:240-330, diffrax_integrator.py:221-228). */
DQB_API int dqb_sesolve_dense_large(const dqb_dense_problem* problem, const dqb_ode_options* options,
                                    const dqb_outputs* outputs, void* workspace, size_t workspace_bytes,
                                    void* stream);

/* dqb_sesolve_dense_large with a time-dependent H(t) = H + sum_m c_m(t) ops_m
 * (dqb_td_hamiltonian with dense ops [M, n, n]), at any 1 <= n <= 8192: H(t) is formed per
 * instance at every stage time into the workspace, the steps are clipped at td->jump_ts
 * with the first stage re-evaluated after each one (as dqb_mesolve_dense_td).  Workspace:
 * dqb_sesolve_large_td_workspace_size(n, h_values = n * n, ...); with DIA storage
 * (dqb_sesolve_dia_td, ops as diagonals on h_offsets [M, h_ndiag, n]) h_values =
 * h_ndiag * n. */
DQB_API size_t dqb_sesolve_large_td_workspace_size(int32_t n, int64_t h_values, int32_t n_exp, int32_t n_tsave,
                                                   int64_t batch);
DQB_API int dqb_sesolve_dense_large_td(const dqb_dense_problem* problem, const dqb_td_hamiltonian* td,
                                       const dqb_ode_options* options, const dqb_outputs* outputs,
                                       void* workspace, size_t workspace_bytes, void* stream);

/* (dqb_sesolve_dia and dqb_sesolve_dia_td, the same solves with H in sparse-DIA storage,
 * are declared with the sparse-DIA operators below.) */

/* Batched adaptive solve of the vectorized master equation d vec(rho)/dt = S vec(rho)
 * (MESolveDiffraxIntegrator.vector_field_vec with options.vectorized=True,
 * diffrax_integrator.py:325-327; S = slindbladian(H, jump_ops), utils/vectorization.py:
 * 213-259), on the engine of dqb_sesolve_dense: the state is vec(rho), the columns of rho
 * stacked (vectorize, utils/vectorization.py:25-59), N = n^2 <= 256 entries, and the error
 * norm is the RMS over those N entries, as in the reference.  `problem` describes the
 * vectorized system: problem->n = N, problem->rho0 = vec(rho0) complex64 [*, N],
 * problem->E = exp_ops read row by row complex64 [n_exp, N] (expects = sum_k E_k y_k =
 * tr(E rho)), problem->H ignored except as a non-NULL check, H_index selecting the
 * instance's superoperator in `superop_t`: complex64 [*, N, N] holding S TRANSPOSED
 * (S[k][l] at superop_t[l * N + k]).  states: vec(rho) complex64 [batch, nsave, N].
 * N <= 128: S in shared memory; 128 < N <= 256: S read from global memory (L2). */
DQB_API int dqb_mesolve_vectorized(const dqb_dense_problem* problem, const void* superop_t,
                                   const dqb_ode_options* options, const dqb_outputs* outputs,
                                   void* workspace, size_t workspace_bytes, void* stream);

/* One Schroedinger right-hand side per instance, out[b] = -i H[H_index[b]] psi[b]
 * (diffrax_integrator.py:225-227); psi, out: complex64 [batch, n]. */
DQB_API int dqb_schrodinger_rhs_dense(const dqb_dense_problem* problem, const void* psi, void* out,
                                      void* stream);

/* ---- ragged batches (serving) ----------------------------------------------------- */
/* One instance of a ragged batch: its own n (<= max_n), jump count (<= max_jumps), tsave
 * grid, start time and output buffers; all pointers are device pointers to the
 * instance's own data (H n x n, L n_jumps x n x n, rho0 n x n or n x 1, E n_exp x n x n,
 * states nsave x n x n, expects n_exp x n_tsave, infos 3, status 1).  The array of
 * descriptors itself lives in device memory. */
typedef struct dqb_ragged_instance {
  int32_t n, n_jumps, n_exp, n_tsave;
  int32_t rho0_is_ket, save_states;
  double t0;
  const void* H;
  const void* L;
  const void* rho0;
  const void* E;
  const double* tsave;
  void* states;
  void* expects;
  int32_t* infos;
  int32_t* status;
  /* NULL, or a word the caller may set nonzero at any time (page-locked host memory the
   * device reaches through unified addressing, or device memory): the kernels read it
   * between RK steps (every 16th step on the n <= 64 kernel, every step on the GEMM
   * path) and end the instance with DQB_INST_CANCELLED, writing its counts and status as
   * for any other end.  Its outputs are then incomplete. */
  const volatile int32_t* cancel;
} dqb_ragged_instance;

/* Scratch bytes for dqb_mesolve_ragged. */
DQB_API size_t dqb_mesolve_ragged_workspace_size(int32_t max_n, int32_t max_jumps, int64_t count);

/* Solve `count` independent problems of different sizes (n <= 64) in one persistent launch:
 * the shape of a continuous-batching server's wave.  Each instance is solved exactly as a
 * batch of one would be (same step sequence, same results); method and tolerances come
 * from `options` (its t0 and save_states are ignored: they are per instance). */
DQB_API int dqb_mesolve_ragged(const dqb_ragged_instance* instances, int64_t count, int32_t max_n,
                               int32_t max_jumps, const dqb_ode_options* options, void* workspace,
                               size_t workspace_bytes, void* stream);

/* ---- dense operators, large n ---------------------------------------------------- */
/* Scratch bytes for dqb_mesolve_dense_large (10 n x n slots per instance, Hnh, K product
 * buffers, one sum buffer, controller state, FP64 expectation accumulators). */
DQB_API size_t dqb_mesolve_dense_large_workspace_size(int32_t n, int32_t n_jumps, int32_t n_exp,
                                                     int32_t n_tsave, int64_t batch);

/* Batched adaptive solve with dense operators of any n (meant for n > 64, where one
 * instance no longer fits a CTA).  Same problem, options and outputs as
 * dqb_mesolve_dense (DiffraxIntegrator.run, diffrax_integrator.py:135-147, 283-378):
 * each right-hand side is T_k = s L_k X, tmp = Hnh X + sum T_k L_k^+ (+ X Hnh^+), then
 * tmp + tmp^+, as batched complex GEMMs; the RK loop runs as a CUDA-graph WHILE node. */
DQB_API int dqb_mesolve_dense_large(const dqb_dense_problem* problem, const dqb_ode_options* options,
                                    const dqb_outputs* outputs, void* workspace,
                                    size_t workspace_bytes, void* stream);

/* dqb_mesolve_dense_large with a time-dependent Hamiltonian H(t) = H + sum_m c_m(t) ops_m
 * (dqb_td_hamiltonian with dense ops [M, n, n]): Hnh at every stage time formed from the
 * constant Hnh0 before each right-hand side, steps clipped at td->jump_ts with the first
 * stage re-evaluated after each one, as dqb_mesolve_dense_td does for n <= 64.  Stage form
 * only (a Krylov request returns DQB_ERR_UNSUPPORTED).  The workspace also holds Hnh0 and the
 * per-instance copies c_k(t) L_k of time-dependent jump operators (td->jump_terms):
 * dqb_mesolve_dense_large_td_workspace_size. */
DQB_API size_t dqb_mesolve_dense_large_td_workspace_size(int32_t n, int32_t n_jumps, int32_t n_exp,
                                                         int32_t n_tsave, int64_t batch);
DQB_API int dqb_mesolve_dense_large_td(const dqb_dense_problem* problem, const dqb_td_hamiltonian* td,
                                       const dqb_ode_options* options, const dqb_outputs* outputs,
                                       void* workspace, size_t workspace_bytes, void* stream);

/* One right-hand side per instance for any n through the GEMM path.  `workspace` needs
 * dqb_mesolve_dense_large_workspace_size(n, n_jumps, 0, 1, batch) bytes. */
DQB_API int dqb_lindblad_rhs_dense_large(const dqb_dense_problem* problem, int32_t form,
                                         const void* rho, void* out, void* workspace,
                                         size_t workspace_bytes, void* stream);

/* Same, with the products in `precision` (DQB_PREC_*).  The tensor-core modes read rho as
 * hermitian (they use rho^+ in place of rho), as every stage input of the hermitian form
 * is. */
DQB_API int dqb_lindblad_rhs_dense_large_prec(const dqb_dense_problem* problem, int32_t form,
                                              int32_t precision, const void* rho, void* out,
                                              void* workspace, size_t workspace_bytes,
                                              void* stream);

/* Ragged batch for the GEMM path: every instance has this n (the caller guarantees it),
 * its own jump count (<= max_jumps), exp_ops (<= max_exp), tsave grid (<= max_tsave
 * points), start time and outputs, as in dqb_ragged_instance.  `count` is a capacity when
 * `count_device` is non-NULL: the number of live instances (<= count) is then read from
 * that device int32 when the solve starts and the rest are skipped.  Launch parameters
 * then depend only on the capacity and the buffers, so repeated waves through the same
 * workspace and descriptor buffers reuse one captured graph. */
DQB_API size_t dqb_mesolve_dense_large_ragged_workspace_size(int32_t n, int32_t max_jumps,
                                                            int32_t max_exp, int32_t max_tsave,
                                                            int64_t count);
DQB_API int dqb_mesolve_dense_large_ragged(const dqb_ragged_instance* instances, int64_t count,
                                           const int32_t* count_device, int32_t n, int32_t max_jumps,
                                           int32_t max_exp,
                                           int32_t max_tsave, const dqb_ode_options* options,
                                           void* workspace, size_t workspace_bytes, void* stream);

/* ---- sparse-DIA operators (large n) ---------------------------------------------- */
/* Storage of the reference's SparseDIADataArray (dynamiqs/qarrays/sparsedia_dataarray.py:
 * 42-71): static offsets (HOST arrays here, as they are static in the reference) and
 * column-indexed diagonals diags[d][j] = A[j - offset_d][j] (DEVICE arrays), zero where
 * the row falls outside the matrix.  Jump operator k owns l_ndiag[k] consecutive entries
 * of l_offsets / of the diagonal axis of l_diags.  exp_ops are dense. */
#define DQB_DIA_MAX_HNH_DIAGS 64
#define DQB_DIA_MAX_JUMP_DIAGS 32
#define DQB_DIA_MAX_JUMPS 16
typedef struct dqb_dia_problem {
  int32_t n, n_jumps, n_exp, n_tsave;
  int64_t batch;
  int32_t h_ndiag;
  const int32_t* h_offsets;  /* HOST int32 [h_ndiag]                       */
  const void* h_diags;       /* complex64 [*, h_ndiag, n]                  */
  const int32_t* l_ndiag;    /* HOST int32 [n_jumps]                       */
  const int32_t* l_offsets;  /* HOST int32 [sum l_ndiag]                   */
  const void* l_diags;       /* complex64 [*, sum l_ndiag, n]              */
  const void* rho0;          /* complex64 [*, n, n] or [*, n, 1] (ket)     */
  int32_t rho0_is_ket;
  const void* E;             /* complex64 [n_exp, n, n] (dense)            */
  const double* tsave;       /* float64 [n_tsave]                          */
  const int32_t* H_index;
  const int32_t* L_index;
  const int32_t* rho0_index;
} dqb_dia_problem;

/* dqb_sesolve_dense_large with H in sparse-DIA storage (n_jumps = 0, psi0 as kets
 * [*, n, 1] in rho0 whatever rho0_is_ket says, dense exp_ops, 1 <= n <= 8192; workspace
 * from dqb_sesolve_large_workspace_size): -i H x as out_i = -i sum_d diag_d[i + k_d]
 * x[i + k_d], one thread per row -- the product matmul_sparsedia_array
 * (qarrays/sparsedia_primitives.py:232-246) with the column-indexed diagonals. */
DQB_API int dqb_sesolve_dia(const dqb_dia_problem* problem, const dqb_ode_options* options,
                            const dqb_outputs* outputs, void* workspace, size_t workspace_bytes, void* stream);
DQB_API int dqb_sesolve_dia_td(const dqb_dia_problem* problem, const dqb_td_hamiltonian* td,
                               const dqb_ode_options* options, const dqb_outputs* outputs, void* workspace,
                               size_t workspace_bytes, void* stream);

/* Scratch bytes for dqb_mesolve_dia (10 n x n complex64 matrices per instance, plus
 * Hnh diagonals, controller state and FP64 expectation accumulators). */
DQB_API size_t dqb_mesolve_dia_workspace_size(const dqb_dia_problem* problem);

/* Batched adaptive solve with sparse-DIA H and jump operators and a dense rho
 * (matmul_sparsedia_array / matmul_array_sparsedia, sparsedia_primitives.py:232-261, in
 * the vector fields of diffrax_integrator.py:312-323).  Hnh = -iH - 1/2 sum L^+L is built
 * once per instance in DIA form (matmul_sparsedia_sparsedia / add_sparsedia_sparsedia,
 * :172-229, hoisted out of the loop).  The RK loop runs as a CUDA graph with a device-side
 * WHILE node: the call enqueues the whole solve on `stream` and returns. */
DQB_API int dqb_mesolve_dia(const dqb_dia_problem* problem, const dqb_ode_options* options,
                            const dqb_outputs* outputs, void* workspace, size_t workspace_bytes,
                            void* stream);

/* dqb_mesolve_dia with a time-dependent Hamiltonian H(t) = H + sum_m c_m(t) ops_m
 * (dqb_td_hamiltonian; the reference's ConstantTimeQArray + PWCTimeQArray /
 * ModulatedTimeQArray sums, time_qarray.py:497-754): td->ops holds each ops_m by its
 * diagonals on the problem's h_offsets, device complex64 [M, h_ndiag, n] column-indexed
 * like h_diags (zero where ops_m has no such diagonal); the prefactors are evaluated at
 * every stage time, Hnh at that time formed from them before each right-hand side, and the
 * controller clips its steps at td->jump_ts (PIDController jump_ts, diffrax_integrator.py:
 * 59-72) with the first stage re-evaluated after each one.  Stage form only (a Krylov
 * request returns DQB_ERR_UNSUPPORTED).  Workspace: dqb_mesolve_dia_workspace_size. */
DQB_API int dqb_mesolve_dia_td(const dqb_dia_problem* problem, const dqb_td_hamiltonian* td,
                               const dqb_ode_options* options, const dqb_outputs* outputs,
                               void* workspace, size_t workspace_bytes, void* stream);

/* One right-hand side per instance with DIA operators: out[b] = f(rho[b]).  `form`:
 * DQB_FORM_HERMITIAN, DQB_FORM_STANDARD or DQB_FORM_HERMITIAN_UPPER.  `workspace` holds
 * the Hnh diagonals (size from dqb_mesolve_dia_workspace_size suffices). */
DQB_API int dqb_lindblad_rhs_dia(const dqb_dia_problem* problem, int32_t form, const void* rho,
                                 void* out, void* workspace, size_t workspace_bytes, void* stream);

/* Same, with the stencil's launch shape `tile` (as dqb_ode_options.tile: 4, 8, 16 or the
 * generic kernel),
 * as dqb_ode_options.tile selects it for dqb_mesolve_dia; the autotuner times the choices
 * through this entry point. */
DQB_API int dqb_lindblad_rhs_dia_tiled(const dqb_dia_problem* problem, int32_t form, int32_t tile,
                                       const void* rho, void* out, void* workspace,
                                       size_t workspace_bytes, void* stream);

/* ---- library info ------------------------------------------------------------- */
/* Largest n handled by the shared-memory persistent kernel for a jump count. */
DQB_API int32_t dqb_dense_small_max_n(int32_t n_jumps);
/* Build string (arch, version). */
DQB_API const char* dqb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* DQB200_H */
