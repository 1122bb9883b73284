/* mma_cpu.h -- the design update of the topology-optimisation loop: the
 * Method of Moving Asymptotes on the host CPU (OpenMP), restated from the
 * reference optimiser that the LBM design loop calls after every gradient.
 *
 * Reference interface replaced (crates/implexity-optim/src/mma.rs):
 *   mma_create        MmaOptimizer::new            mma.rs:269-325
 *   mma_step          MmaOptimizer::step           mma.rs:633-660
 *                     (coerce :478-520, asymptote_update :522-553,
 *                      trust_box :555-571, pq/big_pq :573-615, rhs :617-622,
 *                      ip_residual :862-903, solve_subproblem :906-1131,
 *                      sub_kkt :1133-1148)
 *   mma_kkt_residual  MmaOptimizer::kkt_residual   mma.rs:420-476
 *   mma_state         MmaOptimizer::state_dict     mma.rs:377-387
 *   mma_enable_gcmma  MmaOptimizer::gcmma          mma.rs:339-355
 *   mma_step_gcmma    MmaOptimizer::step_gcmma     mma.rs:666-769
 *   mma_gcmma_state   GcmmaState (rho, nonfinite_trials)  mma.rs:242-248, 360-364
 * The calibration of the objective/constraint scaling and of c lives in the
 * Python driver (implexity_b200/optimize.py; mma_driver.rs:199-251).
 *
 * Conventions: n design variables, m constraints f_j(x) <= 0; dfsdx is
 * row-major m x n.  Errors come back as MMA_E_CONTRACT (inputs; the message
 * follows the reference's) or MMA_E_RUNTIME (non-finite Newton direction,
 * singular system, interior point not converged with strict_subproblem);
 * mma_last_error(NULL) returns this thread's last message.  A handle is used
 * by one host thread at a time. */
#ifndef IMPLEXITY_MMA_CPU_H
#define IMPLEXITY_MMA_CPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MMA_API __attribute__((visibility("default")))
#else
#define MMA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { MMA_OK = 0, MMA_E_CONTRACT = 1, MMA_E_RUNTIME = 2 } mma_status;

/* MmaOptions (mma.rs:87-129); the defaults are those of the reference. */
typedef struct {
    double move_limit;         /* 0.2 */
    double asymptote_init;     /* 0.5 */
    double asymptote_expand;   /* 1.2 */
    double asymptote_contract; /* 0.7 */
    double asymptote_lo;       /* 0.01 */
    double asymptote_hi;       /* 10 */
    double a0;                 /* 1 */
    double raa0;               /* 1e-5 */
    double albefa;             /* 0.1 */
    double epsimin;            /* 1e-7 */
    int64_t max_inner;         /* 200 */
    int32_t strict_subproblem; /* 0 */
} mma_options_t;

/* Diagnostics of the last step (MmaStepInfo, mma.rs:49-62). */
typedef struct {
    int64_t iteration;
    double kkt_residual;          /* of the iterate the step started from */
    double subproblem_kkt;
    int32_t subproblem_converged;
    double subproblem_ip_residual;
    double z;
    int64_t newton_steps;         /* interior-point Newton steps of the subproblem */
    double wallclock_s;
    int64_t inner_iterations;     /* GCMMA: conservative inner iterations (0 for a plain step) */
    int32_t conservative;         /* GCMMA: the accepted approximation bounds the true values */
} mma_info_t;

/* GcmmaOptions (mma.rs:131-145); the defaults are those of the reference. */
typedef struct {
    double rho_min;           /* 1e-6 */
    double rho_init;          /* 0.1 */
    double rho_growth;        /* 10 */
    int64_t max_conservative; /* 15 */
} mma_gcmma_options_t;

/* The true objective and constraint values at a trial point (the
 * reference's EvalTrue closure): writes *f0 and fs[0..m); returns 0, or
 * nonzero to abort the step with MMA_E_RUNTIME.  Non-finite values are not
 * an error: the step raises rho and retries, as the reference does. */
typedef int (*mma_eval_fn)(const double* x, double* f0, double* fs, void* ctx);

typedef struct mma_handle mma_handle;

MMA_API void mma_default_options(mma_options_t* o);
/* a, c, d: m coefficients each (NULL: 0, 1000, 1); x_min, x_max: n values,
 * or 1 value broadcast (n_bounds = 1). */
MMA_API mma_status mma_create(int64_t n, int64_t m, const mma_options_t* o, const double* a, const double* c,
                              const double* d, const double* x_min, const double* x_max, int64_t n_bounds,
                              mma_handle** out);
MMA_API void mma_destroy(mma_handle* h);
MMA_API const char* mma_last_error(const mma_handle* h);
MMA_API mma_status mma_step(mma_handle* h, const double* x_k, const double* x_km1, const double* x_km2, double f0,
                            const double* df0dx, const double* fs, const double* dfsdx, double* x_new,
                            mma_info_t* info);
/* KKT residual of (x, df0dx, fs, dfsdx) with the multipliers of the last
 * step (inf before the first). */
MMA_API double mma_kkt_residual(const mma_handle* h, const double* x, const double* df0dx, const double* fs,
                                const double* dfsdx);
/* Multipliers and asymptotes of the last step: lam, y (m each), z, L, U (n
 * each); any pointer may be NULL.  Returns the iteration count. */
MMA_API int64_t mma_state(const mma_handle* h, double* lam, double* y, double* z, double* low, double* upp);

/* GCMMA.  mma_enable_gcmma turns a handle into a GCMMA optimiser (options
 * NULL: the defaults); mma_step then refuses, as MmaOptimizer::step does for
 * a GCMMA optimiser, and mma_step_gcmma runs the conservative inner loop,
 * calling eval_true once per inner iteration.  mma_step_gcmma on a plain
 * handle is mma_step. */
MMA_API void mma_gcmma_default_options(mma_gcmma_options_t* g);
MMA_API mma_status mma_enable_gcmma(mma_handle* h, const mma_gcmma_options_t* g);
MMA_API mma_status mma_step_gcmma(mma_handle* h, const double* x_k, const double* x_km1, const double* x_km2,
                                  double f0, const double* df0dx, const double* fs, const double* dfsdx,
                                  mma_eval_fn eval_true, void* ctx, double* x_new, mma_info_t* info);
/* rho0 then rho[0..m) of the last GCMMA step (m + 1 values) and the count of
 * trial points with non-finite true values so far.  Returns m + 1, 0 before
 * the first step, -1 for a plain handle. */
MMA_API int64_t mma_gcmma_state(const mma_handle* h, double* rho, int64_t* nonfinite_trials);

#ifdef __cplusplus
}
#endif
#endif
