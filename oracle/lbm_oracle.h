/*
 * lbm_oracle.h -- FP64 CPU restatement of the reference's LBM density-design
 * path.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA library and the
 * timed CPU baseline.  Nothing in the product links or calls it.
 *
 * Parity status: parity unpinned.  The reference (Rust) cannot be compiled in
 * this environment and its LBM crate ships no tests, fixtures or golden
 * vectors (crates/implexity-physics-lbm/Cargo.toml sets `test = false`).  This
 * restatement is checked instead against an independent numpy restatement on
 * small grids (tests/golden/), against known-answer physics (Poiseuille and
 * Brinkman channels, TRT wall placement, MRT-default == TRT), and its adjoint
 * against FP64 central differences and dot-product identities.
 *
 * It takes the same lbm_problem_t as the product (include/lbm_b200.h) so that
 * both see identical inputs.  Populations are cell-major f[cell*Q + q] in FP64,
 * the reference's AoS layout (solver.rs).
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "../include/lbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

typedef struct {
    double maximum_mach;
    double relative_mass_drift;
    double minimum_population;
    double boundary_exchange_total;
    int32_t nonfinite;
    int32_t admitted;
} orc_diag_t;

int orc_create(const lbm_problem_t* p, orc_problem** out);
void orc_destroy(orc_problem* o);
const char* orc_error(void);
void orc_set_threads(int n);
int orc_threads(void);

/* cells, Q, tau, acceleration (lattice), fluid cell count */
void orc_info(const orc_problem* o, int64_t* cells, int32_t* q, double* tau, double* a_lattice,
              int64_t* fluid_cells);

/* design.rs: DesignMap::map then resistance; DesignMap::vjp; resistance' */
void orc_design(const orc_problem* o, const double* raw, double* phi, double* alpha);
void orc_design_vjp(const orc_problem* o, const double* raw, const double* phi_bar, double* out);
void orc_resistance_derivative(const orc_problem* o, const double* phi, double* out);

/* solver.rs:593-601 */
void orc_initial(const orc_problem* o, double* f);

/* solver.rs:604-614: collide -> stream -> ports.  Returns exchanged density. */
double orc_interval(const orc_problem* o, const double* before, const double* alpha, double* after);

/* history + admit over `steps` steps from the initial state, without storing
 * the trajectory.  final_state may be NULL. */
void orc_history(const orc_problem* o, const double* alpha, int64_t steps, double* final_state,
                 orc_diag_t* diag);

/* orc_history plus the per-state fluid mass [steps+1] and the exchange of
 * the step producing each state [steps+1] (entry 0 is zero). */
void orc_history_trace(const orc_problem* o, const double* alpha, int64_t steps, double* final_state,
                       orc_diag_t* diag, double* mass, double* exchange);

/* vector responses (solver.rs:874-893 plus pressure drop and viscous
 * dissipation) and their VJP (solver.rs:896-947) */
void orc_vector(const orc_problem* o, const double* phi, const double* alpha, const double* f, double* out8);
void orc_vector_vjp(const orc_problem* o, const double* phi, const double* alpha, const double* f,
                    const double* w8, double* f_bar, double* alpha_bar, double* phi_bar);

/* solver.rs:642-674 (no post_bar_extra / exchange_bar) */
void orc_interval_vjp(const orc_problem* o, const double* before, const double* alpha,
                      const double* after_bar, double* f_bar, double* alpha_bar);

/* Tau::PerCell (solver.rs:171-187): per-cell relaxation times of the BGK
 * collision (N values; NULL = the problem's uniform tau).  Returns 1 when
 * the collision is not BGK.  orc_interval_vjp_tau also returns the
 * per-cell tau cotangent of interval_vjp (tau_bar, solver.rs:642-674). */
int orc_set_tau(orc_problem* o, const double* tau);
void orc_interval_vjp_tau(const orc_problem* o, const double* before, const double* alpha,
                          const double* after_bar, double* f_bar, double* alpha_bar, double* tau_bar);

/* provider.rs:332-365 chain.  mode 0: fixed horizon with scan Every(K)
 * checkpoints (K <= 0: all states kept); mode 1: steady Neumann series at the
 * final state until |lambda_k| <= tol |lambda_0| or max_iter; mode 2: the
 * fixed horizon for the weighted responses averaged over states 1..steps
 * (responses8 returns the averages).  Pulsatile ports take their values at
 * the time of the state each reconstruction produces.
 * Returns 0 on success, 2 if the steady iteration did not converge. */
typedef struct {
    int64_t iterations;
    int64_t forward_evaluations;
    double residual;
} orc_grad_report_t;
int orc_gradient(const orc_problem* o, const double* raw, const double* w8, int64_t steps, int mode,
                 int64_t K, double tol, int64_t max_iter, double* grad, double* responses8,
                 orc_grad_report_t* report);

/* MRT moment basis (collision.rs:87-153): rows[Q*Q], norms[Q], groups[Q]
 * (0 mass, 1 momentum, 2 bulk, 3 shear, 4 odd, 5 even-high) */
int orc_mrt_basis(int q, double* rows, double* norms, int32_t* groups);

/* Sets the port values (pulsatile signals) to those of the reconstruction
 * producing state t_index; orc_interval / orc_interval_vjp then use them. */
void orc_set_time(const orc_problem* o, int64_t t_index);

/* interval / interval_vjp split into their pieces and restricted to the
 * cells [c0, c1) (x-slab decomposition checks): collide, stream (pull through
 * the source table), ports (returns the exchanged density of the range);
 * apply_ports_vjp, stream_vjp (through the readers table) and the collision
 * VJP with the solid pass-through.  Full-size arrays; only the slots each
 * piece needs are read. */
void orc_collide_range(const orc_problem* o, const double* before, const double* alpha, double* post, int64_t c0,
                       int64_t c1);
void orc_stream_range(const orc_problem* o, const double* post, const double* before, double* after, int64_t c0,
                      int64_t c1);
double orc_ports_range(const orc_problem* o, double* after, int64_t c0, int64_t c1);
void orc_ports_vjp_range(const orc_problem* o, const double* after_bar, double* refl, int64_t c0, int64_t c1);
void orc_stream_vjp_range(const orc_problem* o, const double* refl, double* post_bar, int64_t c0, int64_t c1);
void orc_collide_vjp_range(const orc_problem* o, const double* before, const double* alpha, const double* post_bar,
                           const double* refl, double* f_bar, double* alpha_bar, int64_t c0, int64_t c1);

/* Port reconstruction of one cell (ports.rs:343-406) for port index k. */
void orc_port_apply(const orc_problem* o, int port, const double* f_in, double* f_out);

#ifdef __cplusplus
}
#endif

#endif
