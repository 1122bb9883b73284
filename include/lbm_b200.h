/*
 * lbm_b200.h -- C-ABI of the B200 (sm_100a) differentiable lattice-Boltzmann
 * density-design solver.
 *
 * This library is the GPU implementation of the reference provider
 * `lattice_boltzmann_d3q19` of implexity-physics-lbm, extended with the TRT and
 * MRT collision operators and the D3Q27 lattice of the reference's moving
 * engine.  A host (the reference's Rust provider through a `-sys` crate, the
 * Python binding in implexity_b200/, or any C/C++ caller) hands it a normalised
 * problem description, a raw design field, and asks for the forward trajectory,
 * the responses and the discrete-adjoint design gradient.
 *
 * Reference interface each entry point replaces (paths inside the reference
 * project):
 *   lbm_create        LbmProblem::normalize        crates/implexity-physics-lbm/src/solver.rs:414-550
 *                     normalize_ports / CompiledPort::new  src/ports.rs:106-272, 509-521
 *                     DesignMap::new               src/design.rs:109-171
 *                     Streaming::new               src/solver.rs:84-119
 *   lbm_set_design    LbmProblem::checked_design / fraction / resistance  src/solver.rs:562-590
 *   lbm_forward       LbmProblem::history + admit  src/solver.rs:677-687, 708-793
 *   lbm_responses     LbmProblem::vector           src/solver.rs:874-893
 *   lbm_fields        LbmProblem::fields / flow_fields  src/solver.rs:689-705, src/provider.rs:267-282
 *   lbm_gradient      sensitivities_value chain    src/provider.rs:332-365
 *                     (vector_vjp solver.rs:896-947, history_adjoint :798-815,
 *                      DesignMap::vjp design.rs:219-243)
 *   lbm_set_populations / lbm_get_populations / lbm_advance
 *                     TimeStepper::{initial_state, advance}  implexity-solve/src/time_stepper.rs:81-148
 *   lbm_step_vjp      LbmProblem::interval_vjp     src/solver.rs:642-674
 *   lbm_set_tau / lbm_step_vjp_tau
 *                     Tau::PerCell                 src/solver.rs:171-187 (interval / interval_vjp)
 *
 * Conventions
 *   - Cells are indexed like the reference Grid: cell = (i*ny + j)*nz + k
 *     (d3q19.rs:87-89), i.e. C order of an array of shape (nx, ny, nz).
 *   - Host population arrays are FP64, cell-major: f[cell*Q + q], with the
 *     velocity ordering of d3q19.rs:29-51 (D3Q19) or moving/lattice.rs:93-121
 *     (D3Q27).
 *   - Host arrays passed in are borrowed for the duration of the call only.
 *   - Every call is synchronous at return and runs on the handle's own CUDA
 *     stream.  A handle must be used by one host thread at a time.
 *   - No exception or abort crosses this ABI.  A failing call returns a
 *     status and leaves a message readable with lbm_last_error().
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 6

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

/* Status codes.  LBM_E_CONTRACT mirrors CaeError::Contract and carries the
 * reference's own messages (implexity-core/src/error.rs:34-56); the reference
 * reports trajectory admission failures as contract errors too
 * (solver.rs:717-771).  LBM_E_CONVERGENCE is used by the steady adjoint when
 * it reaches its iteration cap. */
typedef enum {
    LBM_OK = 0,
    LBM_E_CONTRACT = 1,
    LBM_E_CONVERGENCE = 2,
    LBM_E_CUDA = 3,
    LBM_E_STATE = 4 /* call order: e.g. responses requested before a forward run */
} lbm_status;

typedef enum { LBM_D3Q19 = 19, LBM_D3Q27 = 27 } lbm_lattice;

/* Collision operators (moving/collision.rs:38-53).  BGK is the reference
 * density-design provider's operator (solver.rs:298-322); TRT and MRT are the
 * moving engine's, with Guo forcing and the implicit half-step Brinkman
 * velocity of moving/psm.rs:213-226. */
typedef enum { LBM_BGK = 0, LBM_TRT = 1, LBM_MRT = 2 } lbm_collision;

/* Storage type of the populations on the device.  Arithmetic is FP32 in all
 * cases; the 16-bit variants store (f_q - w_q)/w_q. */
typedef enum { LBM_STORE_F32 = 0, LBM_STORE_F16 = 1, LBM_STORE_BF16 = 2 } lbm_storage;

typedef enum { LBM_PORT_VELOCITY = 0, LBM_PORT_PRESSURE = 1 } lbm_port_kind;

/* How a port rebuilds its cells' populations after streaming.
 * LEGACY_MOMENT: the unknown (incoming) populations from the cell's own known
 *   ones with a least-squares moment correction (ports.rs:343-406).
 * NEIGHBOR_NON_EQUILIBRIUM: every population from the inward neighbour's,
 *   f = eq(rho_port, u_t) + f_n - eq(rho_n, u_n), u_t the port velocity with its
 *   axial component taken from the neighbour (ports.rs:484-497; pressure
 *   ports only).
 * NON_EQUILIBRIUM_EXTRAPOLATION: the moving engine's port (moving/boundary.rs:
 *   445-506), f = eq(rho_b, u_b) + f_n - eq(rho_n, u_n) with (rho_n, u_port) on
 *   velocity ports and (rho_port, u_n) on pressure ports.
 * REGULARIZED_KNOWN_STRESS: every population as eq(rho, u) of the legacy
 *   target plus the deviatoric stress fitted to the known populations'
 *   non-equilibrium parts (ports.rs reconstruct_regularized :409-482).
 * The three need zero acceleration (ports.rs:148-157); the extrapolations'
 * inward neighbours must be protected fluid cells that are not port cells
 * (ports.rs:202-219), and their transposes add into the neighbour's
 * cotangent after each transposed step. */
typedef enum {
    LBM_RECON_LEGACY_MOMENT = 0,
    LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM = 1,
    LBM_RECON_NON_EQUILIBRIUM_EXTRAPOLATION = 2,
    LBM_RECON_REGULARIZED_KNOWN_STRESS = 3
} lbm_port_reconstruction;

/* Faces in the order of ports.rs FACES: xmin, xmax, ymin, ymax, zmin, zmax. */
typedef enum {
    LBM_XMIN = 0, LBM_XMAX = 1, LBM_YMIN = 2, LBM_YMAX = 3, LBM_ZMIN = 4, LBM_ZMAX = 5
} lbm_face;

/* Design filters.  CONIC is DesignMap's filter (design.rs:118-158): weights
 * (r - |d|)_+ over editable in-box neighbours.  BOX is a uniform
 * (2h+1)^3 average over the same neighbour set (h = half width in cells);
 * it has no reference counterpart. */
typedef enum { LBM_FILTER_CONIC = 0, LBM_FILTER_BOX = 1 } lbm_filter_kind;

/* Responses (provider.rs:56-63) plus two with no reference counterpart:
 * the inlet-outlet gauge pressure drop (mean over velocity-port cells minus
 * mean over pressure-port cells) and the total viscous dissipation. */
enum {
    LBM_R_MEAN_UX = 0,
    LBM_R_MEAN_UY = 1,
    LBM_R_MEAN_UZ = 2,
    LBM_R_KINETIC = 3,
    LBM_R_POROUS_DISSIPATION = 4,
    LBM_R_FLUID_VOLUME = 5,
    LBM_R_PRESSURE_DROP = 6,
    LBM_R_VISCOUS_DISSIPATION = 7,
    LBM_N_RESPONSES = 8
};

#define LBM_MAX_PORTS 7

/* One planar port (ports.rs:55-68, normalize_ports :106-272), rebuilt by
 * the reconstruction `reconstruction` selects.
 *
 * Pulsatile ports follow the moving engine's port signal
 * (moving/boundary.rs:98-126, Signal::factors; value at time t,
 * moving/field.rs:1002-1013): value(t) = ramp(t) * (wave(t) * amplitude +
 * mean) with wave(t) = sin(2 pi frequency_hz t + phase_rad) (0 when
 * frequency_hz = 0) and the C2 smoothstep ramp(t) = s^3 (10 - 15 s + 6 s^2),
 * s = t / ramp_s, for t < ramp_s (1 otherwise or when ramp_s = 0).  The
 * reconstruction that produces state t uses t = t_index * step_s.  The keys
 * are those of the reference's port parsing (implexity-physics-fsi/src/
 * problem/fluid.rs:256-322). */
typedef struct {
    int32_t kind;             /* lbm_port_kind */
    int32_t face;             /* lbm_face */
    const uint8_t* mask;      /* N booleans, the full-grid port mask */
    double velocity_m_s[3];   /* mean velocity (tangential only on pressure ports) */
    double gauge_pressure_Pa; /* pressure ports only: mean gauge pressure */
    double amplitude_m_s[3];  /* velocity ports: wave amplitude */
    double amplitude_Pa;      /* pressure ports: wave amplitude */
    double frequency_hz;      /* >= 0 */
    double phase_rad;
    double ramp_s;            /* >= 0 */
    int32_t reconstruction;   /* lbm_port_reconstruction */
} lbm_port_t;

/* The problem mapping of solver.rs:46-65 after JSON parsing (key sets and
 * array shapes are the host's job), plus the collision/lattice/storage options
 * of the moving engine (moving/field.rs:79-191).  lbm_create applies the
 * reference's numeric validation with its messages. */
typedef struct {
    int32_t lattice;          /* lbm_lattice */
    int32_t collision;        /* lbm_collision */
    int32_t storage;          /* lbm_storage */
    int32_t shape[3];
    int32_t periodic_axes[3]; /* booleans; false = closed halfway bounce-back walls */
    int32_t n_ports;
    int64_t step_count;
    double spacing_m;
    double step_s;
    double density_kg_m3;
    double kinematic_viscosity_m2_s;
    double acceleration_m_s2[3];
    double drag_max_per_s;
    double drag_shape;
    double mach_limit;
    /* topology map (design.rs:37-93) */
    double filter_radius_m;
    double projection_beta;
    double projection_eta;
    int32_t filter_kind;      /* lbm_filter_kind */
    int32_t box_half_width;   /* cells, LBM_FILTER_BOX only */
    /* collision parameters (moving/collision.rs:36-53); NaN = "None" */
    double trt_magic;         /* TRT magic parameter, default 3/16 */
    double mrt_odd_magic;     /* MRT odd-moment magic, default 3/16 */
    double mrt_bulk_rate;     /* NaN -> shear rate */
    double mrt_even_rate;     /* NaN -> shear rate */
    const uint8_t* solid_mask;     /* N */
    const uint8_t* design_region;  /* N */
    const double* fixed_design;    /* N, in [0,1] */
    const lbm_port_t* ports;       /* n_ports entries */
    /* nonzero: lbm_forward also evaluates the responses of every state
     * t = 1..steps (lbm_time_average), and lbm_gradient accepts
     * LBM_OBJ_TIME_AVERAGE */
    int32_t time_average;
    /* nonzero: the forward steps collide in FP64 arithmetic (FP32 storage
     * only; no reference counterpart, the reference is FP64 throughout).
     * FP32 collision arithmetic rounds the equilibrium momentum coherently
     * over a nearly uniform flow, which biases the steady pressure by ~1e-7
     * in density; FP64 collision removes that bias at ~1.8x the forward
     * step's time.  The adjoint is FP32 in both cases. */
    int32_t collision_fp64;
} lbm_problem_t;

/* Trajectory admission record (solver.rs:708-793).  Filled by lbm_forward
 * and lbm_advance.  A trajectory is admitted when every population of every
 * state is finite and positive, the Mach number stays within mach_limit and
 * the relative mass drift is at most 1e-6 (FP32 storage, the reference's
 * bound), 1e-4 (FP16) or 1e-3 (BF16 storage). */
typedef struct {
    double maximum_mach;          /* sqrt(3) * max |u| over fluid cells and states */
    double relative_mass_drift;   /* max_t |M_t - (M_0 + sum exchange)| / M_0 */
    double relaxation_time;       /* tau */
    double minimum_population;    /* over fluid cells and states */
    double boundary_exchange_total; /* lattice mass exchanged by ports */
    int64_t steps;
    int32_t nonfinite;            /* any non-finite population seen */
    int32_t admitted;             /* 1 if the reference admission passes */
    double device_ms;             /* CUDA-event time of the stepping kernels */
} lbm_diag_t;

/* Adjoint modes.  HORIZON is the reference's fixed-horizon discrete adjoint
 * of all step_count steps (history_adjoint, solver.rs:798-815), with the
 * forward recomputed from checkpoints every `checkpoint_every` steps
 * (implexity-ad/src/scan.rs:140-246, Checkpointing::Every).  STEADY linearises
 * one step at the final state and sums the Neumann series of the transposed
 * step until the relative norm of the newest term is below `tolerance`
 * (implexity-ad/src/implicit.rs:49-67 semantics). */
typedef enum { LBM_ADJ_HORIZON = 0, LBM_ADJ_STEADY = 1 } lbm_adjoint_mode;

/* What the weights apply to: the responses of the final state (the
 * reference's vector of the last state), or their mean over the states
 * t = 1..steps of the horizon (a stage objective: every state seeds the
 * adjoint; HORIZON mode, problems created with time_average). */
typedef enum { LBM_OBJ_FINAL = 0, LBM_OBJ_TIME_AVERAGE = 1 } lbm_objective;

/* Checkpointing of the HORIZON adjoint (implexity-ad/src/scan.rs:108-116,
 * Checkpointing).  EVERY stores the state every checkpoint_every steps
 * (Every(K)); BINOMIAL keeps at most `snapshots` states and follows the
 * binomial (revolve) schedule of implexity-ad/src/revolve.rs:128-330, which
 * minimises the recomputed steps for that number of states. */
typedef enum { LBM_CKPT_EVERY = 0, LBM_CKPT_BINOMIAL = 1 } lbm_checkpointing;

typedef struct {
    int32_t mode;             /* lbm_adjoint_mode */
    int32_t lambda_storage;   /* lbm_storage of the adjoint populations */
    int64_t checkpoint_every; /* HORIZON: K (<= 0 selects sqrt(step_count)) */
    int64_t max_iterations;   /* STEADY: cap */
    int64_t check_every;      /* STEADY: residual readback period */
    double tolerance;         /* STEADY: relative residual */
    int64_t record_budget_bytes; /* HORIZON: device bytes for per-step records (0 = auto) */
    int32_t objective;        /* lbm_objective */
    int32_t checkpointing;    /* HORIZON: lbm_checkpointing */
    int64_t snapshots;        /* HORIZON, BINOMIAL: state slots (>= 1) */
} lbm_adjoint_opts_t;

typedef struct {
    double residual;              /* STEADY: final relative residual */
    int64_t iterations;           /* adjoint steps taken */
    int64_t forward_recomputed;   /* forward steps re-run from checkpoints */
    int64_t peak_state_bytes;     /* checkpoint + record bytes held on device */
    int32_t converged;
    double forward_ms;            /* device time of the recomputation */
    double adjoint_ms;            /* device time of the adjoint steps */
    double sensitivity_ms;        /* device time of seed + design VJP */
} lbm_adjoint_report_t;

typedef struct lbm_handle lbm_handle;

/* ---- lifetime ----------------------------------------------------------- */

/* Validates and normalises the problem (LbmProblem::normalize), builds the
 * link masks, port maps and design filter, and allocates the device buffers
 * on the current CUDA device.  On failure *out is NULL and the message is
 * available from lbm_last_error(NULL). */
LBM_API lbm_status lbm_create(const lbm_problem_t* problem, lbm_handle** out);
LBM_API void lbm_destroy(lbm_handle* h);

/* Message of the last failing call on h (or of the last failing lbm_create
 * in this thread when h is NULL).  Never NULL. */
LBM_API const char* lbm_last_error(const lbm_handle* h);

LBM_API int32_t lbm_abi_version(void);

/* Normalised scalars: tau, lattice acceleration, cell count, Q. */
typedef struct {
    int64_t cells;
    int64_t fluid_cells;
    int32_t q;
    int32_t n_ports;
    double tau;
    double acceleration_lattice[3];
    int64_t device_bytes;     /* bytes allocated on the device by the handle */
} lbm_info_t;
LBM_API lbm_status lbm_info(const lbm_handle* h, lbm_info_t* out);

/* ---- design ------------------------------------------------------------- */

/* checked_design + fraction + resistance (solver.rs:562-590, design.rs:199-216,
 * 284-286).  raw has N entries in [0,1]. */
LBM_API lbm_status lbm_set_design(lbm_handle* h, const double* raw, size_t n);

/* Per-cell relaxation times (Tau::PerCell, solver.rs:171-187), the form the
 * reference's thermal provider steps with (thermal_provider.rs:616,1137):
 * tau has N entries (lattice units, finite, > 0.5) and replaces the problem's
 * uniform tau in the BGK collision of every forward step, transposed step
 * and wall-load evaluation; NULL returns to the uniform tau.  BGK problems
 * only.  The viscous-dissipation response keeps the problem's uniform tau.
 * A forward run must follow before lbm_gradient. */
LBM_API lbm_status lbm_set_tau(lbm_handle* h, const double* tau, size_t n);

/* Copies the mapped fluid fraction phi and the Brinkman resistance alpha
 * (per time step) to the host (either pointer may be NULL). */
LBM_API lbm_status lbm_get_design(lbm_handle* h, double* phi, double* alpha);

/* ---- forward -------------------------------------------------------------- */

/* Initial populations (solver.rs:593-601) followed by `steps` steps
 * (steps <= 0: the problem's step_count), with the admission reductions of
 * every state.  Returns LBM_E_CONTRACT with the reference's messages when
 * the trajectory is not admitted; diag is filled either way. */
LBM_API lbm_status lbm_forward(lbm_handle* h, int64_t steps, lbm_diag_t* diag);

/* TimeStepper-granular access.  lbm_set_populations loads a host state
 * (f[cell*Q+q], FP64) as the current state; lbm_advance runs n more steps
 * from the current state; lbm_get_populations returns the current state with
 * the port reconstruction applied (the reference's "after" state). */
LBM_API lbm_status lbm_set_populations(lbm_handle* h, const double* f, size_t n);
LBM_API lbm_status lbm_get_populations(lbm_handle* h, double* f, size_t n);
LBM_API lbm_status lbm_advance(lbm_handle* h, int64_t steps, lbm_diag_t* diag);

/* Per-state admission record of the last lbm_forward / lbm_advance
 * (admit, solver.rs:708-793): for states t = 0..steps, the fluid mass
 * sum(rho), the port mass exchange of the step that produced the state
 * (0 for t = 0; the reference's boundary_mass_changes_lattice), the minimum
 * population and the maximum speed |u| over fluid cells.  n = steps + 1;
 * any pointer may be NULL. */
LBM_API lbm_status lbm_trajectory(lbm_handle* h, double* mass, double* exchange, double* min_population,
                                  double* max_speed, size_t n);

/* The 8 responses of the current state (LBM_R_*), FP64 compensated sums. */
LBM_API lbm_status lbm_responses(lbm_handle* h, double* out8);

/* The 8 responses averaged over the states t = 1..steps of the last
 * lbm_forward (problems created with time_average; no reference
 * counterpart for the LBM problem: the stage objective of the moving
 * engine's samples, restated). */
LBM_API lbm_status lbm_time_average(lbm_handle* h, double* out8);

/* Fixed-wall momentum-exchange loads of the last interval
 * (wall_exchange::loads, wall_exchange.rs:79-100, as evaluate_value reports
 * them, provider.rs:312-321): one entry per blocked pull link of a fluid cell
 * (cells and links in order; a port cell's links along its port's inward
 * normal are not walls, wall_exchange.rs:44-70).  The state before the last
 * step is collided with the Guo-BGK collision (solver::collide, whatever the
 * problem's collision, as the reference does) and the force on the link is
 * -2 c_q (f*_opp(q) - w_q + w_q datum / (rho c^2 / 3)) rho dx^4 / dt^2 [N].
 * positions_m [n,3] are the link midpoints plus origin_m (NULL: 0);
 * force_n [n,3].  n_links receives the count; with both outputs NULL only the
 * count is returned, otherwise they need capacity >= n_links entries. */
LBM_API lbm_status lbm_wall_loads(lbm_handle* h, double pressure_datum_pa, const double* origin_m,
                                  double* positions_m, double* force_n, size_t capacity, size_t* n_links);

/* Physical fields of the current state (LbmProblem::fields, provider.rs
 * flow_fields): density [N] kg/m^3, velocity [N*3] m/s, gauge pressure [N] Pa.
 * Any pointer may be NULL. */
LBM_API lbm_status lbm_fields(lbm_handle* h, double* density, double* velocity, double* pressure);

/* Diagnostic, no counterpart in the reference: runs one bounded wait of the
 * stepping kernels (an mbarrier wait with the given limit) on an mbarrier that
 * nothing completes, on the current device.  The wait must run out: then
 * *timed_out = 1 and *waited_ms is the device time the wait took (one period
 * of limit_ns waiting before the error flag is set, one more before the
 * kernel returns).  limit_ns in [1e6, 1e9]. */
LBM_API lbm_status lbm_probe_bounded_wait(int64_t limit_ns, int32_t* timed_out, double* waited_ms);

/* ---- adjoint ------------------------------------------------------------ */

/* The binomial checkpoint schedule for `steps` steps and `snapshots` state
 * slots (BinomialSchedule::new, implexity-ad/src/revolve.rs:247-283), built
 * on the host: the forward steps it takes in all (optimal_forward_steps,
 * revolve.rs:117-125) and the most slots it holds at once.  Host only; no
 * device is needed. */
LBM_API lbm_status lbm_binomial_plan(int64_t steps, int64_t snapshots, int64_t* forward_steps,
                                     int64_t* peak_snapshots);

/* Design gradient of sum_k weights[k] * response_k (weights has
 * LBM_N_RESPONSES entries) with respect to the raw design, after a
 * successful lbm_forward.  grad has N entries.  opts may be NULL (HORIZON,
 * FP32 adjoint storage, K = sqrt(step_count)). */
LBM_API lbm_status lbm_gradient(lbm_handle* h, const double* weights, const lbm_adjoint_opts_t* opts,
                        double* grad, lbm_adjoint_report_t* report);

/* One transposed step (interval_vjp without port-exchange cotangents):
 * given a state f_t and the cotangent of f_{t+1}, returns the cotangent of
 * f_t and the per-cell cotangent of alpha.  All arrays FP64 host,
 * populations cell-major.  alpha_bar may be NULL. */
LBM_API lbm_status lbm_step_vjp(lbm_handle* h, const double* state, const double* lambda_next,
                        double* lambda, double* alpha_bar, size_t n_populations);

/* lbm_step_vjp that also returns the per-cell cotangent of the relaxation
 * time (interval_vjp's tau_bar with Tau::PerCell, solver.rs:214-285,
 * 331-356, 642-674): tau_bar has N entries (0 at solid cells).  BGK
 * problems only; the rates are those of lbm_set_tau (or the uniform tau). */
LBM_API lbm_status lbm_step_vjp_tau(lbm_handle* h, const double* state, const double* lambda_next, double* lambda,
                                    double* alpha_bar, double* tau_bar, size_t n_populations);

/* Design-map transpose alone (DesignMap::vjp, design.rs:219-243) for the
 * design last set: out[N] = d phi / d raw ^T phi_bar. */
LBM_API lbm_status lbm_design_vjp(lbm_handle* h, const double* phi_bar, double* out, size_t n);

/* ---- x-slab decomposition (several GPUs) ------------------------------- */

/* The reference parallelises this path over cells in one process (rayon,
 * solver.rs:131-136, moving/field.rs:570-611); here a problem is split along
 * x over one handle per GPU.  lbm_create_slab creates the handle of the owned
 * planes [x_begin, x_end) of `problem` (the whole problem's description)
 * plus `halo` ghost planes on each side that has a neighbour (all sides when
 * x is periodic; halo >= 1 and >= the design filter's reach).  The handle's
 * grid is the slab with its ghost planes: lbm_set_design takes the raw design
 * of those planes (in order, wrapping for periodic x), lbm_slab_gradient
 * returns the gradient contributions over them, to be summed over ranks.
 * Ports must lie on the x faces.  Responses (lbm_responses) are this rank's
 * share, normalised with the whole problem's fluid and port cell counts:
 * their sum over ranks is the problem's.  Not with time_average.
 *
 * One step of the driver: exchange the state halos (lbm_halo_pack of the
 * current state on each side with a neighbour, transfer, lbm_halo_unpack
 * of what arrived), then lbm_slab_step.  A state halo message carries the
 * populations with c_x = +1 (right side) or -1 (left) of the boundary plane;
 * an adjoint message the mirrored sets (lbm_halo_bytes gives the size; device
 * buffers; kind 0 state, 1 adjoint; side 0 left, 1 right).  Each step returns
 * this rank's admission sums of the state it read (mass sum(rho), port
 * exchange, minimum population, maximum |u|^2, non-finite flag); after the
 * last step an exchange and lbm_slab_inspect give the final state's.  The
 * steady adjoint runs the same way: lbm_slab_adjoint_begin seeds it at the
 * current state (FP32, unit scale), then per iteration an adjoint exchange and
 * lbm_slab_adjoint_step (|lambda|^2 of this rank when norm2 is non-NULL),
 * then lbm_slab_gradient.  The scalars are reduced over ranks by the caller
 * (implexity_b200/slabs.py). */
typedef struct {
    double mass;
    double exchange;
    double minimum_population;
    double maximum_speed2;
    int32_t nonfinite;
} lbm_slab_diag_t;

LBM_API lbm_status lbm_create_slab(const lbm_problem_t* problem, int32_t x_begin, int32_t x_end, int32_t halo,
                                   lbm_handle** out);
LBM_API lbm_status lbm_slab_begin(lbm_handle* h);
LBM_API lbm_status lbm_slab_step(lbm_handle* h, lbm_slab_diag_t* diag);
LBM_API lbm_status lbm_slab_inspect(lbm_handle* h, lbm_slab_diag_t* diag);
LBM_API lbm_status lbm_halo_bytes(const lbm_handle* h, int32_t kind, size_t* bytes);
LBM_API lbm_status lbm_halo_pack(lbm_handle* h, int32_t kind, int32_t side, void* device_buffer);
LBM_API lbm_status lbm_halo_unpack(lbm_handle* h, int32_t kind, int32_t side, const void* device_buffer);
LBM_API lbm_status lbm_slab_adjoint_begin(lbm_handle* h, const double* weights, double* norm2);
LBM_API lbm_status lbm_slab_adjoint_step(lbm_handle* h, double* norm2);
LBM_API lbm_status lbm_slab_gradient(lbm_handle* h, double* grad, size_t n);

/* ---- state statistics without device allocation ------------------------ */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- code inside another framework's memory pool or arena (the pool
 * owns all device memory), embedded hosts that fix their device budget up
 * front -- and that already hold a state on the device: the admission statistics of that one
 * state, computed by the same compensated reduction the stepping kernels run
 * every step (LbmProblem::admit quantities, solver.rs:714-755).
 *
 *   populations  device, FP32, plane-major f[q*cells + cell] (unshifted f),
 *                velocity order of the lattice as in lbm_get_populations.
 *                A state held in 16-bit or shifted form (such as this
 *                library's (f - w)/w storage) must be expanded to unshifted
 *                FP32 by the caller first: there is no scratch for a
 *                conversion here.
 *   solid        device uint8 per cell, NULL = all fluid (solid cells skipped)
 *   alpha        device FP32 Brinkman resistance per cell, NULL = 0
 *   acceleration_lattice  host, 3 doubles, NULL = 0
 *   out4         device, 4 doubles: fluid mass sum(rho), minimum population
 *                over fluid cells, maximum |u| over fluid cells (implicit
 *                half-step Brinkman velocity), and 1.0 if any population of
 *                any cell, solid ones included, is non-finite (else 0.0)
 *   stream       cudaStream_t, NULL = the legacy default stream
 *
 * It allocates nothing: its scratch (per-block partials and a ticket counter)
 * is a 65 792-byte static device array that every GPU loading the library
 * holds until the process exits.  Limit: q * cells < 2^31 (larger states are
 * rejected with LBM_E_CONTRACT); any such state is covered with at most 1024
 * blocks.  The first call on a device looks up the array's device address on
 * that device, so make that first call before any stream capture.  The
 * address is kept for the process: after cudaDeviceReset on a device the
 * entry point must not be used on that device again.  The call is
 * asynchronous on `stream`: out4 is written when the stream reaches the
 * kernel.  All calls share the one array, so calls that overlap on the GPU
 * (other streams, other host threads, same device) race and must be ordered
 * by the caller.  Errors are reported through lbm_last_error(NULL). */
LBM_API lbm_status lbm_state_stats_noalloc(int32_t q, int64_t cells, const float* populations,
                                           const uint8_t* solid, const float* alpha,
                                           const double* acceleration_lattice, double* out4, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
