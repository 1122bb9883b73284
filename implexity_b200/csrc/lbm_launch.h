// lbm_launch.h -- host-side launchers of the sm_100a kernels (lbm_forward.cu,
// lbm_adjoint.cu, lbm_misc.cu).
// Every launcher enqueues on the given stream and returns the launch status.
#pragma once

#include <cuda_runtime.h>

#include "lbm_common.cuh"

namespace lbm {

// Population storage.  F32 stores g = f - w; F16/BF16 store g/w.  The state
// and the adjoint each live in two arrays (the step reads one and writes the
// other).  Every array carries pop_pad(G) elements of padding before plane 0
// and after the last plane (the staged runs of the stepping kernels read a
// little outside the planes); per-cell float/uint arrays carry CELL_PAD
// elements after the last cell.
constexpr int64_t CELL_PAD = 1024;
inline int64_t pop_pad(const Geometry& G) { return ((G.sx + G.sy + 1 + 2 * CELL_PAD) + 63) / 64 * 64; }
enum StoreKind { ST_F32 = 0, ST_F16 = 1, ST_BF16 = 2 };
// BGK runs as PAIRS with om == omega; MRT_BULK is MRT whose only correction is
// the bulk moment of the Gram-Schmidt basis (b = |c|^2 - 1), folded at compile time
enum CollKind { CK_PAIRS = 0, CK_MRT = 1, CK_MRT_BULK = 2 };

struct FwdArgs {
    Geometry G;
    Physics P;
    const void* src;         // current array: Q planes of n cells (storage type)
    void* dst;               // output array of the step
    const uint32_t* mask;
    const float* alpha;
    const PortMap* ports;
    int32_t apply_ports;     // the stored state still needs the port reconstruction
    StepDiag* diag;          // per-state admission output (nullptr: off)
    Reduce red;
    float* record;           // (rho-1, ux, uy, uz) planes (nullptr: off)
    int32_t record_s;        // also record the six second moments of g (planes 4..9)
    int32_t collide;         // 0: only load/diag/record (no collision, no store)
    int32_t bulk_store;      // full tiles leave through bulk stores (planes 16-byte aligned)
    uint32_t step;           // absolute step index (seeds the stochastic rounding)
    int* err;                // set when a bounded wait gave up
    // response sums of the state the step reads (16 doubles: 8 compensated
    // sums; nullptr: off), with their own reduction scratch
    double* stage;
    Reduce red2;
    const float* phi;        // design density (response 5)
    SeedParams sp;           // unit conversions of the responses (w unused)
    // staged pull runs: element offset of each direction's 16-byte aligned
    // run for the tile at x0 = 0, and the offset of the tile's first element
    // inside it
    int64_t run0[27];
    int32_t rund[27];
    int32_t dp_collision;    // FP64 collision arithmetic (FP32 storage)
    const float* omega_cell; // per-cell relaxation rate 1/tau (BGK; nullptr: the uniform rate of P)
};

struct AdjArgs {
    Geometry G;
    Physics P;
    const void* src;         // current adjoint array: Q planes of n cells (lambda storage type)
    void* dst;               // output array of the transposed step
    const uint32_t* mask;
    const float* alpha;
    const PortMap* ports;
    const float* record;     // (rho-1, ux, uy, uz[, S xx yy zz xy xz yz]) of the forward state
    int32_t rec_planes;      // 4, or 10 with the second moments (stage seeds)
    int32_t stage;           // add the response VJP of this state (stage objective)
    SeedParams seed;         // weights and scales of that VJP
    float* abar;             // accumulated alpha cotangent
    int32_t port_transpose;  // store Ports^T lambda (1) or lambda itself (0)
    int32_t overwrite_abar;  // abar = (1) or += (0)
    float in_scale_inv;      // true = stored * in_scale_inv
    float out_scale;         // stored = true * out_scale
    float abar_factor;       // abar += factor * d(loss)/d(alpha)
    double* norm2;           // sum of squares of the stored lambda (true units * out_scale), nullptr: off
    Reduce red;
    int* err;                // set when a bounded wait gave up
    int64_t run0[27];        // staged adjoint runs (see FwdArgs)
    int32_t rund[27];
    int64_t rec0[10];        // staged record runs
    int32_t recd[10];
    const float* omega_cell; // per-cell relaxation rate 1/tau (BGK; nullptr: the uniform rate of P)
};

struct ObjArgs {
    Geometry G;
    Physics P;
    const void* pop;
    const uint32_t* mask;
    const float* alpha;
    const float* phi;
    const PortMap* ports;
    int32_t apply_ports;
    float tau;
    // response scales
    float vel, dens, dt_s;
    double w[8];             // weights after the reference's scalings (seed only)
    // outputs
    double* sums;            // responses: 16 doubles (8 compensated pairs)
    Reduce red;
    float* fields;           // optional (rho-1, ux, uy, uz) planes
    // seed outputs
    void* lam;
    float lam_scale;
    float* abar_final;
    float* phibar;
    float* record;
    double* norm2;
    int32_t write_lambda;
    int32_t port_transpose;
    uint32_t c_begin, c_end;  // cells taken into account (an x-slab's owned range; 0, n otherwise)
};

struct DesignArgs {
    Geometry G;
    const float* raw;
    const uint8_t* cls;      // 0 solid, 1 editable, 2 fixed
    const float* fixed;
    const int4* offsets;     // (dx, dy, dz, float-bits weight)
    int32_t n_offsets;
    float beta, eta, proj_a, proj_den;
    float ramp_c, ramp_q;    // alpha = c (1-phi)/(q+phi), c = dt*drag_max*q
    float* phi;
    float* alpha;
    float* den;
    float* slope;
    // sensitivity
    const float* phibar;
    const float* abar;
    const float* abar_final;
    float abar_scale;
    float* scale;
    float* grad;
};

// Fills run0/rund for a tile-staged kernel: direction q's run starts at the
// first used element q*n + x0 + dir*lin(q) (dir -1: forward pull, +1:
// adjoint pull), aligned down to `vec` elements.
void run_table(int Q, const Geometry& G, int dir, int vec, int64_t* run0, int32_t* rund);
// True when base and every run start base + run0[q]*elem are 16-byte aligned.
bool staged_aligned(const void* base, const int64_t* run0, int nrun, size_t elem);

// Sets the message lbm_last_error(NULL) returns on this thread (entry points
// that take no handle report through it).
void set_thread_error(const char* msg);

cudaError_t launch_init(int Q, int storage, const Geometry& G, const Physics& P, void* pop, const uint32_t* mask,
                        int64_t c_begin, int64_t c_end, cudaStream_t s);  // cells [c_begin, c_end)
cudaError_t launch_forward(int Q, int coll, int storage, const FwdArgs& a, int grid, cudaStream_t s);
cudaError_t launch_adjoint(int Q, int coll, int lstorage, const AdjArgs& a, int grid, cudaStream_t s);
cudaError_t launch_wait_probe(int* err, uint64_t limit_ns, unsigned long long* waited_ns, cudaStream_t s);
cudaError_t launch_objective(int Q, int storage, int lstorage, int mode, const ObjArgs& a, int grid,
                             cudaStream_t s);  // mode 0: responses/fields, 1: seed
cudaError_t launch_canon_pop(int Q, int storage, const Geometry& G, const void* pop, const uint32_t* mask,
                             const PortMap* ports, int apply_ports, float* out, int grid, cudaStream_t s);
cudaError_t launch_upload_pop(int Q, int storage, const Geometry& G, void* pop, const uint32_t* mask,
                              const float* in, int grid, cudaStream_t s);
cudaError_t launch_wall_loads(int Q, int storage, const Geometry& G, const Physics& P, const void* A,
                              const uint32_t* mask, const float* alpha, const PortMap* ports, int apply_ports,
                              const uint32_t* cells, const uint8_t* links, int64_t n_links, double* out,
                              const float* omega_cell, cudaStream_t s);
// Per-cell cotangent of the relaxation time of one step (interval_vjp with
// Tau::PerCell, solver.rs:214-285 tau_bar): g = canonical populations g = f - w
// of the state, lam = the stored cotangent of the next state (FP32).
cudaError_t launch_tau_bar(int Q, const Geometry& G, const Physics& P, const float* g, const float* lam,
                           const uint32_t* mask, const float* alpha, const float* omega_cell, double* out, int grid,
                           cudaStream_t s);
// Slab halos: directions `dirs` of the x plane starting at cell plane0 (sx
// cells) of a stored array (storage type) to (unpack = 0) or from (1) buf.
cudaError_t launch_halo_copy(int storage, void* arr, int64_t n, int64_t plane0, int64_t sx, const int32_t* dirs,
                             int ndir, void* buf, int unpack, cudaStream_t s);
cudaError_t launch_canon_lam(int Q, int lstorage, const Geometry& G, const void* lam, const uint32_t* mask,
                             float inv_scale, float* out, int grid, cudaStream_t s);
// rec_next: the (rho-1, u) record of the state lambda belongs to (read at
// the neighbours of extrapolating port cells; nullptr without such ports)
cudaError_t launch_seed_lam(int Q, int lstorage, const Geometry& G, void* lam, const uint32_t* mask,
                            const PortMap* ports, const float* in, float scale, int port_transpose,
                            const float* rec_next, const float* alpha, int grid, cudaStream_t s);
// Moves the neighbour's share of one extrapolating port's cotangents
// (left in the port cells' slots) into the neighbours' slots.
cudaError_t launch_nee_move(int lstorage, void* lam, int64_t n, int Q, const uint32_t* cells, int64_t count,
                            int64_t nb_off, cudaStream_t s);
cudaError_t launch_design_map(const DesignArgs& a, int grid, cudaStream_t s);
cudaError_t launch_sens_scale(const DesignArgs& a, int grid, cudaStream_t s);
cudaError_t launch_filter_transpose(const DesignArgs& a, int grid, cudaStream_t s);

}  // namespace lbm
