// lbm_common.cuh -- lattice tables, cell-mask layout and kernel argument
// blocks shared by the sm_100a kernels (lbm_forward.cu, lbm_adjoint.cu,
// lbm_misc.cu, lbm_noalloc.cu) and the host runtime (lbm_runtime.cpp).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define LBM_HD __host__ __device__ __forceinline__
#else
#define LBM_HD inline
#endif

namespace lbm {

// ------------------------------------------------------------------ lattices
// D3Q19 velocity ordering of d3q19.rs:29-51 and D3Q27 ordering of
// moving/lattice.rs:93-121.  Both are "rest first, then the moving velocities
// in lexicographic (x, y, z) order", so opposite(q) = Q - q for q >= 1.
template <int Q>
struct Lat;

template <>
struct Lat<19> {
    static constexpr int Q = 19;
    static constexpr int NPAIR = 9;
    LBM_HD static constexpr int cx(int q) {
        constexpr int t[19] = {0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1};
        return t[q];
    }
    LBM_HD static constexpr int cy(int q) {
        constexpr int t[19] = {0, -1, 0, 0, 0, 1, -1, -1, -1, 0, 0, 1, 1, 1, -1, 0, 0, 0, 1};
        return t[q];
    }
    LBM_HD static constexpr int cz(int q) {
        constexpr int t[19] = {0, 0, -1, 0, 1, 0, -1, 0, 1, -1, 1, -1, 0, 1, 0, -1, 0, 1, 0};
        return t[q];
    }
    LBM_HD static constexpr float w(int q) {
        return q == 0 ? 1.0f / 3.0f
                      : ((cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q)) == 1 ? 1.0f / 18.0f : 1.0f / 36.0f);
    }
    LBM_HD static constexpr double wd(int q) {
        return q == 0 ? 1.0 / 3.0 : ((cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q)) == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
};

template <>
struct Lat<27> {
    static constexpr int Q = 27;
    static constexpr int NPAIR = 13;
    // index n >= 1 enumerates (a, b, c) in {-1,0,1}^3 \ {0} with c fastest
    LBM_HD static constexpr int code(int q) { return q == 0 ? 13 : (q <= 13 ? q - 1 : q); }
    LBM_HD static constexpr int cx(int q) { return code(q) / 9 - 1; }
    LBM_HD static constexpr int cy(int q) { return (code(q) / 3) % 3 - 1; }
    LBM_HD static constexpr int cz(int q) { return code(q) % 3 - 1; }
    LBM_HD static constexpr float w(int q) {
        return q == 0 ? 8.0f / 27.0f
                      : ((cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q)) == 1
                             ? 2.0f / 27.0f
                             : ((cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q)) == 2 ? 1.0f / 54.0f : 1.0f / 216.0f));
    }
    LBM_HD static constexpr double wd(int q) {
        return q == 0 ? 8.0 / 27.0
                      : ((cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q)) == 1
                             ? 2.0 / 27.0
                             : ((cx(q) * cx(q) + cy(q) * cy(q) + cz(q) * cz(q)) == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
};

template <int Q>
LBM_HD constexpr int opp(int q) {
    return q == 0 ? 0 : Q - q;
}

// ------------------------------------------------------------------ cell mask
// One 32-bit word per cell:
//   bits 0..Q-1  link q blocked for the pull of this cell: the cell x - c_q is
//                solid or outside a closed face (Streaming::new,
//                solver.rs:84-93).  Halfway bounce-back applies there.
//   bit 27       the cell touches a periodic face: neighbour indices wrap
//   bits 28..30  port index + 1 (0: not a port cell)
//   bit 31       solid cell (inert; never read or written by the stepping)
constexpr uint32_t MASK_WRAP = 1u << 27;
constexpr uint32_t LINK_BITS = (1u << 27) - 1u;  // the per-direction blocked-link bits
constexpr uint32_t MASK_PORT_SHIFT = 28;
constexpr uint32_t MASK_PORT = 7u << 28;
constexpr uint32_t MASK_SOLID = 1u << 31;

constexpr int MAX_PORTS = 7;
constexpr int MAX_UNKNOWN = 9;  // populations entering through a face (D3Q27)
constexpr int MAX_PROJ = 8;     // MRT rank-one corrections (bulk + even-high)

// Port reconstruction as an affine map of the streamed populations in
// shifted form g = f - w (ports.rs:343-406 is affine in f for fixed port
// values): g_out[r] = bias[r] + sum_k jac[r][k] g_in[k] for the unknown
// populations r; the other populations pass unchanged.
struct PortMap {
    uint32_t unknown_mask;  // bit q: population q is replaced
    float dp_weight;        // +1/n_inlet (velocity port), -1/n_outlet (pressure port)
    float bias[27];
    float jac[27][27];      // rows of the unknown populations
    // extrapolating ports (recon != 0): every population from the inward
    // neighbour x + nb_off, f = eq(rho_b, u_b) + f_n - eq(rho_n, u_n), where
    // rho_b = rho_n when rb_nb, else 1 + rb1, and u_b[d] = u_n[d] where bit d
    // of ub_nb is set, else u_port[d]
    int32_t recon;
    int32_t nb_off;
    int32_t rb_nb, ub_nb;
    float rb1;
    float u_port[3];
    // regularized known-stress port (recon 3): the least-squares stress fit
    // over the known populations, stress[r] = sum_q sop[r][q] (f_q - eq_q)
    // (zero columns for the unknown populations)
    float sop[6][27];
};

// ------------------------------------------------------------------ arguments
struct Geometry {
    int64_t n;        // cells
    int32_t nx, ny, nz;
    int32_t periodic; // bit a: axis a periodic
    int64_t sx, sy;   // linear strides of axes 0 and 1 (axis 2 is contiguous)
};

struct Physics {
    float a[3];       // lattice acceleration
    float omega;      // shear / symmetric rate 1/tau
    float om;         // odd / antisymmetric rate (TRT magic)
    int32_t n_proj;   // MRT corrections
    float proj_rate[MAX_PROJ];     // (s_g - omega) for each corrected moment
    float proj_left[MAX_PROJ][27]; // w_i b_i / |b|^2_W  (reconstruction side)
    float proj_right[MAX_PROJ][27];// b_i                (projection side)
    float proj_lw[MAX_PROJ][27];   // b_i / |b|^2_W      (reconstruction side, in (f-w)/w units)
    float proj_m0[MAX_PROJ];       // sum_i w_i b_i
    float proj_m2[MAX_PROJ][6];    // sum_i w_i b_i c_ia c_ib (xx yy zz xy xz yz)
};

// Weights (after the reference's scalings) and unit scales of the response
// VJP (response_vjp in lbm_device.cuh).
struct SeedParams {
    float w[8];
    float vel, dens, dt_s, tau;
};

// Per-step admission reductions (solver.rs:714-755) for one state.
struct StepDiag {
    double mass_hi, mass_lo;  // sum of rho over fluid cells (compensated)
    double exch_hi, exch_lo;  // port exchange of the step that produced the state
    float min_f;              // minimum population over fluid cells
    float max_u2;             // maximum |u|^2 over fluid cells
    int32_t nonfinite;
    int32_t pad;
};

struct Reduce {
    double* partial;       // per-block scratch
    unsigned int* counter; // last-block ticket
};

}  // namespace lbm
