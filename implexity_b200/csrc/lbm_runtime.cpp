// lbm_runtime.cpp -- host runtime behind the C-ABI of include/lbm_b200.h:
// problem validation and normalisation (with the reference's contract
// messages), link masks, port maps and design filter, device memory, the
// forward / adjoint schedules and the admission record.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_common.cuh"
#include "lbm_launch.h"
#include "lbm_revolve.h"

using namespace lbm;

namespace {

thread_local std::string g_create_error;

struct ContractError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct ConvergenceError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define CK(expr)                                                                                   \
    do {                                                                                           \
        cudaError_t _e = (expr);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            throw CudaError(std::string(#expr) + ": " + cudaGetErrorString(_e));                   \
    } while (0)

// Python-style shortest float repr (implexity_core::py_repr::repr_float).
std::string repr_float(double v) {
    if (std::isnan(v)) return "nan";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific);
    std::string sci(buf, r.ptr);
    // split mantissa digits and exponent
    size_t epos = sci.find('e');
    std::string mant = sci.substr(0, epos);
    int exp10 = std::stoi(sci.substr(epos + 1));
    bool neg = !mant.empty() && mant[0] == '-';
    if (neg) mant = mant.substr(1);
    std::string digits;
    for (char c : mant)
        if (c != '.') digits += c;
    std::string out;
    if (exp10 >= -4 && exp10 < 16) {
        if (exp10 >= 0) {
            if ((int)digits.size() <= exp10 + 1) out = digits + std::string(exp10 + 1 - digits.size(), '0') + ".0";
            else out = digits.substr(0, exp10 + 1) + "." + digits.substr(exp10 + 1);
        } else {
            out = "0." + std::string(-exp10 - 1, '0') + digits;
        }
    } else {
        out = digits.substr(0, 1);
        if (digits.size() > 1) out += "." + digits.substr(1);
        char e[16];
        std::snprintf(e, sizeof(e), "e%c%02d", exp10 < 0 ? '-' : '+', std::abs(exp10));
        out += e;
    }
    return neg ? "-" + out : out;
}

// ------------------------------------------------------------ lattice (host)
struct HostLat {
    int Q;
    int c[27][3];
    double w[27];
    int opp[27];
};
template <int Q>
HostLat host_lat_t() {
    HostLat L;
    L.Q = Q;
    for (int q = 0; q < Q; ++q) {
        L.c[q][0] = Lat<Q>::cx(q);
        L.c[q][1] = Lat<Q>::cy(q);
        L.c[q][2] = Lat<Q>::cz(q);
        L.w[q] = Lat<Q>::wd(q);
        L.opp[q] = opp<Q>(q);
    }
    return L;
}
HostLat host_lat(int Q) { return Q == 19 ? host_lat_t<19>() : host_lat_t<27>(); }

// Gram-Schmidt moment basis (moving/collision.rs:87-153): candidate
// polynomials mass, momentum, bulk |c|^2, shear, then the monomials of
// degree 3..6 with exponents <= 2, orthogonalised in the w-weighted inner
// product.  Returns rows/norms/groups (0 mass 1 momentum 2 bulk 3 shear
// 4 odd 5 even-high) or false if the basis is incomplete.
bool moment_basis(const HostLat& L, std::vector<std::vector<double>>& rows, std::vector<double>& norms,
                  std::vector<int>& groups) {
    const int Q = L.Q;
    std::vector<std::pair<std::vector<double>, int>> cand;
    auto add = [&](auto fn, int g) {
        std::vector<double> p(Q);
        for (int i = 0; i < Q; ++i) p[i] = fn(L.c[i][0], L.c[i][1], L.c[i][2]);
        cand.push_back({p, g});
    };
    add([](int, int, int) { return 1.0; }, 0);
    add([](int x, int, int) { return (double)x; }, 1);
    add([](int, int y, int) { return (double)y; }, 1);
    add([](int, int, int z) { return (double)z; }, 1);
    add([](int x, int y, int z) { return (double)(x * x + y * y + z * z); }, 2);
    add([](int x, int y, int z) { return (double)(2 * x * x - y * y - z * z); }, 3);
    add([](int, int y, int z) { return (double)(y * y - z * z); }, 3);
    add([](int x, int y, int) { return (double)(x * y); }, 3);
    add([](int x, int, int z) { return (double)(x * z); }, 3);
    add([](int, int y, int z) { return (double)(y * z); }, 3);
    for (int deg = 3; deg <= 6; ++deg)
        for (int a = 0; a <= 2; ++a)
            for (int b = 0; b <= 2; ++b) {
                int c = deg - a - b;
                if (c < 0 || c > 2) continue;
                add([=](int x, int y, int z) { return std::pow(x, a) * std::pow(y, b) * std::pow(z, c); },
                    deg % 2 ? 4 : 5);
            }
    auto inner = [&](const std::vector<double>& x, const std::vector<double>& y) {
        double s = 0;
        for (int i = 0; i < Q; ++i) s += L.w[i] * x[i] * y[i];
        return s;
    };
    rows.clear();
    norms.clear();
    groups.clear();
    for (auto& [p, g] : cand) {
        if ((int)rows.size() == Q) break;
        double scale = inner(p, p);
        if (scale <= 0) continue;
        std::vector<double> v = p;
        for (size_t k = 0; k < rows.size(); ++k) {
            double coef = inner(p, rows[k]) / norms[k];
            for (int i = 0; i < Q; ++i) v[i] -= coef * rows[k][i];
        }
        double n = inner(v, v);
        if (n <= 1e-10 * scale) continue;
        rows.push_back(v);
        norms.push_back(n);
        groups.push_back(g);
    }
    return (int)rows.size() == Q;
}

// Legacy-moment port reconstruction (ports.rs:343-406) in FP64, used once
// per port to tabulate its affine map.
struct PortSpec {
    bool pressure;
    int axis, sign;
    double vel[3];
    double density;
    // pulsatile signal (moving/boundary.rs:98-126): value(t) = ramp(t) (wave(t) amplitude + mean)
    bool pulsatile = false;
    double mean_vel[3] = {0, 0, 0}, amp_vel[3] = {0, 0, 0};  // lattice units
    double mean_rho = 1.0, amp_rho = 0.0;                     // lattice density (mean includes 1)
    double freq = 0, phase = 0, ramp = 0;
    int recon = LBM_RECON_LEGACY_MOMENT;  // lbm_port_reconstruction
    int64_t nb_off = 0;                   // inward neighbour offset (extrapolating ports)
    double sop[6][27] = {};               // regularized port: the known-stress fit
};

// The regularized port's stress fit (ports.rs known_stress_operator
// :409-439): the weighted least-squares inverse of the deviatoric basis
// B_qr = 4.5 w_q (c_a c_b - delta_ab / 3) over the known populations
// (c_axis != sign), sop[r][q] = sum_c (M^T M)^-1_rc B_qc / w_q with
// M_qc = B_qc / sqrt(w_q); zero for the unknown populations.  False when the
// fit is rank deficient (a pivot below 1e-12 of the largest diagonal).
double stress_basis_h(const HostLat& L, int q, int r) {
    static const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    const double qq = L.c[q][ia[r]] * L.c[q][ib[r]] - (ia[r] == ib[r] ? 1.0 / 3.0 : 0.0);
    return 4.5 * L.w[q] * (r < 3 ? qq : 2.0 * qq);
}

bool regularized_fit(const HostLat& L, int axis, int sign, double (&sop)[6][27]) {
    double A[6][12] = {};
    for (int r = 0; r < 6; ++r) {
        for (int c = 0; c < 6; ++c)
            for (int q = 0; q < L.Q; ++q)
                if (L.c[q][axis] != sign) A[r][c] += stress_basis_h(L, q, r) * stress_basis_h(L, q, c) / L.w[q];
        A[r][6 + r] = 1.0;
    }
    double big = 0.0;
    for (int r = 0; r < 6; ++r) big = std::max(big, std::fabs(A[r][r]));
    for (int c = 0; c < 6; ++c) {
        int piv = c;
        for (int r = c + 1; r < 6; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        if (!(std::fabs(A[piv][c]) > 1e-12 * big)) return false;
        for (int j = 0; j < 12; ++j) std::swap(A[c][j], A[piv][j]);
        const double d = A[c][c];
        for (int j = 0; j < 12; ++j) A[c][j] /= d;
        for (int r = 0; r < 6; ++r) {
            if (r == c) continue;
            const double m = A[r][c];
            for (int j = 0; j < 12; ++j) A[r][j] -= m * A[c][j];
        }
    }
    for (int r = 0; r < 6; ++r)
        for (int q = 0; q < 27; ++q) {
            double acc = 0.0;
            if (q < L.Q && L.c[q][axis] != sign)
                for (int c = 0; c < 6; ++c) acc += A[r][6 + c] * stress_basis_h(L, q, c);
            sop[r][q] = q < L.Q ? acc / L.w[q] : 0.0;
        }
    return true;
}

// Signal::factors (moving/boundary.rs:111-125): the C2 smoothstep ramp and
// the sine wave at time t seconds.
void signal_factors(const PortSpec& p, double t, double& ramp, double& wave) {
    ramp = 1.0;
    if (p.ramp > 0.0 && t < p.ramp) {
        double s = t / p.ramp;
        if (s < 0.0) s = 0.0;
        ramp = s * s * s * (10.0 - s * 15.0 + s * s * 6.0);
    }
    wave = p.freq == 0.0 ? 0.0 : std::sin(t * (2.0 * M_PI * p.freq) + p.phase);
}

// The port's values for the reconstruction producing the state at time t
// seconds (moving/field.rs:1002-1013).
PortSpec spec_at(const PortSpec& p, double t) {
    PortSpec q = p;
    if (!p.pulsatile) return q;
    double ramp, wave;
    signal_factors(p, t, ramp, wave);
    for (int d = 0; d < 3; ++d) q.vel[d] = ramp * (wave * p.amp_vel[d] + p.mean_vel[d]);
    if (p.pressure) q.density = 1.0 + ramp * (wave * p.amp_rho + (p.mean_rho - 1.0));
    return q;
}

void reconstruct(const HostLat& L, const PortSpec& p, const double a[3], const double* f, double* out) {
    const int Q = L.Q;
    std::vector<int> unknown;
    double compat = 0, out_sum = 0;
    for (int q = 0; q < Q; ++q) {
        if (L.c[q][p.axis] == p.sign) unknown.push_back(q);
        else if (L.c[q][p.axis] == -p.sign) out_sum += f[q];
        else compat += f[q];
    }
    compat += 2.0 * out_sum;
    int t[2], nt = 0;
    for (int d = 0; d < 3; ++d)
        if (d != p.axis) t[nt++] = d;
    double v[3];
    for (int d = 0; d < 3; ++d) v[d] = p.vel[d] - 0.5 * a[d];
    double rho;
    if (!p.pressure) rho = compat / (1.0 - p.sign * v[p.axis]);
    else {
        rho = p.density;
        v[p.axis] = (1.0 - compat / rho) * p.sign;
    }
    const int U = (int)unknown.size();
    std::vector<double> prop(U);
    for (int k = 0; k < U; ++k) {
        int q = unknown[k];
        double cv = L.c[q][0] * v[0] + L.c[q][1] * v[1] + L.c[q][2] * v[2];
        prop[k] = f[L.opp[q]] + rho * 6.0 * L.w[q] * cv;
    }
    double km = 0, kj[3] = {0, 0, 0};
    for (int q = 0; q < Q; ++q) {
        if (L.c[q][p.axis] == p.sign) continue;
        km += f[q];
        for (int d = 0; d < 3; ++d) kj[d] += f[q] * L.c[q][d];
    }
    double target[3] = {rho - km, rho * v[t[0]] - kj[t[0]], rho * v[t[1]] - kj[t[1]]};
    double pa[3] = {0, 0, 0};
    double R[3][9];
    for (int k = 0; k < U; ++k) {
        int q = unknown[k];
        R[0][k] = 1.0;
        R[1][k] = L.c[q][t[0]];
        R[2][k] = L.c[q][t[1]];
        for (int r = 0; r < 3; ++r) pa[r] += prop[k] * R[r][k];
    }
    double res[3] = {target[0] - pa[0], target[1] - pa[1], target[2] - pa[2]};
    double M[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < U; ++k) s += R[i][k] * R[j][k];
            M[i][j] = s;
        }
    // 3x3 inverse by cofactors
    double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                 M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    double inv[3][3] = {};
    if (det != 0.0) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                int i1 = (j + 1) % 3, i2 = (j + 2) % 3, j1 = (i + 1) % 3, j2 = (i + 2) % 3;
                inv[i][j] = (M[i1][j1] * M[i2][j2] - M[i1][j2] * M[i2][j1]) / det;
            }
    }
    for (int q = 0; q < Q; ++q) out[q] = f[q];
    for (int k = 0; k < U; ++k) {
        double corr = 0;
        for (int j = 0; j < 3; ++j) {
            double rij = R[0][k] * inv[0][j] + R[1][k] * inv[1][j] + R[2][k] * inv[2][j];
            corr += res[j] * rij;
        }
        out[unknown[k]] = prop[k] + corr;
    }
}

// ------------------------------------------------------------ device buffers
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int64_t* counter = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { reset(); }
    void reset() {
        if (p) {
            cudaFree(p);
            if (counter) *counter -= (int64_t)bytes;
        }
        p = nullptr;
        bytes = 0;
    }
    // exactly b bytes (releases a larger buffer)
    void fit(size_t b, int64_t* ctr) {
        if (p && bytes != b) reset();
        alloc(b, ctr);
    }
    void alloc(size_t b, int64_t* ctr) {
        if (p && bytes >= b) return;
        reset();
        counter = ctr;
        CK(cudaMalloc(&p, b));
        bytes = b;
        if (counter) *counter += (int64_t)b;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

size_t storage_bytes(int s) { return s == LBM_STORE_F32 ? 4 : 2; }

}  // namespace

struct Checkpoint {
    std::unique_ptr<DevBuf> buf;  // the current population array (one of the two)
    int64_t t;
    bool pending;
};

namespace {
struct AdjState;
}  // namespace

struct lbm_handle {
    // --- normalised problem
    int Q = 19, coll = LBM_BGK, storage = LBM_STORE_F32;
    bool collision_fp64 = false;  // FP64 collision arithmetic on FP32 storage
    // Tau::PerCell (solver.rs:171-187): per-cell rates 1/tau of the BGK collision (FP32), when set
    bool tau_per_cell = false;
    Geometry G{};
    Physics P{};
    HostLat L{};
    double tau = 0, omega = 0, om = 0;
    double a[3] = {0, 0, 0};
    int64_t step_count = 0;
    double dx = 0, dt = 0, density = 0, mach_limit = 0, drag_max = 0, drag_shape = 0;
    int64_t fluid_cells = 0, n_inlet = 0, n_outlet = 0;
    int n_ports = 0;
    std::vector<uint8_t> cls;
    std::vector<int4> offsets;
    float beta = 0, eta = 0.5f, proj_a = 0, proj_den = 1;
    // --- device
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t device_bytes = 0;
    DevBuf pop, mask, alpha, phi, raw, den, slope, cls_d, fixed_d, offsets_d, ports_d, partial, counter, diag;
    DevBuf lam, record, abar, abar_final, phibar, scale, grad, norm2, sums, scratch, errflag;
    DevBuf omega_cell, tau_state, tau_bar;
    AdjState* slab_adj = nullptr;  // x-slab steady adjoint in progress (lbm_slab_adjoint_begin)
    int lam_storage = LBM_STORE_F32;
    // --- ports: normalised specs with their signals; pulsatile ports keep one
    // set of maps per state index on the device (ensure_port_maps)
    std::vector<PortSpec> port_specs;
    bool pulsatile = false;
    int64_t map_states = 0;
    std::vector<PortMap> maps_host;
    // --- stage objective: the responses of every state of the last forward
    bool time_average = false;
    DevBuf tsums;
    double tavg[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool tavg_valid = false;
    int64_t peak_extra = 0;  // second-level checkpoint bytes of the last horizon gradient
    std::vector<Checkpoint> ckpts;
    std::vector<StepDiag> last_trajectory;
    bool bulk_only = false;  // MRT: the single correction is the bulk moment |c|^2 - 1
    // fixed-wall links of the momentum-exchange loads (wall_exchange.rs layout)
    std::vector<uint32_t> wall_cells;
    std::vector<uint8_t> wall_links;
    DevBuf wall_cells_d, wall_links_d, wall_out;
    // cells of the extrapolating ports, grouped by port: (first, count,
    // port) per group; their transposes move cotangents to the neighbours
    std::vector<std::array<int64_t, 3>> nee_groups;
    DevBuf nee_cells_d;
    bool nonlinear_ports = false;  // a port other than legacy_moment (transposes read a record)
    // --- state
    bool design_set = false, state_valid = false, forward_done = false;
    int cur = 0;   // which population array holds the current state
    int lcur = 0;  // which adjoint array holds the current adjoint state
    bool pending = false;
    // a non-finite population was loaded into a solid cell (lbm_set_populations):
    // solid cells are never stepped, so every later state carries it too
    bool solid_nonfinite = false;
    // x-slab of a larger problem (lbm_create_slab): the owned planes are
    // [slab_hl, slab_hl + slab_own) of the local grid, the others ghost planes;
    // responses, seeds and port pressure weights use the whole problem's counts
    bool slab = false;
    int32_t slab_hl = 0, slab_hr = 0, slab_own = 0;
    int64_t global_fluid = -1, global_inlet = -1, global_outlet = -1;
    int64_t t = 0;
    std::string err;

    int64_t n() const { return G.n; }
    // One array (Q planes plus front and back padding) of the given storage,
    // rounded up so that the second array starts 256-byte aligned like the
    // first (the staged bulk copies need 16-byte aligned runs in both).
    size_t array_bytes(int st) const {
        const size_t b = ((size_t)G.n * Q + 2 * pop_pad(G)) * (st == LBM_STORE_F32 ? 4 : 2);
        return (b + 255) / 256 * 256;
    }
    char* pop_array(int k) const { return static_cast<char*>(pop.p) + (size_t)k * array_bytes(storage); }
    // planes start after the front padding: current (A) and other (B) array
    // A stored state (a checkpoint buffer laid out like a population array)
    // that stands for the current state until the next step: the step reads
    // it in place of the current array, so restoring a state needs no copy.
    const char* restored = nullptr;
    void* popA() const {
        const char* base = restored ? restored : pop_array(cur);
        return const_cast<char*>(base) + pop_pad(G) * (storage == LBM_STORE_F32 ? 4 : 2);
    }
    void* popB() const { return pop_array(cur ^ 1) + pop_pad(G) * (storage == LBM_STORE_F32 ? 4 : 2); }
    void* lam_plane0(int k) const {
        return static_cast<char*>(lam.p) + (size_t)k * array_bytes(lam_storage) +
               pop_pad(G) * (lam_storage == LBM_STORE_F32 ? 4 : 2);
    }
    void* lamA() const { return lam_plane0(lcur); }
    void* lamB() const { return lam_plane0(lcur ^ 1); }
};

namespace {

// ------------------------------------------------------------ validation
void require(bool ok, const char* msg) {
    if (!ok) throw ContractError(msg);
}
bool finite_positive(double v) { return std::isfinite(v) && v > 0; }

// Counts that scale the responses: the whole problem's for an x-slab.
int64_t resp_fluid(const lbm_handle& h) { return h.global_fluid >= 0 ? h.global_fluid : h.fluid_cells; }
bool resp_both_ports(const lbm_handle& h) {
    return (h.global_inlet >= 0 ? h.global_inlet : h.n_inlet) > 0 && (h.global_outlet >= 0 ? h.global_outlet : h.n_outlet) > 0;
}

// The affine port maps (shifted variables) of every port for the values in
// force at time t seconds: bias and Jacobian of the FP64 reconstruction over
// the unknown populations, tabulated at the weights.
std::vector<PortMap> port_maps_at(const lbm_handle& h, double t_s) {
    std::vector<PortMap> maps(h.port_specs.size());
    const int Q = h.Q;
    for (size_t k = 0; k < h.port_specs.size(); ++k) {
        const PortSpec spec = spec_at(h.port_specs[k], t_s);
        PortMap& M = maps[k];
        std::memset(&M, 0, sizeof(M));
        double base[27] = {}, pert[27] = {}, r0[27] = {}, r1[27] = {};
        for (int q = 0; q < Q; ++q) base[q] = h.L.w[q];
        reconstruct(h.L, spec, h.a, base, r0);
        for (int q = 0; q < Q; ++q)
            if (h.L.c[q][spec.axis] == spec.sign) M.unknown_mask |= 1u << q;
        for (int r = 0; r < Q; ++r)
            if (M.unknown_mask & (1u << r)) M.bias[r] = (float)(r0[r] - h.L.w[r]);
        for (int kq = 0; kq < Q; ++kq) {
            for (int q = 0; q < Q; ++q) pert[q] = base[q];
            pert[kq] += 1.0;
            reconstruct(h.L, spec, h.a, pert, r1);
            for (int r = 0; r < Q; ++r)
                if (M.unknown_mask & (1u << r)) M.jac[r][kq] = (float)(r1[r] - r0[r]);
        }
        // extrapolating ports: which of the boundary density / velocity the
        // neighbour supplies (ports.rs:484-497, moving/boundary.rs:445-458)
        M.recon = spec.recon;
        if (spec.recon == LBM_RECON_REGULARIZED_KNOWN_STRESS)
            for (int r = 0; r < 6; ++r)
                for (int q = 0; q < 27; ++q) M.sop[r][q] = (float)spec.sop[r][q];
        if (spec.recon == LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM || spec.recon == LBM_RECON_NON_EQUILIBRIUM_EXTRAPOLATION) {
            M.nb_off = (int32_t)spec.nb_off;
            const bool neighbor = spec.recon == LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM;
            M.rb_nb = (!neighbor && !spec.pressure) ? 1 : 0;
            M.ub_nb = neighbor ? (1 << spec.axis) : (spec.pressure ? 7 : 0);
            M.rb1 = (float)(spec.density - 1.0);
            for (int d = 0; d < 3; ++d) M.u_port[d] = (float)spec.vel[d];
        }
        const int64_t ni = h.global_inlet >= 0 ? h.global_inlet : h.n_inlet;
        const int64_t no = h.global_outlet >= 0 ? h.global_outlet : h.n_outlet;
        M.dp_weight = !resp_both_ports(h) ? 0.f : spec.pressure ? (float)(-1.0 / no) : (float)(1.0 / ni);
    }
    return maps;
}

// Pulsatile ports: the maps of the reconstructions producing states
// 0..t_max (state t at time t * step_s) are on the device afterwards.
void ensure_port_maps(lbm_handle& h, int64_t t_max) {
    if (!h.pulsatile || t_max < h.map_states) return;
    const int64_t states = std::max<int64_t>({t_max + 1, 2 * h.map_states, h.step_count + 1});
    h.maps_host.resize((size_t)states * h.n_ports);
    for (int64_t t = h.map_states; t < states; ++t) {
        const std::vector<PortMap> m = port_maps_at(h, (double)t * h.dt);
        std::copy(m.begin(), m.end(), h.maps_host.begin() + (size_t)t * h.n_ports);
    }
    // kernels queued on the stream may still read the old table
    CK(cudaStreamSynchronize(h.stream));
    h.ports_d.reset();
    h.ports_d.alloc(h.maps_host.size() * sizeof(PortMap), &h.device_bytes);
    CK(cudaMemcpy(h.ports_d.p, h.maps_host.data(), h.maps_host.size() * sizeof(PortMap), cudaMemcpyHostToDevice));
    h.map_states = states;
}

// Device port maps in force when state t is loaded.
const PortMap* ports_at(lbm_handle& h, int64_t t) {
    if (!h.pulsatile) return h.ports_d.as<PortMap>();
    ensure_port_maps(h, t);
    return h.ports_d.as<PortMap>() + (size_t)t * h.n_ports;
}

void validate_and_build(lbm_handle& h, const lbm_problem_t& p) {
    // solver.rs:414-550 in order; key-set and array-shape checks belong to the
    // JSON layer of the caller.
    require(p.lattice == 19 || p.lattice == 27, "lattice must be D3Q19 or D3Q27");
    require(p.collision >= LBM_BGK && p.collision <= LBM_MRT, "collision must be bgk, trt or mrt");
    require(p.storage >= LBM_STORE_F32 && p.storage <= LBM_STORE_BF16, "storage must be float32, float16 or bfloat16");
    require(p.shape[0] >= 2 && p.shape[1] >= 2 && p.shape[2] >= 2, "LBM shape must contain three integers >= 2");
    const char* names[7] = {"spacing_m", "step_s", "density_kg_m3", "kinematic_viscosity_m2_s", "drag_max_per_s",
                            "drag_shape", "mach_limit"};
    double vals[7] = {p.spacing_m,      p.step_s,     p.density_kg_m3, p.kinematic_viscosity_m2_s,
                      p.drag_max_per_s, p.drag_shape, p.mach_limit};
    for (int i = 0; i < 7; ++i)
        if (!finite_positive(vals[i])) throw ContractError(std::string(names[i]) + " must be a finite positive scalar");
    require(p.mach_limit <= 0.2, "LBM mach_limit must be <= 0.2; this is not a compressible gas solver");
    require(p.step_count >= 1 && p.step_count <= 1000000, "step_count must be an integer in [1,1000000]");
    const int64_t n = (int64_t)p.shape[0] * p.shape[1] * p.shape[2];
    require(p.solid_mask && p.design_region && p.fixed_design, "solid_mask must be a shape-matched boolean array");
    for (int64_t x = 0; x < n; ++x) {
        double v = p.fixed_design[x];
        require(std::isfinite(v) && v >= 0.0 && v <= 1.0, "fixed_design must be finite and in [0,1]");
    }
    bool all_solid = true, overlap = false;
    for (int64_t x = 0; x < n; ++x) {
        all_solid = all_solid && p.solid_mask[x];
        overlap = overlap || (p.solid_mask[x] && p.design_region[x]);
    }
    require(!all_solid && !overlap, "Need fluid cells; fixed solid cells cannot be designable");
    for (int d = 0; d < 3; ++d)
        require(std::isfinite(p.acceleration_m_s2[d]), "acceleration_m_s2 requires three finite components");
    double tau = 0.5 + 3.0 * p.kinematic_viscosity_m2_s * p.step_s / (p.spacing_m * p.spacing_m);
    require(tau >= 0.51 && tau <= 2.0, "Choose spacing/time step such that 0.51 <= relaxation time <= 2");
    // topology map, design.rs:52-83
    require(std::isfinite(p.filter_radius_m) && std::isfinite(p.projection_beta) && std::isfinite(p.projection_eta),
            "topology_map.filter_radius_m must be finite real scalar");
    require(p.filter_radius_m >= 0.0 && p.filter_radius_m <= 4.0 * p.spacing_m,
            "filter_radius_m must lie in [0,4*spacing_m]");
    require(p.projection_beta >= 0.0 && p.projection_beta <= 32.0 && p.projection_eta > 0.0 && p.projection_eta < 1.0,
            "Require beta in [0,32] and eta in (0,1)");
    require(p.filter_kind == LBM_FILTER_CONIC || p.filter_kind == LBM_FILTER_BOX, "filter_kind must be conic or box");
    require(p.filter_kind != LBM_FILTER_BOX || (p.box_half_width >= 0 && p.box_half_width <= 4),
            "box filter half width must lie in [0,4] cells");
    // collision parameters, moving/collision.rs:236-256
    if (p.collision == LBM_TRT) {
        double m = std::isnan(p.trt_magic) ? 3.0 / 16.0 : p.trt_magic;
        require(std::isfinite(m) && m > 0, "TRT magic parameter must be finite and positive");
    }
    if (p.collision == LBM_MRT) {
        double m = std::isnan(p.mrt_odd_magic) ? 3.0 / 16.0 : p.mrt_odd_magic;
        require(std::isfinite(m) && m > 0, "MRT odd_magic must be finite and positive");
        auto ok = [](double r) { return std::isnan(r) || (std::isfinite(r) && r > 0 && r < 2); };
        require(ok(p.mrt_bulk_rate) && ok(p.mrt_even_rate), "MRT relaxation rates must lie in (0, 2)");
    }

    require((uint64_t)n * (uint64_t)p.lattice < (1ull << 32),
            "grid too large for one device: Q * cells must stay below 2^32 populations");
    require(!p.collision_fp64 || p.storage == LBM_STORE_F32,
            "collision_arithmetic float64 needs population_storage float32");
    h.Q = p.lattice;
    h.coll = p.collision;
    h.storage = p.storage;
    h.collision_fp64 = p.collision_fp64 != 0;
    h.L = host_lat(h.Q);
    h.G.n = n;
    h.G.nx = p.shape[0];
    h.G.ny = p.shape[1];
    h.G.nz = p.shape[2];
    h.G.periodic = (p.periodic_axes[0] ? 1 : 0) | (p.periodic_axes[1] ? 2 : 0) | (p.periodic_axes[2] ? 4 : 0);
    h.G.sx = (int64_t)p.shape[1] * p.shape[2];
    h.G.sy = p.shape[2];
    h.tau = tau;
    h.dx = p.spacing_m;
    h.dt = p.step_s;
    h.density = p.density_kg_m3;
    h.mach_limit = p.mach_limit;
    h.drag_max = p.drag_max_per_s;
    h.drag_shape = p.drag_shape;
    h.step_count = p.step_count;
    for (int d = 0; d < 3; ++d) h.a[d] = p.acceleration_m_s2[d] * p.step_s * p.step_s / p.spacing_m;
    h.omega = 1.0 / tau;
    double magic = p.collision == LBM_MRT ? p.mrt_odd_magic : p.trt_magic;
    if (std::isnan(magic)) magic = 3.0 / 16.0;
    h.om = p.collision == LBM_BGK ? h.omega : 1.0 / (0.5 + magic / (tau - 0.5));
    h.P.omega = (float)h.omega;
    h.P.om = (float)h.om;
    for (int d = 0; d < 3; ++d) h.P.a[d] = (float)h.a[d];
    h.P.n_proj = 0;
    h.bulk_only = false;
    if (p.collision == LBM_MRT) {
        std::vector<std::vector<double>> rows;
        std::vector<double> norms;
        std::vector<int> groups;
        require(moment_basis(h.L, rows, norms, groups), "MRT moment basis is incomplete");
        for (int k = 0; k < h.Q; ++k) {
            double rate;
            if (groups[k] == 2) rate = std::isnan(p.mrt_bulk_rate) ? h.omega : p.mrt_bulk_rate;
            else if (groups[k] == 5) rate = std::isnan(p.mrt_even_rate) ? h.omega : p.mrt_even_rate;
            else continue;
            if (rate == h.omega) continue;
            int j = h.P.n_proj++;
            h.P.proj_rate[j] = (float)(rate - h.omega);
            // the bulk row is |c|^2 - 1 with |b|^2_W = 2/3: the forward step can
            // fold it at compile time when it is the only correction
            bool bulk_row = groups[k] == 2 && std::fabs(norms[k] - 2.0 / 3.0) < 1e-12;
            for (int i = 0; i < h.Q; ++i) {
                const int c2 = h.L.c[i][0] * h.L.c[i][0] + h.L.c[i][1] * h.L.c[i][1] + h.L.c[i][2] * h.L.c[i][2];
                bulk_row = bulk_row && std::fabs(rows[k][i] - (c2 - 1.0)) < 1e-12;
            }
            h.bulk_only = (j == 0) && bulk_row;
            for (int i = 0; i < h.Q; ++i) {
                h.P.proj_left[j][i] = (float)(h.L.w[i] * rows[k][i] / norms[k]);
                h.P.proj_right[j][i] = (float)rows[k][i];
                h.P.proj_lw[j][i] = (float)(rows[k][i] / norms[k]);
            }
            double m0 = 0, m2[6] = {0, 0, 0, 0, 0, 0};
            const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
            for (int i = 0; i < h.Q; ++i) {
                m0 += h.L.w[i] * rows[k][i];
                for (int e = 0; e < 6; ++e) m2[e] += h.L.w[i] * rows[k][i] * h.L.c[i][ia[e]] * h.L.c[i][ib[e]];
            }
            h.P.proj_m0[j] = (float)m0;
            for (int e = 0; e < 6; ++e) h.P.proj_m2[j][e] = (float)m2[e];
        }
    }

    // ports (ports.rs:106-272)
    require(p.n_ports >= 0 && (p.n_ports == 0 || p.ports), "ports must be a list");
    require(p.n_ports <= LBM_MAX_PORTS, "at most 7 ports are supported");
    std::vector<uint8_t> used(n, 0);
    std::vector<PortSpec> specs;
    std::vector<std::vector<int64_t>> port_cells;
    const bool periodic[3] = {p.periodic_axes[0] != 0, p.periodic_axes[1] != 0, p.periodic_axes[2] != 0};
    const int64_t shape[3] = {p.shape[0], p.shape[1], p.shape[2]};
    for (int k = 0; k < p.n_ports; ++k) {
        const lbm_port_t& pt = p.ports[k];
        require(pt.kind == LBM_PORT_VELOCITY || pt.kind == LBM_PORT_PRESSURE, "Port kind must be velocity or pressure");
        require(pt.face >= 0 && pt.face <= 5, "Port must identify one Cartesian face");
        PortSpec s;
        s.pressure = pt.kind == LBM_PORT_PRESSURE;
        s.axis = pt.face / 2;
        s.sign = pt.face % 2 == 0 ? 1 : -1;
        require(!periodic[s.axis], "A periodic face cannot be a port");
        bool any = false;
        if (pt.mask)
            for (int64_t x = 0; x < n; ++x) any = any || pt.mask[x];
        require(any, "Nonempty shape-matched boolean port mask required");
        const int64_t face_index = s.sign == 1 ? 0 : shape[s.axis] - 1;
        std::vector<int64_t> cells;
        for (int64_t x = 0; x < n; ++x) {
            if (!pt.mask[x]) continue;
            int64_t c[3] = {x / h.G.sx, (x / h.G.sy) % shape[1], x % shape[2]};
            require(c[s.axis] == face_index && !used[x], "Port mask must lie on its face and cannot overlap another port");
            cells.push_back(x);
        }
        for (int a2 = 0; a2 < 3; ++a2) {
            if (a2 == s.axis || periodic[a2]) continue;
            for (int64_t x : cells) {
                int64_t c[3] = {x / h.G.sx, (x / h.G.sy) % shape[1], x % shape[2]};
                require(!(c[a2] == 0 || c[a2] == shape[a2] - 1),
                        "Port corners/edges with other closed faces require an unsupported corner closure");
            }
        }
        for (int64_t x : cells)
            require(!(p.solid_mask[x] || p.design_region[x] || p.fixed_design[x] != 1.0),
                    "Port cells must be protected, unobstructed, fixed-design fluid");
        // reconstruction (ports.rs:134-157, 202-219)
        require(pt.reconstruction >= LBM_RECON_LEGACY_MOMENT && pt.reconstruction <= LBM_RECON_REGULARIZED_KNOWN_STRESS,
                "Port reconstruction must be legacy_moment, regularized_known_stress, neighbor_non_equilibrium or "
                "non_equilibrium_extrapolation");
        s.recon = pt.reconstruction;
        const bool accelerated = p.acceleration_m_s2[0] != 0.0 || p.acceleration_m_s2[1] != 0.0 ||
                                 p.acceleration_m_s2[2] != 0.0;
        require(!(s.recon == LBM_RECON_REGULARIZED_KNOWN_STRESS && accelerated),
                "regularized_known_stress ports require zero acceleration; forcing-consistent stress reconstruction is "
                "not implemented");
        require(!(s.recon == LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM && (!s.pressure || accelerated)),
                "neighbor_non_equilibrium currently requires a pressure port and zero acceleration");
        require(!(s.recon == LBM_RECON_NON_EQUILIBRIUM_EXTRAPOLATION && accelerated),
                "non_equilibrium_extrapolation requires zero acceleration");
        if (s.recon == LBM_RECON_REGULARIZED_KNOWN_STRESS)
            require(regularized_fit(h.L, s.axis, s.sign, s.sop),
                    "Regularized port stress fit is rank deficient or ill conditioned");
        if (s.recon == LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM || s.recon == LBM_RECON_NON_EQUILIBRIUM_EXTRAPOLATION) {
            require(shape[s.axis] >= 2, "Neighbor pressure reconstruction requires an inward fluid plane");
            const int64_t stride[3] = {h.G.sx, h.G.sy, 1};
            s.nb_off = s.sign * stride[s.axis];
            for (int64_t x : cells) {
                const int64_t y = x + s.nb_off;
                require(!(p.solid_mask[y] || p.design_region[y] || p.fixed_design[y] != 1.0),
                        "Neighbor pressure reconstruction requires protected, unobstructed, fixed-design inward fluid "
                        "cells");
            }
        }
        for (int d = 0; d < 3; ++d)
            require(std::isfinite(pt.velocity_m_s[d]), "Port velocity requires three finite components");
        for (int d = 0; d < 3; ++d) s.vel[d] = pt.velocity_m_s[d] * p.step_s / p.spacing_m;
        require(!(s.pressure && pt.velocity_m_s[s.axis] != 0.0),
                "Pressure port velocity specifies tangential components only; normal component must be zero");
        // pulsatile signal (keys of implexity-physics-fsi problem/fluid.rs:256-322)
        require(std::isfinite(pt.frequency_hz) && pt.frequency_hz >= 0.0, "Port frequency_hz must be nonnegative");
        require(std::isfinite(pt.phase_rad), "Port phase_rad must be finite");
        require(std::isfinite(pt.ramp_s) && pt.ramp_s >= 0.0, "Port ramp_s must be nonnegative");
        s.freq = pt.frequency_hz;
        s.phase = pt.phase_rad;
        s.ramp = pt.ramp_s;
        s.pulsatile = s.freq != 0.0 || s.ramp != 0.0;
        for (int d = 0; d < 3; ++d) {
            require(std::isfinite(pt.amplitude_m_s[d]), "Port amplitude_m_s requires three finite components");
            s.mean_vel[d] = s.vel[d];
            s.amp_vel[d] = s.pressure ? 0.0 : pt.amplitude_m_s[d] * p.step_s / p.spacing_m;
        }
        // the largest speed the signal reaches (moving/field.rs:884)
        double un2 = 0.0;
        for (int d = 0; d < 3; ++d) un2 += std::pow(std::fabs(s.mean_vel[d]) + std::fabs(s.amp_vel[d]), 2);
        require(!(std::sqrt(un2) * std::sqrt(3.0) > p.mach_limit), "Authored port velocity exceeds Mach limit");
        s.density = 1.0;
        if (s.pressure) {
            require(std::isfinite(pt.gauge_pressure_Pa), "Finite scalar gauge pressure required");
            require(std::isfinite(pt.amplitude_Pa), "Port amplitude_Pa must be finite");
            double unit = p.spacing_m / p.step_s;
            const double to_rho = 3.0 / (p.density_kg_m3 * unit * unit);
            double rho = 1.0 + pt.gauge_pressure_Pa * to_rho;
            const double swing = std::fabs(pt.amplitude_Pa) * to_rho;
            require(rho - swing >= 0.9 && rho + swing <= 1.1, "Pressure port density must remain within 10% of reference");
            s.density = rho;
            s.mean_rho = rho;
            s.amp_rho = pt.amplitude_Pa * to_rho;
        }
        if (s.pulsatile) s = spec_at(s, 0.0);
        for (int64_t x : cells) used[x] = 1;
        specs.push_back(s);
        port_cells.push_back(cells);
    }
    h.n_ports = (int)specs.size();
    // an extrapolating port reads its neighbours' streamed populations, which
    // must not be rebuilt by a port themselves
    h.nonlinear_ports = false;
    for (size_t k = 0; k < specs.size(); ++k) h.nonlinear_ports = h.nonlinear_ports || specs[k].recon != 0;
    for (size_t k = 0; k < specs.size(); ++k)
        if (specs[k].recon == LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM || specs[k].recon == LBM_RECON_NON_EQUILIBRIUM_EXTRAPOLATION)
            for (int64_t x : port_cells[k])
                require(!used[x + specs[k].nb_off], "The inward neighbours of an extrapolating port cannot be port cells");
    h.n_inlet = h.n_outlet = 0;
    for (size_t k = 0; k < specs.size(); ++k) (specs[k].pressure ? h.n_outlet : h.n_inlet) += (int64_t)port_cells[k].size();

    // port affine maps in shifted variables (for pulsatile ports: one set per
    // state index, built on demand by ensure_port_maps)
    h.port_specs = specs;
    h.pulsatile = false;
    for (const PortSpec& sp : specs) h.pulsatile = h.pulsatile || sp.pulsatile;
    std::vector<PortMap> maps = port_maps_at(h, 0.0);

    // link masks (Streaming::new, solver.rs:84-119)
    std::vector<uint32_t> mask(n, 0);
    h.fluid_cells = 0;
    for (int64_t x = 0; x < n; ++x) {
        int64_t c[3] = {x / h.G.sx, (x / h.G.sy) % shape[1], x % shape[2]};
        uint32_t m = 0;
        if (p.solid_mask[x]) m |= MASK_SOLID;
        else ++h.fluid_cells;
        bool wraps = false;
        for (int a2 = 0; a2 < 3; ++a2)
            if (periodic[a2] && (c[a2] == 0 || c[a2] == shape[a2] - 1)) wraps = true;
        if (wraps) m |= MASK_WRAP;
        for (int q = 0; q < h.Q; ++q) {
            int64_t s[3];
            bool outside = false;
            for (int a2 = 0; a2 < 3; ++a2) {
                s[a2] = c[a2] - h.L.c[q][a2];
                if (s[a2] < 0 || s[a2] >= shape[a2]) {
                    if (!periodic[a2]) outside = true;
                    s[a2] = (s[a2] % shape[a2] + shape[a2]) % shape[a2];
                }
            }
            int64_t src = (s[0] * shape[1] + s[1]) * shape[2] + s[2];
            if (outside || p.solid_mask[src]) m |= 1u << q;
        }
        mask[x] = m;
    }
    for (size_t k = 0; k < port_cells.size(); ++k)
        for (int64_t x : port_cells[k]) mask[x] |= (uint32_t)(k + 1) << MASK_PORT_SHIFT;
    std::vector<uint32_t> nee_cells;
    h.nee_groups.clear();
    for (size_t k = 0; k < port_cells.size(); ++k) {
        if (specs[k].recon != LBM_RECON_NEIGHBOR_NON_EQUILIBRIUM && specs[k].recon != LBM_RECON_NON_EQUILIBRIUM_EXTRAPOLATION)
            continue;
        h.nee_groups.push_back({(int64_t)nee_cells.size(), (int64_t)port_cells[k].size(), (int64_t)k});
        for (int64_t x : port_cells[k]) nee_cells.push_back((uint32_t)x);
    }

    // wall links of the momentum-exchange loads (wall_exchange.rs:44-70): every
    // blocked pull link of a fluid cell, cells and links in order, except the
    // links of a port cell that point along its port's inward normal
    h.wall_cells.clear();
    h.wall_links.clear();
    for (int64_t x = 0; x < n; ++x) {
        const uint32_t m = mask[x];
        if (m & MASK_SOLID) continue;
        const int port = (int)((m >> MASK_PORT_SHIFT) & 7u) - 1;
        for (int q = 0; q < h.Q; ++q) {
            if (!((m >> q) & 1u)) continue;
            if (port >= 0 && h.L.c[q][specs[port].axis] == specs[port].sign) continue;
            h.wall_cells.push_back((uint32_t)x);
            h.wall_links.push_back((uint8_t)q);
        }
    }

    // design map (design.rs:109-171); box filter is the documented extension
    h.cls.assign(n, 0);
    std::vector<float> fixed(n);
    for (int64_t x = 0; x < n; ++x) {
        h.cls[x] = p.solid_mask[x] ? 0 : (p.design_region[x] ? 1 : 2);
        fixed[x] = (float)p.fixed_design[x];
    }
    h.offsets.clear();
    if (p.filter_kind == LBM_FILTER_BOX) {
        int hw = p.box_half_width;
        if (hw > 0)
            for (int i = -hw; i <= hw; ++i)
                for (int j = -hw; j <= hw; ++j)
                    for (int k = -hw; k <= hw; ++k) {
                        float w = 1.f;
                        int wb;
                        std::memcpy(&wb, &w, 4);
                        h.offsets.push_back(make_int4(i, j, k, wb));
                    }
    } else {
        double radius = p.filter_radius_m / p.spacing_m;
        if (radius > 0) {
            int reach = (int)std::ceil(radius);
            for (int i = -reach; i <= reach; ++i)
                for (int j = -reach; j <= reach; ++j)
                    for (int k = -reach; k <= reach; ++k) {
                        double wgt = std::max(radius - std::sqrt((double)(i * i + j * j + k * k)), 0.0);
                        if (wgt == 0.0) continue;
                        float w = (float)wgt;
                        int wb;
                        std::memcpy(&wb, &w, 4);
                        h.offsets.push_back(make_int4(i, j, k, wb));
                    }
        }
    }
    h.beta = (float)p.projection_beta;
    h.eta = (float)p.projection_eta;
    if (p.projection_beta > 0) {
        double pa = std::tanh(p.projection_beta * p.projection_eta);
        h.proj_a = (float)pa;
        h.proj_den = (float)(pa + std::tanh(p.projection_beta * (1.0 - p.projection_eta)));
    }

    // --- device
    CK(cudaGetDevice(&h.device));
    CK(cudaDeviceGetAttribute(&h.sms, cudaDevAttrMultiProcessorCount, h.device));
    CK(cudaStreamCreateWithFlags(&h.stream, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h.ev0));
    CK(cudaEventCreate(&h.ev1));
    int64_t* ctr = &h.device_bytes;
    h.pop.alloc(2 * h.array_bytes(h.storage), ctr);
    h.mask.alloc((size_t)(n + CELL_PAD) * 4, ctr);
    h.alpha.alloc((size_t)(n + CELL_PAD) * 4, ctr);
    h.errflag.alloc(sizeof(int), ctr);
    h.phi.alloc((size_t)n * 4, ctr);
    h.raw.alloc((size_t)n * 4, ctr);
    h.den.alloc((size_t)n * 4, ctr);
    h.slope.alloc((size_t)n * 4, ctr);
    h.cls_d.alloc((size_t)n, ctr);
    h.fixed_d.alloc((size_t)n * 4, ctr);
    h.offsets_d.alloc(std::max<size_t>(1, h.offsets.size()) * sizeof(int4), ctr);
    h.ports_d.alloc(std::max<size_t>(1, maps.size()) * sizeof(PortMap), ctr);
    h.partial.alloc((size_t)h.sms * 32 * 16 * sizeof(double), ctr);
    h.counter.alloc(2 * sizeof(unsigned), ctr);  // [0] step/objective sums, [1] fused response sums
    h.sums.alloc(64 * sizeof(double), ctr);
    CK(cudaMemsetAsync(h.mask.p, 0xff, (size_t)(n + CELL_PAD) * 4, h.stream));  // padding reads as solid
    CK(cudaMemcpyAsync(h.mask.p, mask.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h.stream));
    CK(cudaMemsetAsync(h.alpha.p, 0, (size_t)(n + CELL_PAD) * 4, h.stream));
    CK(cudaMemcpyAsync(h.cls_d.p, h.cls.data(), (size_t)n, cudaMemcpyHostToDevice, h.stream));
    CK(cudaMemcpyAsync(h.fixed_d.p, fixed.data(), (size_t)n * 4, cudaMemcpyHostToDevice, h.stream));
    if (!h.offsets.empty())
        CK(cudaMemcpyAsync(h.offsets_d.p, h.offsets.data(), h.offsets.size() * sizeof(int4), cudaMemcpyHostToDevice,
                           h.stream));
    if (!nee_cells.empty()) {
        h.nee_cells_d.alloc(nee_cells.size() * sizeof(uint32_t), ctr);
        CK(cudaMemcpyAsync(h.nee_cells_d.p, nee_cells.data(), nee_cells.size() * sizeof(uint32_t),
                           cudaMemcpyHostToDevice, h.stream));
    }
    if (!maps.empty())
        CK(cudaMemcpyAsync(h.ports_d.p, maps.data(), maps.size() * sizeof(PortMap), cudaMemcpyHostToDevice,
                           h.stream));
    CK(cudaMemsetAsync(h.counter.p, 0, 2 * sizeof(unsigned), h.stream));
    CK(cudaMemsetAsync(h.errflag.p, 0, sizeof(int), h.stream));
    CK(cudaMemsetAsync(h.pop.p, 0, h.pop.bytes, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    h.time_average = p.time_average != 0;
    if (h.pulsatile) ensure_port_maps(h, h.step_count);
}

// ------------------------------------------------------------ stepping
int grid_for(const lbm_handle& h) {
    int64_t b = (h.n() + 255) / 256;
    int64_t cap = (int64_t)h.sms * 8;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

Reduce reduce_of(lbm_handle& h) { return Reduce{h.partial.as<double>(), h.counter.as<unsigned>()}; }

FwdArgs fwd_args(lbm_handle& h) {
    FwdArgs a{};
    a.G = h.G;
    a.P = h.P;
    a.src = h.popA();
    a.dst = h.popB();
    a.bulk_store = h.G.n % (int64_t)(16 / storage_bytes(h.storage)) == 0 ? 1 : 0;
    a.mask = h.mask.as<uint32_t>();
    a.alpha = h.alpha.as<float>();
    a.ports = ports_at(h, h.t);
    a.red = reduce_of(h);
    a.err = h.errflag.as<int>();
    // the fused response sums reduce through the upper half of the scratch
    a.red2 = Reduce{h.partial.as<double>() + (size_t)h.sms * 32 * 8, h.counter.as<unsigned>() + 1};
    a.phi = h.phi.as<float>();
    a.sp.vel = (float)(h.dx / h.dt);
    a.sp.dens = (float)h.density;
    a.sp.dt_s = (float)h.dt;
    a.sp.tau = (float)h.tau;
    a.dp_collision = h.collision_fp64 ? 1 : 0;
    a.omega_cell = h.tau_per_cell ? h.omega_cell.as<float>() : nullptr;
    return a;
}

// The stepping kernels' collision: MRT whose only correction is the bulk
// moment runs the compile-time folded branch.
int coll_kernel(const lbm_handle& h) {
    if (h.coll != LBM_MRT) return CK_PAIRS;
    return (h.P.n_proj == 1 && h.bulk_only) ? CK_MRT_BULK : CK_MRT;
}

// One step of the current state; diag / record / the current state's
// response sums (16 doubles) optional.
void step(lbm_handle& h, StepDiag* diag, float* record, bool record_s = false, double* stage = nullptr) {
    FwdArgs a = fwd_args(h);
    a.stage = stage;
    a.apply_ports = h.pending ? 1 : 0;
    a.diag = diag;
    a.record = record;
    a.record_s = record_s ? 1 : 0;
    a.collide = 1;
    a.step = (uint32_t)h.t;
    CK(launch_forward(h.Q, coll_kernel(h), h.storage, a, grid_for(h), h.stream));
    h.cur ^= 1;
    h.restored = nullptr;
    h.pending = h.n_ports > 0;
    ++h.t;
}

// Load-only pass of the current state (admission reductions and/or record).
void inspect(lbm_handle& h, StepDiag* diag, float* record, bool record_s = false, double* stage = nullptr) {
    FwdArgs a = fwd_args(h);
    a.stage = stage;
    a.dst = nullptr;
    a.apply_ports = h.pending ? 1 : 0;
    a.diag = diag;
    a.record = record;
    a.record_s = record_s ? 1 : 0;
    a.collide = 0;
    CK(launch_forward(h.Q, coll_kernel(h), h.storage, a, grid_for(h), h.stream));
}

void init_state(lbm_handle& h) {
    // both arrays: solid cells keep their populations in either
    const int64_t c0 = h.slab ? (int64_t)h.slab_hl * h.G.sx : 0;
    const int64_t c1 = h.slab ? (int64_t)(h.slab_hl + h.slab_own) * h.G.sx : h.n();
    CK(launch_init(h.Q, h.storage, h.G, h.P, h.popA(), h.mask.as<uint32_t>(), c0, c1, h.stream));
    CK(launch_init(h.Q, h.storage, h.G, h.P, h.popB(), h.mask.as<uint32_t>(), c0, c1, h.stream));
    h.pending = false;
    h.t = 0;
    h.state_valid = true;
    h.solid_nonfinite = false;
}

void require_design(const lbm_handle& h) {
    if (!h.design_set) throw StateError("lbm_set_design must be called before stepping");
}

// Relative mass-drift bound of the admission.  FP32 storage keeps the
// reference's 1e-6 (solver.rs:766).  The 16-bit formats resolve a population
// to about 2^-11 (FP16) or 2^-8 (BF16) of (f - w)/w, so the mass of a small
// grid random-walks past 1e-6 within a few thousand steps however unbiased the
// rounding; they are admitted against the storage resolution instead.
double mass_drift_limit(int storage) {
    return storage == LBM_STORE_F32 ? 1e-6 : (storage == LBM_STORE_F16 ? 1e-4 : 1e-3);
}

// Admission from the per-state records (solver.rs:708-793).
lbm_status admit(lbm_handle& h, const std::vector<StepDiag>& d, lbm_diag_t* out, double ms) {
    const size_t T = d.size();
    // finiteness covers every cell (solid ones through the load-time check),
    // the minimum only fluid cells (solver.rs:714-726)
    bool nonfinite = h.solid_nonfinite;
    double minimum = INFINITY, maxu2 = 0;
    for (auto& s : d) {
        nonfinite = nonfinite || s.nonfinite;
        minimum = std::min(minimum, (double)s.min_f);
        maxu2 = std::max(maxu2, (double)s.max_u2);
    }
    const double mach = std::sqrt(maxu2) * std::sqrt(3.0);
    const bool use_changes = h.n_ports > 0;
    double cum = 0, err = 0, total = 0;
    bool changes_finite = true;
    const double m0 = (double)h.fluid_cells + d[0].mass_hi + d[0].mass_lo;
    for (size_t t = 0; t < T; ++t) {
        double mt = (double)h.fluid_cells + d[t].mass_hi + d[t].mass_lo;
        if (t > 0 && use_changes) {
            double e = d[t].exch_hi + d[t].exch_lo;
            changes_finite = changes_finite && std::isfinite(e);
            cum += e;
            total += e;
        }
        err = std::max(err, std::fabs(mt - (m0 + cum)));
    }
    err /= m0;
    if (out) {
        out->maximum_mach = mach;
        out->relative_mass_drift = err;
        out->relaxation_time = h.tau;
        out->minimum_population = minimum;
        out->boundary_exchange_total = use_changes ? total : 0.0;
        out->steps = (int64_t)T - 1;
        out->nonfinite = nonfinite ? 1 : 0;
        out->admitted = 0;
        out->device_ms = ms;
    }
    if (nonfinite || !(minimum > 0)) throw ContractError("LBM trajectory has nonpositive or nonfinite populations");
    if (!changes_finite) throw ContractError("Invalid boundary mass exchange history");
    if (mach > h.mach_limit || err > mass_drift_limit(h.storage))
        throw ContractError("LBM trajectory rejected: Mach=" + repr_float(mach) + ", mass drift=" + repr_float(err));
    if (out) out->admitted = 1;
    return LBM_OK;
}

// Device-side bounded waits report through errflag; the step that set it
// computed nothing for the affected tile.
void check_errflag(lbm_handle& h) {
    int e = 0;
    CK(cudaMemcpyAsync(&e, h.errflag.p, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    if (e) {
        CK(cudaMemsetAsync(h.errflag.p, 0, sizeof(int), h.stream));
        throw CudaError("a staged bulk copy did not complete within its bounded wait");
    }
}

// Runs `steps` steps from the current state with admission of every state
// including the current one.  Optionally stores checkpoints every K steps.
void finish_time_average(lbm_handle& h, int64_t steps);

// With `averages`, the responses of every state 1..steps are summed on the
// device as well (the stage objective's value, lbm_time_average): the step
// that reads state t sums its responses into slot t, the final inspection
// those of the last state.
lbm_status run_admitted(lbm_handle& h, int64_t steps, lbm_diag_t* out, int64_t K, bool averages = false) {
    require_design(h);
    int64_t* ctr = &h.device_bytes;
    h.diag.alloc((size_t)(steps + 1) * sizeof(StepDiag), ctr);
    StepDiag* d = h.diag.as<StepDiag>();
    ensure_port_maps(h, h.t + steps);
    h.tavg_valid = false;
    if (averages) h.tsums.alloc((size_t)(steps + 1) * 16 * sizeof(double), ctr);
    CK(cudaEventRecord(h.ev0, h.stream));
    for (int64_t s = 0; s < steps; ++s) {
        if (K > 0 && s % K == 0) {
            // checkpoint of the state entering step s (scan.rs:181-196)
            Checkpoint c;
            c.buf = std::make_unique<DevBuf>();
            const size_t ab = h.array_bytes(h.storage);
            c.buf->alloc(ab, ctr);
            CK(cudaMemcpyAsync(c.buf->p, h.pop_array(h.cur), ab, cudaMemcpyDeviceToDevice, h.stream));
            c.t = h.t;
            c.pending = h.pending;
            h.ckpts.push_back(std::move(c));
        }
        double* slot = averages && s > 0 ? h.tsums.as<double>() + (size_t)s * 16 : nullptr;
        step(h, d + s, nullptr, false, slot);
    }
    inspect(h, d + steps, nullptr, false, averages ? h.tsums.as<double>() + (size_t)steps * 16 : nullptr);
    CK(cudaEventRecord(h.ev1, h.stream));
    std::vector<StepDiag>& hd = h.last_trajectory;
    hd.resize((size_t)steps + 1);
    CK(cudaMemcpyAsync(hd.data(), d, hd.size() * sizeof(StepDiag), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h.ev0, h.ev1));
    check_errflag(h);
    if (averages) finish_time_average(h, steps);
    return admit(h, hd, out, ms);
}

void ensure_scratch(lbm_handle& h) { h.scratch.alloc((size_t)h.n() * h.Q * sizeof(float), &h.device_bytes); }

ObjArgs obj_args(lbm_handle& h) {
    ObjArgs a{};
    a.G = h.G;
    a.P = h.P;
    a.pop = h.popA();
    a.mask = h.mask.as<uint32_t>();
    a.alpha = h.alpha.as<float>();
    a.phi = h.phi.as<float>();
    a.ports = ports_at(h, h.t);
    a.apply_ports = h.pending ? 1 : 0;
    a.tau = (float)h.tau;
    a.vel = (float)(h.dx / h.dt);
    a.dens = (float)h.density;
    a.dt_s = (float)h.dt;
    a.red = reduce_of(h);
    const int64_t sxo = h.G.sx;
    a.c_begin = h.slab ? (uint32_t)(h.slab_hl * sxo) : 0u;
    a.c_end = h.slab ? (uint32_t)((h.slab_hl + h.slab_own) * sxo) : (uint32_t)h.n();
    return a;
}

double visc_scale(const lbm_handle& h) { return h.density * std::pow(h.dx, 5) / std::pow(h.dt, 3); }

// The 8 responses from the 8 compensated sums of the objective kernel.
void sums_to_responses(const lbm_handle& h, const double* s, double* out8) {
    double v[8];
    for (int k = 0; k < 8; ++k) v[k] = s[2 * k] + s[2 * k + 1];
    const double nf = (double)resp_fluid(h), dv = h.dx * h.dx * h.dx;
    out8[0] = v[0] / nf;
    out8[1] = v[1] / nf;
    out8[2] = v[2] / nf;
    out8[3] = 0.5 * v[3] * dv;
    out8[4] = v[4] * dv;
    out8[5] = v[5] * dv;
    out8[6] = resp_both_ports(h) ? v[6] : 0.0;
    out8[7] = v[7] * visc_scale(h);
}

void responses(lbm_handle& h, double* out8, float* fields) {
    ObjArgs a = obj_args(h);
    a.sums = h.sums.as<double>();
    a.fields = fields;
    CK(launch_objective(h.Q, h.storage, LBM_STORE_F32, 0, a, grid_for(h), h.stream));
    double s[16];
    CK(cudaMemcpyAsync(s, h.sums.p, sizeof(s), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    sums_to_responses(h, s, out8);
}

// Mean of the responses of states 1..steps (slots filled by the steps).
void finish_time_average(lbm_handle& h, int64_t steps) {
    std::vector<double> all((size_t)(steps + 1) * 16);
    CK(cudaMemcpy(all.data(), h.tsums.p, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0}, r[8];
    for (int64_t t = 1; t <= steps; ++t) {
        sums_to_responses(h, all.data() + (size_t)t * 16, r);
        for (int k = 0; k < 8; ++k) acc[k] += r[k];
    }
    for (int k = 0; k < 8; ++k) h.tavg[k] = steps > 0 ? acc[k] / (double)steps : 0.0;
    h.tavg_valid = steps > 0;
}

DesignArgs design_args(lbm_handle& h) {
    DesignArgs a{};
    a.G = h.G;
    a.raw = h.raw.as<float>();
    a.cls = h.cls_d.as<uint8_t>();
    a.fixed = h.fixed_d.as<float>();
    a.offsets = h.offsets_d.as<int4>();
    a.n_offsets = (int)h.offsets.size();
    a.beta = h.beta;
    a.eta = h.eta;
    a.proj_a = h.proj_a;
    a.proj_den = h.proj_den;
    a.ramp_c = (float)(h.dt * h.drag_max * h.drag_shape);
    a.ramp_q = (float)h.drag_shape;
    a.phi = h.phi.as<float>();
    a.alpha = h.alpha.as<float>();
    a.den = h.den.as<float>();
    a.slope = h.slope.as<float>();
    return a;
}

// phi_bar -> raw gradient on the device (grad buffer), scaled abar optional.
void design_transpose(lbm_handle& h, const float* phibar, const float* abar, float abar_scale,
                      const float* abar_final) {
    int64_t* ctr = &h.device_bytes;
    h.scale.alloc((size_t)h.n() * 4, ctr);
    h.grad.alloc((size_t)h.n() * 4, ctr);
    DesignArgs a = design_args(h);
    a.phibar = phibar;
    a.abar = abar;
    a.abar_scale = abar_scale;
    a.abar_final = abar_final;
    a.scale = h.scale.as<float>();
    a.grad = h.grad.as<float>();
    const int grid = (int)std::min<int64_t>((h.n() + 255) / 256, (int64_t)h.sms * 8);
    CK(launch_sens_scale(a, grid, h.stream));
    CK(launch_filter_transpose(a, grid, h.stream));
}

// ------------------------------------------------------------ adjoint
struct AdjState {
    float scale = 1.f;      // stored = true * scale for the lambda now in memory
    float target = 1.f;     // scale the next adjoint step writes with
    float s0 = 1.f;         // abar is accumulated in units of 1/s0
    bool first = true;
    int64_t steps = 0;
};

// Second half of the extrapolating ports' transposes on the cotangent array
// `lam` (launch_nee_move), one port after another.
void nee_move(lbm_handle& h, void* lam, int lam_storage) {
    for (const auto& g : h.nee_groups)
        CK(launch_nee_move(lam_storage, lam, h.n(), h.Q, h.nee_cells_d.as<uint32_t>() + g[0], g[1],
                           h.port_specs[(size_t)g[2]].nb_off, h.stream));
}

AdjArgs adj_args(lbm_handle& h) {
    AdjArgs a{};
    a.G = h.G;
    a.P = h.P;
    a.src = h.lamA();
    a.dst = h.lamB();
    a.mask = h.mask.as<uint32_t>();
    a.alpha = h.alpha.as<float>();
    a.ports = ports_at(h, h.t);
    a.rec_planes = 4;
    a.abar = h.abar.as<float>();
    a.red = reduce_of(h);
    a.err = h.errflag.as<int>();
    a.omega_cell = h.tau_per_cell ? h.omega_cell.as<float>() : nullptr;
    return a;
}

// One transposed step linearised at record slot `rec`; returns nothing, the
// norm (if requested) lands in norm2[0..1].
void adjoint_step(lbm_handle& h, AdjState& st, const float* rec, bool want_norm, int64_t t_state = -1,
                  const SeedParams* stage = nullptr, int rec_planes = 4) {
    AdjArgs a = adj_args(h);
    a.record = rec;
    a.rec_planes = rec_planes;
    a.ports = ports_at(h, t_state >= 0 ? t_state : h.t);
    a.stage = stage ? 1 : 0;
    if (stage) a.seed = *stage;
    a.port_transpose = 1;
    a.overwrite_abar = st.first ? 1 : 0;
    a.in_scale_inv = 1.f / st.scale;
    a.out_scale = st.target;
    a.abar_factor = st.s0;
    a.norm2 = want_norm ? h.norm2.as<double>() : nullptr;
    CK(launch_adjoint(h.Q, coll_kernel(h), h.lam_storage, a, grid_for(h), h.stream));
    h.lcur ^= 1;
    nee_move(h, h.lamA(), h.lam_storage);
    st.scale = st.target;
    st.first = false;
    ++st.steps;
}

double read_norm(lbm_handle& h) {
    double s[2];
    CK(cudaMemcpyAsync(s, h.norm2.p, sizeof(s), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    return std::sqrt(std::max(0.0, s[0] + s[1]));
}

// Objective VJP at the current state: lambda seed, abar_final, phibar and
// the (rho, u) record.  Returns |mu_0| (true units).
// The weights of vector_vjp after the reference's response scalings
// (solver.rs:896-947); every weight but the fluid volume's is multiplied by
// `scale` (1/T for a state of a time average: the fluid volume does not
// change in time, so its mean is itself).
void response_weights(const lbm_handle& h, const double* w, double scale, double* out8) {
    const double nf = (double)resp_fluid(h), dv = h.dx * h.dx * h.dx;
    out8[0] = scale * w[0] / nf;
    out8[1] = scale * w[1] / nf;
    out8[2] = scale * w[2] / nf;
    out8[3] = scale * 0.5 * w[3] * dv;
    out8[4] = scale * w[4] * dv;
    out8[5] = w[5] * dv;
    out8[6] = resp_both_ports(h) ? scale * w[6] : 0.0;
    out8[7] = scale * w[7] * visc_scale(h);
}

// Stage seed parameters of the adjoint kernel (the response VJP of one state).
SeedParams stage_seed(const lbm_handle& h, const double* w, double scale) {
    double ws[8];
    response_weights(h, w, scale, ws);
    SeedParams sp{};
    for (int k = 0; k < 8; ++k) sp.w[k] = (float)ws[k];
    sp.w[5] = 0.f;  // phi enters through phibar, seeded once
    sp.vel = (float)(h.dx / h.dt);
    sp.dens = (float)h.density;
    sp.dt_s = (float)h.dt;
    sp.tau = (float)h.tau;
    return sp;
}

double seed(lbm_handle& h, const double* w, AdjState& st, float* record, double stage_scale = 1.0) {
    int64_t* ctr = &h.device_bytes;
    const int64_t n = h.n();
    h.abar_final.alloc((size_t)n * 4, ctr);
    h.phibar.alloc((size_t)n * 4, ctr);
    h.norm2.alloc(2 * sizeof(double), ctr);
    ObjArgs a = obj_args(h);
    response_weights(h, w, stage_scale, a.w);
    a.lam = h.lamA();
    a.abar_final = h.abar_final.as<float>();
    a.phibar = h.phibar.as<float>();
    a.record = record;
    a.port_transpose = 1;
    a.norm2 = h.norm2.as<double>();
    a.write_lambda = 0;
    a.lam_scale = 1.f;
    CK(launch_objective(h.Q, h.storage, h.lam_storage, 1, a, grid_for(h), h.stream));
    const double n0 = read_norm(h);
    const double entries = (double)h.fluid_cells * h.Q;
    st.s0 = n0 > 0 ? (float)(std::sqrt(entries) / n0) : 1.f;
    if (!std::isfinite(st.s0) || st.s0 == 0.f) st.s0 = 1.f;
    st.scale = st.s0;
    st.target = st.s0;
    a.write_lambda = 1;
    a.lam_scale = st.s0;
    a.norm2 = nullptr;
    a.record = nullptr;
    CK(launch_objective(h.Q, h.storage, h.lam_storage, 1, a, grid_for(h), h.stream));
    nee_move(h, h.lamA(), h.lam_storage);
    st.first = true;
    return n0;
}

void alloc_adjoint(lbm_handle& h, int lam_storage) {
    int64_t* ctr = &h.device_bytes;
    const int64_t n = h.n();
    if (h.lam.p && h.lam_storage != lam_storage) h.lam.reset();
    h.lam_storage = lam_storage;
    h.lam.alloc(2 * h.array_bytes(lam_storage), ctr);
    h.abar.alloc((size_t)n * 4, ctr);
    h.norm2.alloc(2 * sizeof(double), ctr);
}

float next_scale(const lbm_handle& h, double true_norm, float cur) {
    if (!(true_norm > 0) || !std::isfinite(true_norm)) return cur;
    double s = std::sqrt((double)h.fluid_cells * h.Q) / true_norm;
    if (!std::isfinite(s) || s <= 0 || s > 3e38) return cur;
    return (float)s;
}

void finish_gradient(lbm_handle& h, const AdjState& st, bool any_adjoint, double* grad) {
    design_transpose(h, h.phibar.as<float>(), any_adjoint ? h.abar.as<float>() : nullptr, 1.f / st.s0,
                     h.abar_final.as<float>());
    std::vector<float> g((size_t)h.n());
    CK(cudaMemcpyAsync(g.data(), h.grad.p, g.size() * 4, cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    bool finite = true;
    for (int64_t x = 0; x < h.n(); ++x) {
        grad[x] = g[x];
        finite = finite && std::isfinite(g[x]);
    }
    if (!finite) throw ContractError("Nonfinite LBM sensitivity");
}

lbm_status gradient_steady(lbm_handle& h, const double* w, const lbm_adjoint_opts_t& o, double* grad,
                           lbm_adjoint_report_t* rep) {
    if (!h.forward_done) throw StateError("lbm_forward must succeed before lbm_gradient");
    alloc_adjoint(h, o.lambda_storage);
    int64_t* ctr = &h.device_bytes;
    h.record.alloc(((size_t)h.n() * 4 + CELL_PAD) * sizeof(float), ctr);
    AdjState st;
    CK(cudaEventRecord(h.ev0, h.stream));
    const double n0 = seed(h, w, st, h.record.as<float>());
    double resid = 0;
    bool converged = (n0 == 0);
    const int64_t check = o.check_every > 0 ? o.check_every : 50;
    const int64_t cap = o.max_iterations > 0 ? o.max_iterations : 100000;
    float ms_adj = 0;
    if (!converged) {
        cudaEvent_t e2, e3;
        CK(cudaEventCreate(&e2));
        CK(cudaEventCreate(&e3));
        CK(cudaEventRecord(e2, h.stream));
        while (st.steps < cap) {
            const int64_t chunk = std::min(check, cap - st.steps);
            for (int64_t i = 0; i < chunk; ++i) adjoint_step(h, st, h.record.as<float>(), i == chunk - 1);
            const double nrm = read_norm(h) / st.scale;
            resid = nrm / n0;
            if (resid <= o.tolerance) {
                converged = true;
                break;
            }
            // keep the stored adjoint near unit RMS (the 16-bit formats need
            // it; the next step reads with the old scale, writes with the new)
            st.target = next_scale(h, nrm, st.scale);
        }
        CK(cudaEventRecord(e3, h.stream));
        CK(cudaEventSynchronize(e3));
        CK(cudaEventElapsedTime(&ms_adj, e2, e3));
        cudaEventDestroy(e2);
        cudaEventDestroy(e3);
    }
    check_errflag(h);
    cudaEvent_t e4;
    CK(cudaEventCreate(&e4));
    CK(cudaEventRecord(e4, h.stream));
    finish_gradient(h, st, st.steps > 0, grad);
    float ms_sens = 0;
    CK(cudaEventRecord(h.ev1, h.stream));
    CK(cudaEventSynchronize(h.ev1));
    CK(cudaEventElapsedTime(&ms_sens, e4, h.ev1));
    cudaEventDestroy(e4);
    if (rep) {
        rep->residual = resid;
        rep->iterations = st.steps;
        rep->forward_recomputed = 0;
        rep->peak_state_bytes = (int64_t)(h.record.bytes + h.lam.bytes);
        rep->converged = converged ? 1 : 0;
        rep->forward_ms = 0;
        rep->adjoint_ms = ms_adj;
        rep->sensitivity_ms = ms_sens;
    }
    if (!converged)
        throw ConvergenceError("steady adjoint did not reach the residual tolerance within max_iterations (residual=" +
                               repr_float(resid) + ")");
    return LBM_OK;
}

lbm_status gradient_horizon(lbm_handle& h, const double* w, const lbm_adjoint_opts_t& o, double* grad,
                            lbm_adjoint_report_t* rep) {
    require_design(h);
    const int64_t T = h.step_count;
    int64_t K = o.checkpoint_every;
    if (K <= 0) {
        K = 1;
        while (K * K < T) ++K;
    }
    K = std::min(K, T);
    // the stage objective (time average over states 1..T) seeds every state;
    // its records carry the second moments as well
    const bool stage = o.objective == LBM_OBJ_TIME_AVERAGE;
    const int rec_planes = stage ? 10 : 4;
    alloc_adjoint(h, o.lambda_storage);
    int64_t* ctr = &h.device_bytes;
    const size_t rec_bytes = (size_t)h.n() * rec_planes * sizeof(float);
    // Records for KR steps.  When a segment's K records do not fit (the
    // caller's record budget, or ~80% of the device memory left after the
    // T/K checkpoints), a second checkpoint level splits each segment into
    // spans of KR steps: the segment is recomputed once storing a state every
    // KR steps, then each span once more with its records (scan.rs Every(K)
    // nested in itself; one more recomputed forward).
    int64_t KR = K;
    h.record.reset();  // sized below from the memory left
    {
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        const size_t ab = h.array_bytes(h.storage);
        const double ckpt_bytes = (double)((T + K - 1) / K + 2) * (double)ab;
        double budget = 0.8 * ((double)free_b - ckpt_bytes) - (double)(1ull << 30);
        if (o.record_budget_bytes > 0) budget = std::min(budget, (double)o.record_budget_bytes);
        const int64_t fit = budget > 0 ? (int64_t)(budget / (double)rec_bytes) : 0;
        if (fit < 1) throw ContractError("checkpoint interval needs more record memory than record_budget_bytes");
        // the fewest spans, of equal length: the same recomputation as the
        // longest spans that fit, with less record memory
        const int64_t spans = (K + fit - 1) / fit;
        KR = (K + spans - 1) / spans;
    }
    h.record.fit(rec_bytes * (size_t)KR + CELL_PAD * sizeof(float), ctr);
    h.ckpts.clear();
    // forward with checkpoints, then admission (the reference re-runs parts())
    init_state(h);
    cudaEvent_t ef0, ef1;
    CK(cudaEventCreate(&ef0));
    CK(cudaEventCreate(&ef1));
    lbm_diag_t dg{};
    run_admitted(h, T, &dg, K);
    h.forward_done = true;
    AdjState st;
    const double n0 = seed(h, w, st, nullptr, stage ? 1.0 / (double)T : 1.0);
    const SeedParams sp = stage_seed(h, w, 1.0 / (double)T);
    float* rec = h.record.as<float>();
    const size_t rec_stride = (size_t)h.n() * rec_planes;
    int64_t recomputed = 0;
    float ms_fwd = 0, ms_adj = 0;
    if (n0 > 0 || stage) {
        cudaEvent_t ea0, ea1;
        CK(cudaEventCreate(&ea0));
        CK(cudaEventCreate(&ea1));
        int64_t peak_sub = 0;
        // records of states [s0, e0), then their transposed steps in reverse
        auto reverse_span = [&](int64_t s0, int64_t e0, int64_t seg_start) {
            CK(cudaEventRecord(ef0, h.stream));
            for (int64_t t = s0; t < e0; ++t) {
                float* r = rec + (size_t)(t - s0) * rec_stride;
                if (t + 1 < e0) {
                    step(h, nullptr, r, stage);
                    ++recomputed;
                } else {
                    inspect(h, nullptr, r, stage);
                }
            }
            CK(cudaEventRecord(ef1, h.stream));
            CK(cudaEventRecord(ea0, h.stream));
            for (int64_t t = e0 - 1; t >= s0; --t)
                adjoint_step(h, st, rec + (size_t)(t - s0) * rec_stride, t == seg_start, t,
                             stage && t >= 1 ? &sp : nullptr, rec_planes);
            CK(cudaEventRecord(ea1, h.stream));
            CK(cudaEventSynchronize(ea1));
            float a1 = 0, a2 = 0;
            CK(cudaEventElapsedTime(&a1, ef0, ef1));
            CK(cudaEventElapsedTime(&a2, ea0, ea1));
            ms_fwd += a1;
            ms_adj += a2;
        };
        auto restore = [&](const Checkpoint& c) {
            CK(cudaMemcpyAsync(h.pop_array(h.cur), c.buf->p, c.buf->bytes, cudaMemcpyDeviceToDevice, h.stream));
            h.pending = c.pending;
            h.t = c.t;
        };
        for (int64_t ci = (int64_t)h.ckpts.size() - 1; ci >= 0; --ci) {
            Checkpoint& c = h.ckpts[ci];
            const int64_t start = c.t, end = std::min(start + K, T);
            restore(c);
            if (end - start <= KR) {
                reverse_span(start, end, start);
            } else {
                // second level: a state every KR steps of the segment
                std::vector<Checkpoint> sub;
                cudaEvent_t es0, es1;
                CK(cudaEventCreate(&es0));
                CK(cudaEventCreate(&es1));
                CK(cudaEventRecord(es0, h.stream));
                const int64_t last = start + ((end - 1 - start) / KR) * KR;  // the last span's first state
                for (int64_t t = start; t <= last; ++t) {
                    if ((t - start) % KR == 0) {
                        Checkpoint sc;
                        sc.buf = std::make_unique<DevBuf>();
                        const size_t ab = h.array_bytes(h.storage);
                        sc.buf->alloc(ab, ctr);
                        CK(cudaMemcpyAsync(sc.buf->p, h.pop_array(h.cur), ab, cudaMemcpyDeviceToDevice, h.stream));
                        sc.t = h.t;
                        sc.pending = h.pending;
                        sub.push_back(std::move(sc));
                    }
                    if (t < last) {
                        step(h, nullptr, nullptr);
                        ++recomputed;
                    }
                }
                CK(cudaEventRecord(es1, h.stream));
                CK(cudaEventSynchronize(es1));
                float a0 = 0;
                CK(cudaEventElapsedTime(&a0, es0, es1));
                ms_fwd += a0;
                cudaEventDestroy(es0);
                cudaEventDestroy(es1);
                int64_t held = 0;
                for (auto& sc : sub) held += (int64_t)sc.buf->bytes;
                peak_sub = std::max(peak_sub, held);
                for (int64_t si = (int64_t)sub.size() - 1; si >= 0; --si) {
                    restore(sub[si]);
                    reverse_span(sub[si].t, std::min(sub[si].t + KR, end), start);
                }
            }
            // rescale the stored adjoint at segment boundaries
            st.target = next_scale(h, read_norm(h) / st.scale, st.scale);
        }
        h.peak_extra = peak_sub;
        cudaEventDestroy(ea0);
        cudaEventDestroy(ea1);
    }
    cudaEventDestroy(ef0);
    cudaEventDestroy(ef1);
    int64_t peak = (int64_t)h.record.bytes + h.peak_extra;
    for (auto& c : h.ckpts) peak += (int64_t)c.buf->bytes;
    h.peak_extra = 0;
    h.ckpts.clear();
    // the current state is the one of checkpoint 0's segment end; re-mark
    h.forward_done = false;
    h.state_valid = false;
    check_errflag(h);
    cudaEvent_t e4;
    CK(cudaEventCreate(&e4));
    CK(cudaEventRecord(e4, h.stream));
    finish_gradient(h, st, st.steps > 0, grad);
    float ms_sens = 0;
    CK(cudaEventRecord(h.ev1, h.stream));
    CK(cudaEventSynchronize(h.ev1));
    CK(cudaEventElapsedTime(&ms_sens, e4, h.ev1));
    cudaEventDestroy(e4);
    if (rep) {
        rep->residual = 0;
        rep->iterations = st.steps;
        rep->forward_recomputed = recomputed;
        rep->peak_state_bytes = peak;
        rep->converged = 1;
        rep->forward_ms = ms_fwd;
        rep->adjoint_ms = ms_adj;
        rep->sensitivity_ms = ms_sens;
    }
    return LBM_OK;
}

// Horizon adjoint with binomial checkpointing (scan.rs binomial_scan,
// :285-390): the actions of revolve_plan drive the device state.  The forward
// sweep is the admitted forward (every state's admission record, as
// run_admitted); after its last step the state before it is still in the
// other population array, which is where the reverse sweep starts.  A
// reversed step k takes the record of state k-1 from a load-only pass and
// applies the transposed step linearised there (with the state's stage seed
// for the time-averaged objective).  One record slot suffices.
lbm_status gradient_binomial(lbm_handle& h, const double* w, const lbm_adjoint_opts_t& o, double* grad,
                             lbm_adjoint_report_t* rep) {
    require_design(h);
    const int64_t T = h.step_count;
    const RevolvePlan plan = revolve_plan(T, o.snapshots);
    const bool stage = o.objective == LBM_OBJ_TIME_AVERAGE;
    const int rec_planes = stage ? 10 : 4;
    alloc_adjoint(h, o.lambda_storage);
    int64_t* ctr = &h.device_bytes;
    h.record.fit((size_t)h.n() * rec_planes * sizeof(float) + CELL_PAD * sizeof(float), ctr);
    const size_t ab = h.array_bytes(h.storage);
    std::vector<Checkpoint> slots((size_t)o.snapshots);
    // a restored slot stands for the current state only while the slots live
    // (declared after them, so it is cleared first on every exit path)
    struct ClearRestored {
        lbm_handle& h;
        ~ClearRestored() { h.restored = nullptr; }
    } clear_restored{h};
    auto store = [&](int64_t slot) {
        Checkpoint& c = slots[(size_t)slot];
        if (!c.buf) {
            c.buf = std::make_unique<DevBuf>();
            c.buf->alloc(ab, ctr);
        }
        const char* cur = h.restored ? h.restored : h.pop_array(h.cur);
        CK(cudaMemcpyAsync(c.buf->p, cur, ab, cudaMemcpyDeviceToDevice, h.stream));
        c.t = h.t;
        c.pending = h.pending;
    };
    auto need = [](bool ok) {
        if (!ok) throw CudaError("binomial schedule and device state disagree");
    };
    // forward sweep with the admission record of every state
    init_state(h);
    h.diag.alloc((size_t)(T + 1) * sizeof(StepDiag), ctr);
    StepDiag* d = h.diag.as<StepDiag>();
    ensure_port_maps(h, T);
    bool prev_pending = false;
    CK(cudaEventRecord(h.ev0, h.stream));
    for (size_t i = 0; i < plan.reverse_start; ++i) {
        const RevolveAction& x = plan.actions[i];
        if (x.kind == RevolveAction::SNAPSHOT) {
            need(h.t == x.a);
            store(x.b);
        } else if (x.kind == RevolveAction::ADVANCE) {
            need(h.t == x.a);
            for (int64_t t = x.a; t < x.b; ++t) {
                prev_pending = h.pending;
                step(h, d + t, nullptr);
            }
        } else {
            need(false);
        }
    }
    need(h.t == T);
    inspect(h, d + T, nullptr);
    CK(cudaEventRecord(h.ev1, h.stream));
    std::vector<StepDiag>& hd = h.last_trajectory;
    hd.resize((size_t)T + 1);
    CK(cudaMemcpyAsync(hd.data(), d, hd.size() * sizeof(StepDiag), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    float ms_sweep = 0;
    CK(cudaEventElapsedTime(&ms_sweep, h.ev0, h.ev1));
    check_errflag(h);
    lbm_diag_t dg{};
    admit(h, hd, &dg, ms_sweep);
    h.forward_done = true;
    AdjState st;
    const double n0 = seed(h, w, st, nullptr, stage ? 1.0 / (double)T : 1.0);
    const SeedParams sp = stage_seed(h, w, 1.0 / (double)T);
    // back to state T-1, which the last step left in the other array
    h.cur ^= 1;
    h.t = T - 1;
    h.pending = prev_pending;
    int64_t rescale = 1;
    while (rescale * rescale < T) ++rescale;
    int64_t recomputed = 0, reversed = 0;
    float ms_fwd = 0, ms_adj = 0;
    if (n0 > 0 || stage) {
        // event pairs around runs of forward-type work (steps, record passes,
        // state copies) and adjoint steps, from a pool created up front (at
        // most two runs per action)
        std::vector<cudaEvent_t> evs(2 * (plan.actions.size() - plan.reverse_start) + 2);
        for (auto& e : evs) CK(cudaEventCreate(&e));
        size_t used = 0;
        std::vector<int> kinds;  // 0 forward, 1 adjoint, per pair
        int open = -1;
        auto mark = [&](int kind) {
            if (open == kind) return;
            CK(cudaEventRecord(evs[used++], h.stream));
            if (open >= 0) kinds.push_back(open);
            open = kind;
        };
        for (size_t i = plan.reverse_start; i < plan.actions.size(); ++i) {
            const RevolveAction& x = plan.actions[i];
            switch (x.kind) {
                case RevolveAction::RESTORE: {
                    // the next step or record pass reads the slot in place
                    const Checkpoint& c = slots[(size_t)x.b];
                    need(c.buf && c.t == x.a);
                    h.restored = static_cast<const char*>(c.buf->p);
                    h.t = c.t;
                    h.pending = c.pending;
                    break;
                }
                case RevolveAction::SNAPSHOT:
                    need(h.t == x.a);
                    mark(0);
                    store(x.b);
                    break;
                case RevolveAction::ADVANCE:
                    need(h.t == x.a);
                    mark(0);
                    for (int64_t t = x.a; t < x.b; ++t) step(h, nullptr, nullptr);
                    recomputed += x.b - x.a;
                    break;
                case RevolveAction::REVERSE: {
                    need(h.t == x.a - 1);
                    const int64_t t = x.a - 1;
                    mark(0);
                    inspect(h, nullptr, h.record.as<float>(), stage);
                    mark(1);
                    ++reversed;
                    const bool norm = reversed % rescale == 0;
                    adjoint_step(h, st, h.record.as<float>(), norm, t, stage && t >= 1 ? &sp : nullptr, rec_planes);
                    // keep the stored adjoint near unit RMS, as the segments of Every(K) do
                    if (norm) st.target = next_scale(h, read_norm(h) / st.scale, st.scale);
                    break;
                }
                case RevolveAction::RELEASE:
                    break;
            }
        }
        mark(-1);
        CK(cudaStreamSynchronize(h.stream));
        for (size_t k = 0; k < kinds.size(); ++k) {
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, evs[k], evs[k + 1]));
            (kinds[k] == 0 ? ms_fwd : ms_adj) += ms;
        }
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
    }
    h.restored = nullptr;
    int64_t held = 0;
    for (auto& c : slots)
        if (c.buf) held += (int64_t)c.buf->bytes;
    const int64_t peak = (int64_t)h.record.bytes + held;
    slots.clear();
    h.forward_done = false;
    h.state_valid = false;
    check_errflag(h);
    cudaEvent_t e4;
    CK(cudaEventCreate(&e4));
    CK(cudaEventRecord(e4, h.stream));
    finish_gradient(h, st, st.steps > 0, grad);
    float ms_sens = 0;
    CK(cudaEventRecord(h.ev1, h.stream));
    CK(cudaEventSynchronize(h.ev1));
    CK(cudaEventElapsedTime(&ms_sens, e4, h.ev1));
    cudaEventDestroy(e4);
    if (rep) {
        rep->residual = 0;
        rep->iterations = st.steps;
        rep->forward_recomputed = recomputed;
        rep->peak_state_bytes = peak;
        rep->converged = 1;
        rep->forward_ms = ms_fwd;
        rep->adjoint_ms = ms_adj;
        rep->sensitivity_ms = ms_sens;
    }
    return LBM_OK;
}

template <typename F>
lbm_status guarded(lbm_handle* h, F&& fn) {
    if (!h) return LBM_E_STATE;
    try {
        h->err.clear();
        return fn();
    } catch (const ContractError& e) {
        h->err = e.what();
        return LBM_E_CONTRACT;
    } catch (const ConvergenceError& e) {
        h->err = e.what();
        return LBM_E_CONVERGENCE;
    } catch (const StateError& e) {
        h->err = e.what();
        return LBM_E_STATE;
    } catch (const CudaError& e) {
        h->err = e.what();
        return LBM_E_CUDA;
    } catch (const std::bad_alloc&) {
        h->err = "host allocation failed";
        return LBM_E_CUDA;
    } catch (const std::exception& e) {
        h->err = e.what();
        return LBM_E_CUDA;
    }
}

void check_n(const lbm_handle& h, size_t n, size_t expect, const char* what) {
    if (n != expect) throw ContractError(std::string(what) + " must be a finite shape-matched array");
}

}  // namespace

namespace lbm {
void set_thread_error(const char* msg) { g_create_error = msg; }
}  // namespace lbm

// ================================================================ C ABI
extern "C" {

int32_t lbm_abi_version(void) { return LBM_ABI_VERSION; }

const char* lbm_last_error(const lbm_handle* h) { return h ? h->err.c_str() : g_create_error.c_str(); }

lbm_status lbm_create(const lbm_problem_t* problem, lbm_handle** out) {
    if (!out) return LBM_E_CONTRACT;
    *out = nullptr;
    if (!problem) {
        g_create_error = "problem must not be NULL";
        return LBM_E_CONTRACT;
    }
    auto h = std::make_unique<lbm_handle>();
    try {
        validate_and_build(*h, *problem);
    } catch (const ContractError& e) {
        g_create_error = e.what();
        return LBM_E_CONTRACT;
    } catch (const CudaError& e) {
        g_create_error = e.what();
        return LBM_E_CUDA;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return LBM_E_CUDA;
    }
    g_create_error.clear();
    *out = h.release();
    return LBM_OK;
}

void lbm_destroy(lbm_handle* h) {
    if (!h) return;
    delete h->slab_adj;
    h->slab_adj = nullptr;
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->ckpts.clear();
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

lbm_status lbm_info(const lbm_handle* h, lbm_info_t* out) {
    if (!h || !out) return LBM_E_STATE;
    out->cells = h->G.n;
    out->fluid_cells = h->fluid_cells;
    out->q = h->Q;
    out->n_ports = h->n_ports;
    out->tau = h->tau;
    for (int d = 0; d < 3; ++d) out->acceleration_lattice[d] = h->a[d];
    out->device_bytes = h->device_bytes;
    return LBM_OK;
}

lbm_status lbm_set_design(lbm_handle* h, const double* raw, size_t n) {
    return guarded(h, [&]() {
        check_n(*h, n, (size_t)h->n(), "model:control");
        std::vector<float> r(n);
        for (size_t x = 0; x < n; ++x) {
            double v = raw[x];
            if (!std::isfinite(v) || v < 0.0 || v > 1.0)
                throw ContractError("model:control must be a finite shape-matched array in [0,1]");
            r[x] = (float)v;
        }
        CK(cudaMemcpyAsync(h->raw.p, r.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
        DesignArgs a = design_args(*h);
        const int grid = (int)std::min<int64_t>((h->n() + 255) / 256, (int64_t)h->sms * 8);
        CK(launch_design_map(a, grid, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->design_set = true;
        h->forward_done = false;
        return LBM_OK;
    });
}

lbm_status lbm_set_tau(lbm_handle* h, const double* tau, size_t n) {
    return guarded(h, [&]() {
        if (!tau) {
            h->tau_per_cell = false;
            h->forward_done = false;
            return LBM_OK;
        }
        if (h->coll != LBM_BGK)
            throw ContractError("per-cell relaxation times need the BGK collision (Tau::PerCell of the density-design "
                                "solver)");
        check_n(*h, n, (size_t)h->n(), "tau");
        std::vector<float> om(n);
        for (size_t x = 0; x < n; ++x) {
            if (!std::isfinite(tau[x]) || !(tau[x] > 0.5))
                throw ContractError("per-cell relaxation times must be finite and greater than 0.5");
            om[x] = (float)(1.0 / tau[x]);
        }
        h->omega_cell.alloc((n + CELL_PAD) * sizeof(float), &h->device_bytes);
        CK(cudaMemcpyAsync(h->omega_cell.p, om.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->tau_per_cell = true;
        h->forward_done = false;
        return LBM_OK;
    });
}

lbm_status lbm_get_design(lbm_handle* h, double* phi, double* alpha) {
    return guarded(h, [&]() {
        require_design(*h);
        std::vector<float> b((size_t)h->n());
        if (phi) {
            CK(cudaMemcpy(b.data(), h->phi.p, b.size() * 4, cudaMemcpyDeviceToHost));
            for (size_t x = 0; x < b.size(); ++x) phi[x] = b[x];
        }
        if (alpha) {
            CK(cudaMemcpy(b.data(), h->alpha.p, b.size() * 4, cudaMemcpyDeviceToHost));
            for (size_t x = 0; x < b.size(); ++x) alpha[x] = b[x];
        }
        return LBM_OK;
    });
}

lbm_status lbm_forward(lbm_handle* h, int64_t steps, lbm_diag_t* diag) {
    return guarded(h, [&]() {
        require_design(*h);
        h->forward_done = false;
        h->ckpts.clear();
        init_state(*h);
        const int64_t T = steps > 0 ? steps : h->step_count;
        lbm_status s = run_admitted(*h, T, diag, 0, h->time_average);
        h->forward_done = true;
        return s;
    });
}

lbm_status lbm_advance(lbm_handle* h, int64_t steps, lbm_diag_t* diag) {
    return guarded(h, [&]() {
        if (!h->state_valid) throw StateError("no current state: call lbm_forward or lbm_set_populations first");
        if (steps < 0) throw ContractError("steps must be non-negative");
        lbm_status s = run_admitted(*h, steps, diag, 0);
        h->forward_done = true;
        return s;
    });
}

lbm_status lbm_set_populations(lbm_handle* h, const double* f, size_t n) {
    return guarded(h, [&]() {
        const int64_t N = h->n();
        const int Q = h->Q;
        check_n(*h, n, (size_t)(N * Q), "populations");
        std::vector<float> g((size_t)N * Q);
        bool solid_nonfinite = false;
    // x-slab of a larger problem (lbm_create_slab): the owned planes are
    // [slab_hl, slab_hl + slab_own) of the local grid, the others ghost planes;
    // responses, seeds and port pressure weights use the whole problem's counts
    bool slab = false;
    int32_t slab_hl = 0, slab_hr = 0, slab_own = 0;
    int64_t global_fluid = -1, global_inlet = -1, global_outlet = -1;
        for (int64_t x = 0; x < N; ++x) {
            for (int q = 0; q < Q; ++q) g[(size_t)q * N + x] = (float)(f[x * Q + q] - h->L.w[q]);
            if (h->cls[x] == 0)  // solid
                for (int q = 0; q < Q; ++q) solid_nonfinite = solid_nonfinite || !std::isfinite(f[x * Q + q]);
        }
        ensure_scratch(*h);
        CK(cudaMemcpyAsync(h->scratch.p, g.data(), g.size() * 4, cudaMemcpyHostToDevice, h->stream));
        const int grid = grid_for(*h);
        // both arrays: solid cells keep their populations in either
        for (int k = 0; k < 2; ++k)
            CK(launch_upload_pop(Q, h->storage, h->G, k ? h->popB() : h->popA(), h->mask.as<uint32_t>(),
                                 h->scratch.as<float>(), grid, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        h->pending = false;
        h->t = 0;
        h->state_valid = true;
        h->forward_done = false;
        h->solid_nonfinite = solid_nonfinite;
        return LBM_OK;
    });
}

lbm_status lbm_get_populations(lbm_handle* h, double* f, size_t n) {
    return guarded(h, [&]() {
        if (!h->state_valid) throw StateError("no current state");
        const int64_t N = h->n();
        const int Q = h->Q;
        check_n(*h, n, (size_t)(N * Q), "populations");
        ensure_scratch(*h);
        CK(launch_canon_pop(Q, h->storage, h->G, h->popA(), h->mask.as<uint32_t>(), ports_at(*h, h->t),
                            h->pending ? 1 : 0, h->scratch.as<float>(), grid_for(*h), h->stream));
        std::vector<float> g((size_t)N * Q);
        CK(cudaMemcpyAsync(g.data(), h->scratch.p, g.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int64_t x = 0; x < N; ++x)
            for (int q = 0; q < Q; ++q) f[x * Q + q] = h->L.w[q] + (double)g[(size_t)q * N + x];
        return LBM_OK;
    });
}

lbm_status lbm_trajectory(lbm_handle* h, double* mass, double* exchange, double* min_population,
                          double* max_speed, size_t n) {
    return guarded(h, [&]() {
        const auto& d = h->last_trajectory;
        if (d.empty()) throw StateError("no trajectory: call lbm_forward or lbm_advance first");
        if (n != d.size()) throw ContractError("trajectory arrays must have steps + 1 entries");
        for (size_t t = 0; t < n; ++t) {
            if (mass) mass[t] = (double)h->fluid_cells + d[t].mass_hi + d[t].mass_lo;
            if (exchange) exchange[t] = t == 0 ? 0.0 : d[t].exch_hi + d[t].exch_lo;
            if (min_population) min_population[t] = d[t].min_f;
            if (max_speed) max_speed[t] = std::sqrt((double)d[t].max_u2);
        }
        return LBM_OK;
    });
}

lbm_status lbm_responses(lbm_handle* h, double* out8) {
    return guarded(h, [&]() {
        if (!h->state_valid) throw StateError("no current state");
        require_design(*h);
        responses(*h, out8, nullptr);
        return LBM_OK;
    });
}

lbm_status lbm_wall_loads(lbm_handle* h, double pressure_datum_pa, const double* origin_m, double* positions_m,
                          double* force_n, size_t capacity, size_t* n_links) {
    return guarded(h, [&]() {
        const size_t nl = h->wall_cells.size();
        if (n_links) *n_links = nl;
        if (!positions_m && !force_n) return LBM_OK;
        if (capacity < nl) throw ContractError("wall load outputs need room for n_links links");
        if (!std::isfinite(pressure_datum_pa)) throw ContractError("pressure datum must be finite");
        const double org[3] = {origin_m ? origin_m[0] : 0.0, origin_m ? origin_m[1] : 0.0,
                               origin_m ? origin_m[2] : 0.0};
        if (positions_m)
            for (size_t i = 0; i < nl; ++i) {
                const int64_t x = h->wall_cells[i];
                const int q = h->wall_links[i];
                const int64_t c[3] = {x / h->G.sx, (x / h->G.sy) % h->G.ny, x % h->G.nz};
                for (int a = 0; a < 3; ++a)
                    positions_m[3 * i + a] = org[a] + ((double)c[a] + 0.5 - 0.5 * h->L.c[q][a]) * h->dx;
            }
        if (!force_n) return LBM_OK;
        if (!h->forward_done || !h->state_valid || h->t < 1)
            throw StateError("wall loads need the states of a successful lbm_forward");
        require_design(*h);
        int64_t* ctr = &h->device_bytes;
        if (nl > 0) {
            h->wall_cells_d.alloc(nl * sizeof(uint32_t), ctr);
            h->wall_links_d.alloc(nl, ctr);
            h->wall_out.alloc(nl * sizeof(double), ctr);
            CK(cudaMemcpyAsync(h->wall_cells_d.p, h->wall_cells.data(), nl * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               h->stream));
            CK(cudaMemcpyAsync(h->wall_links_d.p, h->wall_links.data(), nl, cudaMemcpyHostToDevice, h->stream));
            // the state before the last step, pulled from the previous array
            const int64_t tb = h->t - 1;
            const void* prev = h->pop_array(h->cur ^ 1) + pop_pad(h->G) * storage_bytes(h->storage);
            CK(launch_wall_loads(h->Q, h->storage, h->G, h->P, prev, h->mask.as<uint32_t>(), h->alpha.as<float>(),
                                 ports_at(*h, tb), (tb >= 1 && h->n_ports > 0) ? 1 : 0, h->wall_cells_d.as<uint32_t>(),
                                 h->wall_links_d.as<uint8_t>(), (int64_t)nl, h->wall_out.as<double>(),
                                 h->tau_per_cell ? h->omega_cell.as<float>() : nullptr, h->stream));
        }
        std::vector<double> g(nl);
        if (nl > 0) CK(cudaMemcpyAsync(g.data(), h->wall_out.p, nl * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        // loads_from_post (wall_exchange.rs:86-100) in shifted populations:
        // f*_opp - w_q + w_q datum / unit = g*_opp + w_q datum / unit
        const double scale = h->density * std::pow(h->dx, 4) / (h->dt * h->dt);
        const double unit = h->density * (h->dx / h->dt) * (h->dx / h->dt) / 3.0;
        for (size_t i = 0; i < nl; ++i) {
            const int q = h->wall_links[i];
            const double mag = g[i] + h->L.w[q] * pressure_datum_pa / unit;
            for (int a = 0; a < 3; ++a) force_n[3 * i + a] = -2.0 * h->L.c[q][a] * mag * scale;
        }
        return LBM_OK;
    });
}

lbm_status lbm_probe_bounded_wait(int64_t limit_ns, int32_t* timed_out, double* waited_ms) {
    if (!timed_out || limit_ns < 1000000 || limit_ns > 1000000000) return LBM_E_CONTRACT;
    int* err = nullptr;
    unsigned long long* waited = nullptr;
    lbm_status st = LBM_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == LBM_OK) st = LBM_E_CUDA;
        return e == cudaSuccess;
    };
    if (ok(cudaMalloc(&err, sizeof(int))) && ok(cudaMalloc(&waited, sizeof(unsigned long long))) &&
        ok(cudaMemset(err, 0, sizeof(int))) && ok(launch_wait_probe(err, (uint64_t)limit_ns, waited, 0)) &&
        ok(cudaDeviceSynchronize())) {
        int e = 0;
        unsigned long long ns = 0;
        if (ok(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost)) &&
            ok(cudaMemcpy(&ns, waited, sizeof(ns), cudaMemcpyDeviceToHost))) {
            *timed_out = e ? 1 : 0;
            if (waited_ms) *waited_ms = (double)ns * 1e-6;
        }
    }
    if (err) cudaFree(err);
    if (waited) cudaFree(waited);
    return st;
}

lbm_status lbm_binomial_plan(int64_t steps, int64_t snapshots, int64_t* forward_steps, int64_t* peak_snapshots) {
    try {
        const RevolvePlan p = revolve_plan(steps, snapshots);
        if (forward_steps) *forward_steps = p.forward_steps;
        if (peak_snapshots) *peak_snapshots = p.peak;
        return LBM_OK;
    } catch (const std::invalid_argument&) {
        return LBM_E_CONTRACT;
    } catch (...) {
        return LBM_E_STATE;
    }
}

lbm_status lbm_time_average(lbm_handle* h, double* out8) {
    return guarded(h, [&]() {
        if (!h->time_average) throw ContractError("time averages need a problem created with time_average");
        if (!h->tavg_valid) throw StateError("no time average: call lbm_forward first");
        if (!out8) throw ContractError("out8 must not be NULL");
        for (int k = 0; k < 8; ++k) out8[k] = h->tavg[k];
        return LBM_OK;
    });
}

lbm_status lbm_fields(lbm_handle* h, double* density, double* velocity, double* pressure) {
    return guarded(h, [&]() {
        if (!h->state_valid) throw StateError("no current state");
        require_design(*h);
        const int64_t N = h->n();
        ensure_scratch(*h);
        double r8[8];
        responses(*h, r8, h->scratch.as<float>());
        std::vector<float> fl((size_t)N * 4);
        CK(cudaMemcpyAsync(fl.data(), h->scratch.p, fl.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        const double vel = h->dx / h->dt;
        const double unit = vel * vel / 3.0;
        for (int64_t x = 0; x < N; ++x) {
            const bool solid = h->cls[x] == 0;
            // solid cells keep their equilibrium populations: rho = 1, u = 0
            const double rp = solid ? 0.0 : (double)fl[x];
            const double rho = (1.0 + rp) * h->density;
            if (density) density[x] = rho;
            if (pressure) pressure[x] = (rho - h->density) * unit;
            if (velocity)
                for (int d = 0; d < 3; ++d) velocity[3 * x + d] = solid ? 0.0 : (double)fl[(size_t)(d + 1) * N + x] * vel;
        }
        return LBM_OK;
    });
}

lbm_status lbm_gradient(lbm_handle* h, const double* weights, const lbm_adjoint_opts_t* opts, double* grad,
                        lbm_adjoint_report_t* report) {
    return guarded(h, [&]() {
        lbm_adjoint_opts_t o{};
        o.mode = LBM_ADJ_HORIZON;
        o.lambda_storage = LBM_STORE_F32;
        o.checkpoint_every = 0;
        o.max_iterations = 100000;
        o.check_every = 50;
        o.tolerance = 1e-8;
        if (opts) o = *opts;
        if (!weights || !grad) throw ContractError("weights and grad must not be NULL");
        for (int k = 0; k < LBM_N_RESPONSES; ++k)
            if (!std::isfinite(weights[k])) throw ContractError("response weights must be finite");
        if (o.lambda_storage < LBM_STORE_F32 || o.lambda_storage > LBM_STORE_BF16)
            throw ContractError("lambda_storage must be float32, float16 or bfloat16");
        if (o.objective != LBM_OBJ_FINAL && o.objective != LBM_OBJ_TIME_AVERAGE)
            throw ContractError("objective must be final or time_average");
        if (o.objective == LBM_OBJ_TIME_AVERAGE && (o.mode != LBM_ADJ_HORIZON || !h->time_average))
            throw ContractError("the time-averaged objective needs the horizon adjoint and a problem created with "
                                "time_average");
        if (o.mode == LBM_ADJ_STEADY) {
            if (!(o.tolerance > 0)) throw ContractError("steady adjoint tolerance must be positive");
            return gradient_steady(*h, weights, o, grad, report);
        }
        if (o.mode != LBM_ADJ_HORIZON) throw ContractError("adjoint mode must be horizon or steady");
        if (o.checkpointing == LBM_CKPT_BINOMIAL) {
            if (o.snapshots < 1) throw ContractError("binomial checkpointing needs at least one snapshot");
            return gradient_binomial(*h, weights, o, grad, report);
        }
        if (o.checkpointing != LBM_CKPT_EVERY) throw ContractError("checkpointing must be every or binomial");
        return gradient_horizon(*h, weights, o, grad, report);
    });
}

namespace {
// interval_vjp (solver.rs:642-674) of one step from a host state: the
// cotangent of the state, of alpha and (tau_bar != NULL) of the per-cell
// relaxation times.
lbm_status step_vjp_impl(lbm_handle* h, const double* state, const double* lambda_next, double* lambda,
                         double* alpha_bar, double* tau_bar, size_t n_populations) {
    require_design(*h);
    const int64_t N = h->n();
    const int Q = h->Q;
    check_n(*h, n_populations, (size_t)(N * Q), "populations");
    lbm_status s = lbm_set_populations(h, state, n_populations);
    if (s != LBM_OK) throw ContractError(h->err);
    int64_t* ctr = &h->device_bytes;
    if (tau_bar) {
        // lbm_set_populations left the state's g = f - w planes in the scratch array
        h->tau_state.alloc((size_t)N * Q * sizeof(float), ctr);
        CK(cudaMemcpyAsync(h->tau_state.p, h->scratch.p, (size_t)N * Q * sizeof(float), cudaMemcpyDeviceToDevice,
                           h->stream));
        h->tau_bar.alloc((size_t)N * sizeof(double), ctr);
    }
    alloc_adjoint(*h, LBM_STORE_F32);
    h->record.alloc(((size_t)N * 4 + CELL_PAD) * sizeof(float), ctr);
    // nonlinear ports transpose at the next state (the extrapolations at the
    // neighbours, the regularized port at the port cell): its (rho - 1, u)
    // record from one step into the other array, which leaves the current
    // one (this state) in place
    DevBuf rec_next;
    if (h->nonlinear_ports) {
        rec_next.alloc(((size_t)N * 4 + CELL_PAD) * sizeof(float), ctr);
        const int cur = h->cur;
        const int64_t t0 = h->t;
        const bool pend = h->pending;
        step(*h, nullptr, nullptr);
        inspect(*h, nullptr, rec_next.as<float>());
        h->cur = cur;
        h->t = t0;
        h->pending = pend;
    }
    inspect(*h, nullptr, h->record.as<float>());
    std::vector<float> v((size_t)N * Q);
    for (int64_t x = 0; x < N; ++x)
        for (int q = 0; q < Q; ++q) v[(size_t)q * N + x] = (float)lambda_next[x * Q + q];
    ensure_scratch(*h);
    CK(cudaMemcpyAsync(h->scratch.p, v.data(), v.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CK(launch_seed_lam(Q, LBM_STORE_F32, h->G, h->lamA(), h->mask.as<uint32_t>(), ports_at(*h, h->t + 1),
                       h->scratch.as<float>(), 1.f, 1, rec_next.as<float>(), h->alpha.as<float>(), grid_for(*h),
                       h->stream));
    nee_move(*h, h->lamA(), LBM_STORE_F32);
    if (tau_bar)
        CK(launch_tau_bar(Q, h->G, h->P, h->tau_state.as<float>(), static_cast<const float*>(h->lamA()),
                          h->mask.as<uint32_t>(), h->alpha.as<float>(),
                          h->tau_per_cell ? h->omega_cell.as<float>() : nullptr, h->tau_bar.as<double>(),
                          grid_for(*h), h->stream));
    AdjArgs a = adj_args(*h);
    a.record = h->record.as<float>();
    a.port_transpose = 0;
    a.overwrite_abar = 1;
    a.in_scale_inv = 1.f;
    a.out_scale = 1.f;
    a.abar_factor = 1.f;
    CK(launch_adjoint(Q, coll_kernel(*h), LBM_STORE_F32, a, grid_for(*h), h->stream));
    h->lcur ^= 1;
    check_errflag(*h);
    CK(launch_canon_lam(Q, LBM_STORE_F32, h->G, h->lamA(), h->mask.as<uint32_t>(), 1.f, h->scratch.as<float>(),
                        grid_for(*h), h->stream));
    CK(cudaMemcpyAsync(v.data(), h->scratch.p, v.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    std::vector<float> ab((size_t)N);
    CK(cudaMemcpyAsync(ab.data(), h->abar.p, ab.size() * 4, cudaMemcpyDeviceToHost, h->stream));
    if (tau_bar)
        CK(cudaMemcpyAsync(tau_bar, h->tau_bar.p, (size_t)N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int64_t x = 0; x < N; ++x) {
        for (int q = 0; q < Q; ++q) lambda[x * Q + q] = v[(size_t)q * N + x];
        if (alpha_bar) alpha_bar[x] = h->cls[x] == 0 ? 0.0 : (double)ab[x];
    }
    return LBM_OK;
}
}  // namespace

lbm_status lbm_step_vjp(lbm_handle* h, const double* state, const double* lambda_next, double* lambda,
                        double* alpha_bar, size_t n_populations) {
    return guarded(h, [&]() { return step_vjp_impl(h, state, lambda_next, lambda, alpha_bar, nullptr, n_populations); });
}

lbm_status lbm_step_vjp_tau(lbm_handle* h, const double* state, const double* lambda_next, double* lambda,
                            double* alpha_bar, double* tau_bar, size_t n_populations) {
    return guarded(h, [&]() {
        if (!tau_bar) throw ContractError("tau_bar must not be NULL");
        if (h->coll != LBM_BGK)
            throw ContractError("per-cell relaxation times need the BGK collision (Tau::PerCell of the density-design "
                                "solver)");
        return step_vjp_impl(h, state, lambda_next, lambda, alpha_bar, tau_bar, n_populations);
    });
}

// ------------------------------------------------------------ x-slab decomposition
lbm_status lbm_create_slab(const lbm_problem_t* problem, int32_t x_begin, int32_t x_end, int32_t halo,
                           lbm_handle** out) {
    if (!out) return LBM_E_CONTRACT;
    *out = nullptr;
    try {
        if (!problem) throw ContractError("problem must not be NULL");
        const lbm_problem_t& P = *problem;
        const int nx = P.shape[0], ny = P.shape[1], nz = P.shape[2];
        require(nx >= 2 && ny >= 2 && nz >= 2, "LBM shape must contain three integers >= 2");
        require(P.solid_mask && P.design_region && P.fixed_design, "solid_mask must be a shape-matched boolean array");
        require(x_begin >= 0 && x_end <= nx && x_end - x_begin >= 2,
                "x-slab: the owned planes [x_begin, x_end) must lie in the grid and number two at least");
        require(!P.time_average, "x-slab decomposition does not run the time-averaged objective");
        const bool per = P.periodic_axes[0] != 0;
        int reach = 0;
        if (P.filter_kind == LBM_FILTER_BOX) reach = P.box_half_width;
        else if (P.filter_radius_m > 0 && P.spacing_m > 0) reach = (int)std::ceil(P.filter_radius_m / P.spacing_m);
        require(halo >= 1 && halo >= reach, "x-slab: halo must be at least 1 and cover the design filter's reach");
        const int hl = per ? halo : std::min(halo, (int)x_begin);
        const int hr = per ? halo : std::min(halo, nx - (int)x_end);
        const int own = x_end - x_begin, nxl = hl + own + hr;
        require(!per || nxl <= nx, "x-slab: the slab and its ghost planes must not wrap onto themselves");
        const int64_t sx = (int64_t)ny * nz, nl = (int64_t)nxl * sx, ng = (int64_t)nx * sx;
        auto gplane = [&](int pl) { return (int64_t)(((x_begin - hl + pl) % nx + nx) % nx); };
        std::vector<uint8_t> solid(nl), design(nl);
        std::vector<double> fixed(nl);
        for (int pl = 0; pl < nxl; ++pl)
            for (int64_t j = 0; j < sx; ++j) {
                const int64_t g = gplane(pl) * sx + j, l = (int64_t)pl * sx + j;
                solid[l] = P.solid_mask[g] ? 1 : 0;
                design[l] = P.design_region[g] ? 1 : 0;
                fixed[l] = P.fixed_design[g];
            }
        // ports: on the x faces only (their cells then lie in one slab); the
        // pressure-drop weights keep the whole problem's port cell counts
        std::vector<lbm_port_t> ports;
        std::vector<std::vector<uint8_t>> pmask;
        int64_t gin = 0, gout = 0;
        for (int k = 0; k < P.n_ports; ++k) {
            const lbm_port_t& pt = P.ports[k];
            require(pt.mask != nullptr, "Port mask must be a shape-matched boolean array");
            require(pt.face == LBM_XMIN || pt.face == LBM_XMAX, "x-slab decomposition supports ports on the x faces only");
            require(pt.reconstruction == LBM_RECON_LEGACY_MOMENT,
                    "x-slab decomposition supports legacy_moment ports only");
            int64_t cnt = 0;
            for (int64_t x = 0; x < ng; ++x) cnt += pt.mask[x] ? 1 : 0;
            (pt.kind == LBM_PORT_PRESSURE ? gout : gin) += cnt;
            std::vector<uint8_t> m(nl, 0);
            bool any = false;
            for (int pl = hl; pl < hl + own; ++pl)
                for (int64_t j = 0; j < sx; ++j) {
                    const uint8_t v = pt.mask[gplane(pl) * sx + j] ? 1 : 0;
                    m[(int64_t)pl * sx + j] = v;
                    any = any || v;
                }
            if (any) {
                pmask.push_back(std::move(m));
                ports.push_back(pt);
            }
        }
        for (size_t k = 0; k < ports.size(); ++k) ports[k].mask = pmask[k].data();
        int64_t gf = 0;
        for (int64_t x = 0; x < ng; ++x) gf += P.solid_mask[x] ? 0 : 1;
        lbm_problem_t L = P;
        L.shape[0] = nxl;
        L.periodic_axes[0] = 0;
        L.solid_mask = solid.data();
        L.design_region = design.data();
        L.fixed_design = fixed.data();
        L.n_ports = (int32_t)ports.size();
        L.ports = ports.empty() ? nullptr : ports.data();
        auto h = std::make_unique<lbm_handle>();
        h->slab = true;
        h->slab_hl = hl;
        h->slab_hr = hr;
        h->slab_own = own;
        h->global_fluid = gf;
        h->global_inlet = gin;
        h->global_outlet = gout;
        validate_and_build(*h, L);
        // ghost planes hold exchanged values and are never stepped
        std::vector<uint32_t> mask((size_t)nl);
        CK(cudaMemcpy(mask.data(), h->mask.p, (size_t)nl * 4, cudaMemcpyDeviceToHost));
        int64_t fluid_own = 0;
        for (int64_t x = 0; x < nl; ++x) {
            const int64_t pl = x / sx;
            if (pl < hl || pl >= hl + own) mask[x] |= MASK_SOLID;
            else fluid_own += solid[x] ? 0 : 1;
        }
        CK(cudaMemcpy(h->mask.p, mask.data(), (size_t)nl * 4, cudaMemcpyHostToDevice));
        h->fluid_cells = fluid_own;
        g_create_error.clear();
        *out = h.release();
        return LBM_OK;
    } catch (const ContractError& e) {
        g_create_error = e.what();
        return LBM_E_CONTRACT;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return LBM_E_CUDA;
    }
}

namespace {
void require_slab(const lbm_handle& h) {
    if (!h.slab) throw StateError("not an x-slab handle (lbm_create_slab)");
}

// Directions of a halo message: the state sends c_x = +1 to the right and
// -1 to the left, the adjoint the mirrored sets.
int halo_dirs(const lbm_handle& h, int kind, int side, int32_t* dirs) {
    const int sign = ((kind == 0) == (side == 1)) ? 1 : -1;
    int nd = 0;
    for (int q = 0; q < h.Q; ++q)
        if (h.L.c[q][0] == sign) dirs[nd++] = q;
    return nd;
}

void read_slab_diag(lbm_handle& h, lbm_slab_diag_t* out) {
    StepDiag d{};
    CK(cudaMemcpyAsync(&d, h.diag.p, sizeof(d), cudaMemcpyDeviceToHost, h.stream));
    CK(cudaStreamSynchronize(h.stream));
    check_errflag(h);
    if (out) {
        out->mass = (double)h.fluid_cells + d.mass_hi + d.mass_lo;
        out->exchange = d.exch_hi + d.exch_lo;
        out->minimum_population = d.min_f;
        out->maximum_speed2 = d.max_u2;
        out->nonfinite = d.nonfinite;
    }
}
}  // namespace

lbm_status lbm_slab_begin(lbm_handle* h) {
    return guarded(h, [&]() {
        require_slab(*h);
        require_design(*h);
        init_state(*h);
        h->forward_done = false;
        return LBM_OK;
    });
}

lbm_status lbm_slab_step(lbm_handle* h, lbm_slab_diag_t* diag) {
    return guarded(h, [&]() {
        require_slab(*h);
        if (!h->state_valid) throw StateError("no current state: call lbm_slab_begin first");
        h->diag.alloc(sizeof(StepDiag), &h->device_bytes);
        step(*h, h->diag.as<StepDiag>(), nullptr);
        read_slab_diag(*h, diag);
        h->forward_done = false;
        return LBM_OK;
    });
}

lbm_status lbm_slab_inspect(lbm_handle* h, lbm_slab_diag_t* diag) {
    return guarded(h, [&]() {
        require_slab(*h);
        if (!h->state_valid) throw StateError("no current state: call lbm_slab_begin first");
        h->diag.alloc(sizeof(StepDiag), &h->device_bytes);
        inspect(*h, h->diag.as<StepDiag>(), nullptr);
        read_slab_diag(*h, diag);
        h->forward_done = true;
        return LBM_OK;
    });
}

lbm_status lbm_halo_bytes(const lbm_handle* h, int32_t kind, size_t* bytes) {
    if (!h || !bytes || (kind != 0 && kind != 1)) return LBM_E_CONTRACT;
    int32_t dirs[27];
    const int nd = halo_dirs(*h, kind, 1, dirs);
    const int st = kind == 0 ? h->storage : LBM_STORE_F32;
    *bytes = (size_t)nd * (size_t)h->G.sx * storage_bytes(st);
    return LBM_OK;
}

namespace {
lbm_status halo_move(lbm_handle* h, int32_t kind, int32_t side, void* buf, int unpack) {
    return guarded(h, [&]() {
        require_slab(*h);
        if ((kind != 0 && kind != 1) || (side != 0 && side != 1) || !buf)
            throw ContractError("halo: kind must be 0 (state) or 1 (adjoint), side 0 (left) or 1 (right), buffer non-NULL");
        if (side == 0 ? h->slab_hl < 1 : h->slab_hr < 1)
            throw ContractError("halo: this slab has no neighbour on that side");
        if (kind == 0 && !h->state_valid) throw StateError("halo: no current state");
        if (kind == 1 && !h->slab_adj) throw StateError("halo: no adjoint in progress (lbm_slab_adjoint_begin)");
        int32_t dirs[27];
        // what arrives from a side is the neighbour's message travelling the other way
        const int nd = halo_dirs(*h, kind, unpack ? 1 - side : side, dirs);
        const int64_t sx = h->G.sx;
        const int64_t plane = unpack ? (side == 0 ? h->slab_hl - 1 : h->slab_hl + h->slab_own)
                                     : (side == 0 ? h->slab_hl : h->slab_hl + h->slab_own - 1);
        void* arr = kind == 0 ? h->popA() : h->lamA();
        const int st = kind == 0 ? h->storage : LBM_STORE_F32;
        if (kind == 0 && h->restored) throw StateError("halo: the current state is a restored checkpoint");
        CK(launch_halo_copy(st, arr, h->n(), plane * sx, sx, dirs, nd, buf, unpack, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return LBM_OK;
    });
}
}  // namespace

lbm_status lbm_halo_pack(lbm_handle* h, int32_t kind, int32_t side, void* device_buffer) {
    return halo_move(h, kind, side, device_buffer, 0);
}

lbm_status lbm_halo_unpack(lbm_handle* h, int32_t kind, int32_t side, const void* device_buffer) {
    return halo_move(h, kind, side, const_cast<void*>(device_buffer), 1);
}

lbm_status lbm_slab_adjoint_begin(lbm_handle* h, const double* weights, double* norm2) {
    return guarded(h, [&]() {
        require_slab(*h);
        if (!h->forward_done) throw StateError("lbm_slab_inspect must follow the last step before the adjoint");
        if (!weights) throw ContractError("weights must not be NULL");
        alloc_adjoint(*h, LBM_STORE_F32);
        int64_t* ctr = &h->device_bytes;
        const int64_t n = h->n();
        h->record.alloc(((size_t)n * 4 + CELL_PAD) * sizeof(float), ctr);
        h->abar_final.alloc((size_t)n * 4, ctr);
        h->phibar.alloc((size_t)n * 4, ctr);
        delete h->slab_adj;
        h->slab_adj = new AdjState();  // unit scale: the values cross ranks as they are
        // cotangents of the ghost planes belong to other ranks
        CK(cudaMemsetAsync(h->abar.p, 0, (size_t)n * 4, h->stream));
        CK(cudaMemsetAsync(h->abar_final.p, 0, (size_t)n * 4, h->stream));
        CK(cudaMemsetAsync(h->phibar.p, 0, (size_t)n * 4, h->stream));
        ObjArgs a = obj_args(*h);
        response_weights(*h, weights, 1.0, a.w);
        a.lam = h->lamA();
        a.abar_final = h->abar_final.as<float>();
        a.phibar = h->phibar.as<float>();
        a.record = h->record.as<float>();
        a.port_transpose = 1;
        a.norm2 = h->norm2.as<double>();
        a.write_lambda = 1;
        a.lam_scale = 1.f;
        CK(launch_objective(h->Q, h->storage, LBM_STORE_F32, 1, a, grid_for(*h), h->stream));
        double s2[2];
        CK(cudaMemcpyAsync(s2, h->norm2.p, sizeof(s2), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (norm2) *norm2 = s2[0] + s2[1];
        return LBM_OK;
    });
}

lbm_status lbm_slab_adjoint_step(lbm_handle* h, double* norm2) {
    return guarded(h, [&]() {
        require_slab(*h);
        if (!h->slab_adj) throw StateError("no adjoint in progress (lbm_slab_adjoint_begin)");
        adjoint_step(*h, *h->slab_adj, h->record.as<float>(), norm2 != nullptr);
        if (norm2) {
            double s2[2];
            CK(cudaMemcpyAsync(s2, h->norm2.p, sizeof(s2), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            *norm2 = s2[0] + s2[1];
        }
        return LBM_OK;
    });
}

lbm_status lbm_slab_gradient(lbm_handle* h, double* grad, size_t n) {
    return guarded(h, [&]() {
        require_slab(*h);
        if (!h->slab_adj) throw StateError("no adjoint in progress (lbm_slab_adjoint_begin)");
        check_n(*h, n, (size_t)h->n(), "grad");
        // the steps' alpha cotangents exist on owned fluid cells only; the
        // other entries were cleared when the adjoint began
        finish_gradient(*h, *h->slab_adj, h->slab_adj->steps > 0, grad);
        check_errflag(*h);
        return LBM_OK;
    });
}

lbm_status lbm_design_vjp(lbm_handle* h, const double* phi_bar, double* out, size_t n) {
    return guarded(h, [&]() {
        require_design(*h);
        check_n(*h, n, (size_t)h->n(), "phi_bar");
        int64_t* ctr = &h->device_bytes;
        h->phibar.alloc(n * 4, ctr);
        std::vector<float> v(n);
        for (size_t x = 0; x < n; ++x) v[x] = (float)phi_bar[x];
        CK(cudaMemcpyAsync(h->phibar.p, v.data(), n * 4, cudaMemcpyHostToDevice, h->stream));
        design_transpose(*h, h->phibar.as<float>(), nullptr, 1.f, nullptr);
        CK(cudaMemcpyAsync(v.data(), h->grad.p, n * 4, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (size_t x = 0; x < n; ++x) out[x] = v[x];
        return LBM_OK;
    });
}

}  // extern "C"
