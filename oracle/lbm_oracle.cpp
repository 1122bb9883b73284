// lbm_oracle.cpp -- FP64 CPU restatement of the reference's LBM density-design
// path.  TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline);
// the product never links it.  Parity unpinned: the reference ships no LBM
// tests or golden vectors and cannot be compiled here (no Rust toolchain); see
// lbm_oracle.h for how this restatement is checked instead.
//
// Every function cites the reference routine it restates (paths inside the
// reference project, crates/implexity-physics-lbm/src unless stated).
#include "lbm_oracle.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_error;

constexpr uint32_t NONE = 0xffffffffu;

// ---------------------------------------------------------------- lattices
// D3Q19: d3q19.rs:29-57.  D3Q27: moving/lattice.rs:93-121 (rest first, then
// the 26 moving velocities with x slowest, z fastest).
struct Lattice {
    int Q = 0;
    int c[27][3] = {};
    double w[27] = {};
    int opp[27] = {};
};

Lattice make_lattice(int q) {
    Lattice L;
    L.Q = q;
    if (q == 19) {
        const int C[19][3] = {{0, 0, 0},  {-1, -1, 0}, {-1, 0, -1}, {-1, 0, 0}, {-1, 0, 1},
                              {-1, 1, 0}, {0, -1, -1}, {0, -1, 0},  {0, -1, 1}, {0, 0, -1},
                              {0, 0, 1},  {0, 1, -1},  {0, 1, 0},   {0, 1, 1},  {1, -1, 0},
                              {1, 0, -1}, {1, 0, 0},   {1, 0, 1},   {1, 1, 0}};
        for (int i = 0; i < 19; ++i) {
            for (int d = 0; d < 3; ++d) L.c[i][d] = C[i][d];
            int n = std::abs(C[i][0]) + std::abs(C[i][1]) + std::abs(C[i][2]);
            L.w[i] = n == 0 ? 1.0 / 3.0 : (n == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
        }
    } else {
        int n = 1;
        for (int a = -1; a <= 1; ++a)
            for (int b = -1; b <= 1; ++b)
                for (int cc = -1; cc <= 1; ++cc) {
                    if (a == 0 && b == 0 && cc == 0) continue;
                    L.c[n][0] = a;
                    L.c[n][1] = b;
                    L.c[n][2] = cc;
                    ++n;
                }
        for (int i = 0; i < 27; ++i) {
            int m = std::abs(L.c[i][0]) + std::abs(L.c[i][1]) + std::abs(L.c[i][2]);
            L.w[i] = m == 0 ? 8.0 / 27.0 : m == 1 ? 2.0 / 27.0 : m == 2 ? 1.0 / 54.0 : 1.0 / 216.0;
        }
    }
    for (int i = 0; i < q; ++i)
        for (int j = 0; j < q; ++j)
            if (L.c[j][0] == -L.c[i][0] && L.c[j][1] == -L.c[i][1] && L.c[j][2] == -L.c[i][2]) L.opp[i] = j;
    return L;
}

// ---------------------------------------------------------------- MRT basis
// MomentBasis::new, moving/collision.rs:87-153.
struct Basis {
    std::vector<double> rows;  // Q*Q
    std::vector<double> norms; // Q
    std::vector<int> groups;   // Q
};

enum { G_MASS = 0, G_MOMENTUM = 1, G_BULK = 2, G_SHEAR = 3, G_ODD = 4, G_EVEN = 5 };

bool make_basis(const Lattice& L, Basis& B) {
    const int Q = L.Q;
    struct Cand {
        std::vector<double> p;
        int g;
    };
    std::vector<Cand> cands;
    auto poly = [&](auto fn, int g) {
        Cand c;
        c.p.resize(Q);
        c.g = g;
        for (int i = 0; i < Q; ++i) c.p[i] = fn((double)L.c[i][0], (double)L.c[i][1], (double)L.c[i][2]);
        cands.push_back(c);
    };
    poly([](double, double, double) { return 1.0; }, G_MASS);
    poly([](double x, double, double) { return x; }, G_MOMENTUM);
    poly([](double, double y, double) { return y; }, G_MOMENTUM);
    poly([](double, double, double z) { return z; }, G_MOMENTUM);
    poly([](double x, double y, double z) { return x * x + y * y + z * z; }, G_BULK);
    poly([](double x, double y, double z) { return 2 * x * x - y * y - z * z; }, G_SHEAR);
    poly([](double, double y, double z) { return y * y - z * z; }, G_SHEAR);
    poly([](double x, double y, double) { return x * y; }, G_SHEAR);
    poly([](double x, double, double z) { return x * z; }, G_SHEAR);
    poly([](double, double y, double z) { return y * z; }, G_SHEAR);
    for (int degree = 3; degree <= 6; ++degree)
        for (int a = 0; a <= 2; ++a)
            for (int b = 0; b <= 2; ++b) {
                int cc = degree - a - b;
                if (cc < 0 || cc > 2) continue;
                int g = degree % 2 == 1 ? G_ODD : G_EVEN;
                poly([=](double x, double y, double z) { return std::pow(x, a) * std::pow(y, b) * std::pow(z, cc); },
                     g);
            }
    auto inner = [&](const std::vector<double>& x, const std::vector<double>& y) {
        double s = 0;
        for (int i = 0; i < Q; ++i) s += L.w[i] * x[i] * y[i];
        return s;
    };
    std::vector<std::vector<double>> rows;
    B.norms.assign(Q, 0.0);
    B.groups.assign(Q, 0);
    for (auto& cand : cands) {
        if ((int)rows.size() == Q) break;
        double scale = inner(cand.p, cand.p);
        if (scale <= 0) continue;
        std::vector<double> v = cand.p;
        for (size_t k = 0; k < rows.size(); ++k) {
            double coef = inner(cand.p, rows[k]) / B.norms[k];
            for (int i = 0; i < Q; ++i) v[i] -= coef * rows[k][i];
        }
        double n = inner(v, v);
        if (n <= 1e-10 * scale) continue;
        B.norms[rows.size()] = n;
        B.groups[rows.size()] = cand.g;
        rows.push_back(v);
    }
    if ((int)rows.size() != Q) return false;
    B.rows.resize(Q * Q);
    for (int k = 0; k < Q; ++k)
        for (int i = 0; i < Q; ++i) B.rows[k * Q + i] = rows[k][i];
    return true;
}

// ---------------------------------------------------------------- problem
struct Port {
    bool pressure = false;
    int axis = 0, sign = 1;
    // 0: legacy moment (ports.rs:343-406); 1: neighbor_non_equilibrium
    // (ports.rs:484-497); 2: the moving engine's non-equilibrium extrapolation
    // (moving/boundary.rs:445-460); 3: regularized_known_stress
    // (ports.rs:409-482).  1 and 2 read the inward neighbour.
    int recon = 0;
    int64_t nb_off = 0;
    std::vector<double> sop;  // 3: the known-stress fit, 6 x Q (zero columns for the unknown populations)
    double vel[3] = {0, 0, 0};  // value in force at the current time
    double density = 1.0;
    std::vector<int64_t> cells;
    std::vector<double> jac;  // Q*Q, cell_jacobian at W (ports.rs:512-519)
    // pulsatile signal (moving/boundary.rs:98-126; value, moving/field.rs:1002-1013)
    bool pulsatile = false;
    double mean_vel[3] = {0, 0, 0}, amp_vel[3] = {0, 0, 0};  // lattice units
    double mean_p = 0, amp_p = 0;                              // Pa
    double freq = 0, phase = 0, ramp = 0;
};

struct Row {
    std::vector<std::pair<int64_t, double>> terms;
};

}  // namespace

struct orc_problem {
    Lattice L;
    // Tau::PerCell (solver.rs:171-187): per-cell relaxation times of the BGK
    // collision; empty = Tau::Uniform(tau)
    std::vector<double> tau_cell;
    int Q = 19;
    int coll = LBM_BGK;
    int64_t shape[3] = {0, 0, 0};
    bool periodic[3] = {false, false, false};
    int64_t N = 0;
    double dx = 0, dt = 0, density = 0, nu = 0, tau = 0;
    double a[3] = {0, 0, 0};
    double drag_max = 0, drag_shape = 0, mach_limit = 0;
    std::vector<uint8_t> solid, editable;
    std::vector<double> fixed;
    // design map
    bool filtered = false;
    std::vector<Row> rows;
    std::vector<double> den;
    double beta = 0, eta = 0.5;
    // streaming
    std::vector<uint8_t> blocked;
    std::vector<uint32_t> source;
    std::vector<uint32_t> readers;  // 2 per slot
    // ports (values follow the port signal: set_port_time)
    mutable std::vector<Port> ports;
    double pressure_unit = 1.0;  // 3 / (rho_phys c^2), Pa -> lattice density
    std::vector<int8_t> port_role;  // +1 inlet (velocity), -1 outlet (pressure), 0 otherwise
    int64_t n_inlet = 0, n_outlet = 0;
    // collision
    double omega = 0, om = 0;  // shear and odd rates
    Basis basis;
    double bulk_rate = NAN, even_rate = NAN;
    int64_t fluid_cells = 0;
};

namespace {

// Grid::coords / wrap / inside (d3q19.rs:91-123)
inline void coords(const orc_problem& o, int64_t x, int64_t out[3]) {
    int64_t k = x % o.shape[2];
    int64_t ij = x / o.shape[2];
    out[0] = ij / o.shape[1];
    out[1] = ij % o.shape[1];
    out[2] = k;
}
inline int64_t index3(const orc_problem& o, int64_t i, int64_t j, int64_t k) {
    return (i * o.shape[1] + j) * o.shape[2] + k;
}
inline int64_t wrap(const orc_problem& o, int64_t x, const int64_t off[3]) {
    int64_t c[3];
    coords(o, x, c);
    int64_t r[3];
    for (int a = 0; a < 3; ++a) {
        int64_t n = o.shape[a];
        int64_t v = (c[a] + off[a]) % n;
        if (v < 0) v += n;
        r[a] = v;
    }
    return index3(o, r[0], r[1], r[2]);
}
inline bool inside(const orc_problem& o, int64_t x, const int64_t off[3]) {
    int64_t c[3];
    coords(o, x, c);
    for (int a = 0; a < 3; ++a) {
        int64_t v = c[a] + off[a];
        if (!o.periodic[a] && (v < 0 || v >= o.shape[a])) return false;
    }
    return true;
}

// ports.rs:274-316
inline void moments(const Lattice& L, const double* f, double& rho, double m[3]) {
    rho = 0;
    m[0] = m[1] = m[2] = 0;
    for (int q = 0; q < L.Q; ++q) {
        rho += f[q];
        for (int d = 0; d < 3; ++d) m[d] += f[q] * L.c[q][d];
    }
}
inline double dotc(const Lattice& L, int q, const double v[3]) {
    return v[0] * L.c[q][0] + v[1] * L.c[q][1] + v[2] * L.c[q][2];
}

// ports.rs:343-406 (legacy moment reconstruction), generalised to the
// lattice's own velocity set.
void reconstruct(const orc_problem& o, const Port& p, const double* f, double* out) {
    const Lattice& L = o.L;
    const int Q = L.Q;
    int axis = p.axis, sign = p.sign;
    std::vector<int> unknown, outgoing, zero;
    for (int q = 0; q < Q; ++q) {
        if (L.c[q][axis] == sign) unknown.push_back(q);
        else if (L.c[q][axis] == -sign) outgoing.push_back(q);
        else zero.push_back(q);
    }
    int t0 = -1, t1 = -1;
    for (int a = 0; a < 3; ++a)
        if (a != axis) (t0 < 0 ? t0 : t1) = a;
    double v0[3];
    for (int d = 0; d < 3; ++d) v0[d] = p.vel[d] - 0.5 * o.a[d];
    double compat = 0;
    for (int q : zero) compat += f[q];
    double out_sum = 0;
    for (int q : outgoing) out_sum += f[q];
    compat += 2.0 * out_sum;
    double sgn = sign;
    double rho, v[3] = {v0[0], v0[1], v0[2]};
    if (!p.pressure) {
        rho = compat / (1.0 - sgn * v0[axis]);
    } else {
        rho = p.density;
        v[axis] = (1.0 - compat / rho) * sgn;
    }
    const int U = (int)unknown.size();
    std::vector<double> proposal(U);
    for (int k = 0; k < U; ++k) {
        int q = unknown[k];
        proposal[k] = f[L.opp[q]] + rho * (6.0 * L.w[q]) * dotc(L, q, v);
    }
    double known_mass = 0, known_mom[3] = {0, 0, 0};
    for (int q = 0; q < Q; ++q) {
        if (L.c[q][axis] == sign) continue;
        known_mass += f[q];
        for (int d = 0; d < 3; ++d) known_mom[d] += f[q] * L.c[q][d];
    }
    double target[3] = {rho - known_mass, rho * v[t0] - known_mom[t0], rho * v[t1] - known_mom[t1]};
    double pa[3] = {0, 0, 0};
    for (int k = 0; k < U; ++k) {
        int q = unknown[k];
        pa[0] += proposal[k];
        pa[1] += proposal[k] * L.c[q][t0];
        pa[2] += proposal[k] * L.c[q][t1];
    }
    double res[3] = {target[0] - pa[0], target[1] - pa[1], target[2] - pa[2]};
    // right_inverse (ports.rs:320-341): R^T (R R^T)^-1 with rows 1, c_t0, c_t1
    double M[3][3] = {};
    std::vector<double> rw[3];
    for (int r = 0; r < 3; ++r) rw[r].resize(U);
    for (int k = 0; k < U; ++k) {
        rw[0][k] = 1.0;
        rw[1][k] = L.c[unknown[k]][t0];
        rw[2][k] = L.c[unknown[k]][t1];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < U; ++k) s += rw[i][k] * rw[j][k];
            M[i][j] = s;
        }
    double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                 M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    double inv[3][3] = {};
    if (det != 0) {
        inv[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
        inv[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        inv[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
        inv[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        inv[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
        inv[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        inv[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
        inv[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        inv[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
    }
    for (int q = 0; q < Q; ++q) out[q] = f[q];
    for (int k = 0; k < U; ++k) {
        double ri[3];
        for (int j = 0; j < 3; ++j) ri[j] = rw[0][k] * inv[0][j] + rw[1][k] * inv[1][j] + rw[2][k] * inv[2][j];
        out[unknown[k]] = proposal[k] + res[0] * ri[0] + res[1] * ri[1] + res[2] * ri[2];
    }
}

// design.rs:282-294
// Signal::factors (moving/boundary.rs:111-125): C2 smoothstep ramp and the
// sine wave at time t seconds.
void signal_factors(const Port& p, double t, double& ramp, double& wave) {
    ramp = 1.0;
    if (p.ramp > 0.0 && t < p.ramp) {
        double s = t / p.ramp;
        if (s < 0.0) s = 0.0;
        ramp = s * s * s * (10.0 - s * 15.0 + s * s * 6.0);
    }
    wave = p.freq == 0.0 ? 0.0 : std::sin(t * (2.0 * M_PI * p.freq) + p.phase);
}

// cell_jacobian at W (ports.rs:512-519) for the port's current value.
void port_jacobian(const orc_problem& o, Port& pt) {
    const int Q = o.Q;
    pt.jac.assign(Q * Q, 0.0);
    double base[27] = {}, pert[27] = {}, r0[27] = {}, r1[27] = {};
    for (int q = 0; q < Q; ++q) base[q] = o.L.w[q];
    reconstruct(o, pt, base, r0);
    for (int kq = 0; kq < Q; ++kq) {
        for (int q = 0; q < Q; ++q) pert[q] = base[q];
        pert[kq] += 1.0;
        reconstruct(o, pt, pert, r1);
        for (int r = 0; r < Q; ++r) pt.jac[r * Q + kq] = r1[r] - r0[r];
    }
}

// Port values of the reconstruction that produces state t_index
// (t = t_index * dt; moving/field.rs:1002-1013): ramp (wave amplitude + mean).
// Non-equilibrium extrapolation from the inward neighbour's populations nb
// (f form): out = eq(rho_b, u_b) + nb - eq(rho_n, u_n), u_n = j_n / rho_n.
// ports.rs reconstruct_neighbor (:484-497, pressure ports): rho_b = the port
// density, u_b = the port velocity with its axial component taken from u_n.
// moving/boundary.rs port_populations (:445-460): velocity ports rho_b =
// rho_n, u_b = the port velocity; pressure ports rho_b = the port density,
// u_b = u_n.
void nee_targets(const orc_problem& o, const Port& p, double rho_n, const double u_n[3], double& rho_b, double u_b[3]) {
    for (int d = 0; d < 3; ++d) u_b[d] = p.vel[d];
    if (p.recon == 1) {
        rho_b = p.density;
        u_b[p.axis] = u_n[p.axis];
    } else if (p.pressure) {
        rho_b = p.density;
        for (int d = 0; d < 3; ++d) u_b[d] = u_n[d];
    } else {
        rho_b = rho_n;
    }
}

void nee_apply(const orc_problem& o, const Port& p, const double* nb, double* out) {
    const Lattice& L = o.L;
    double rho_n, j[3], u_n[3], rho_b, u_b[3];
    moments(L, nb, rho_n, j);
    for (int d = 0; d < 3; ++d) u_n[d] = j[d] / rho_n;
    nee_targets(o, p, rho_n, u_n, rho_b, u_b);
    const double ub2 = u_b[0] * u_b[0] + u_b[1] * u_b[1] + u_b[2] * u_b[2];
    const double un2 = u_n[0] * u_n[0] + u_n[1] * u_n[1] + u_n[2] * u_n[2];
    for (int q = 0; q < L.Q; ++q) {
        const double cb = dotc(L, q, u_b), cn = dotc(L, q, u_n);
        const double eb = rho_b * L.w[q] * (1.0 + 3.0 * cb + 4.5 * cb * cb - 1.5 * ub2);
        const double en = rho_n * L.w[q] * (1.0 + 3.0 * cn + 4.5 * cn * cn - 1.5 * un2);
        out[q] = eb + nb[q] - en;
    }
}

// equilibrium_vjp: cotangents of rho and u of sum_q g_q eq_q(rho, u)
void eq_vjp(const orc_problem& o, double rho, const double u[3], const double* g, double sign, double& rb,
            double ub[3]) {
    const Lattice& L = o.L;
    const double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int q = 0; q < L.Q; ++q) {
        const double gq = sign * g[q], cu = dotc(L, q, u);
        rb += gq * L.w[q] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2);
        for (int d = 0; d < 3; ++d) ub[d] += gq * rho * L.w[q] * (3.0 * L.c[q][d] + 9.0 * cu * L.c[q][d] - 3.0 * u[d]);
    }
}

// port_populations_vjp (moving/boundary.rs:462-506) for both extrapolations:
// nb_bar = d out / d nb ^T g at the neighbour populations nb.
void nee_vjp(const orc_problem& o, const Port& p, const double* nb, const double* g, double* nb_bar) {
    const Lattice& L = o.L;
    double rho_n, j[3], u_n[3], rho_b, u_b[3];
    moments(L, nb, rho_n, j);
    for (int d = 0; d < 3; ++d) u_n[d] = j[d] / rho_n;
    nee_targets(o, p, rho_n, u_n, rho_b, u_b);
    double rb = 0, ub[3] = {0, 0, 0}, rn = 0, un[3] = {0, 0, 0};
    eq_vjp(o, rho_b, u_b, g, 1.0, rb, ub);
    eq_vjp(o, rho_n, u_n, g, -1.0, rn, un);
    if (p.recon == 1) {
        un[p.axis] += ub[p.axis];
    } else if (p.pressure) {
        for (int d = 0; d < 3; ++d) un[d] += ub[d];
    } else {
        rn += rb;
    }
    double jb[3];
    for (int d = 0; d < 3; ++d) {
        jb[d] = un[d] / rho_n;
        rn -= un[d] * j[d] / (rho_n * rho_n);
    }
    for (int q = 0; q < L.Q; ++q) {
        double v = g[q] + rn;
        for (int d = 0; d < 3; ++d) v += jb[d] * L.c[q][d];
        nb_bar[q] = v;
    }
}

// Regularized known-stress port (ports.rs known_stress_operator :409-439,
// reconstruct_regularized :455-482).  Basis of the deviatoric second
// moment: B[q][r] = 4.5 w_q (c_a c_b - delta_ab / 3) over (xx, yy, zz, 2xy,
// 2xz, 2yz).  The stress is the weighted least-squares fit of the known
// populations' non-equilibrium parts (known: c_axis != sign), sop = pinv(M)
// with M[k][r] = B[known_k][r] / sqrt(w), columns rescaled by 1 / sqrt(w).
double stress_basis(const Lattice& L, int q, int r) {
    static const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    const double qq = L.c[q][ia[r]] * L.c[q][ib[r]] - (ia[r] == ib[r] ? 1.0 / 3.0 : 0.0);
    return 4.5 * L.w[q] * (r < 3 ? qq : 2.0 * qq);
}

bool regularized_operator(const Lattice& L, Port& pt) {
    const int Q = L.Q;
    std::vector<int> known;
    for (int q = 0; q < Q; ++q)
        if (L.c[q][pt.axis] != pt.sign) known.push_back(q);
    const int K = (int)known.size();
    // pinv of the full-column-rank K x 6 matrix M: (M^T M)^-1 M^T
    double G[6][12] = {};
    for (int r = 0; r < 6; ++r) {
        for (int c2 = 0; c2 < 6; ++c2) {
            double acc = 0;
            for (int k = 0; k < K; ++k) {
                const double wq = L.w[known[k]];
                acc += stress_basis(L, known[k], r) * stress_basis(L, known[k], c2) / wq;
            }
            G[r][c2] = acc;
        }
        G[r][6 + r] = 1.0;
    }
    double scale = 0;
    for (int r = 0; r < 6; ++r) scale = std::max(scale, std::fabs(G[r][r]));
    for (int c2 = 0; c2 < 6; ++c2) {
        int piv = c2;
        for (int r = c2 + 1; r < 6; ++r)
            if (std::fabs(G[r][c2]) > std::fabs(G[piv][c2])) piv = r;
        if (std::fabs(G[piv][c2]) <= 1e-12 * scale) return false;  // rank deficient
        for (int j = 0; j < 12; ++j) std::swap(G[c2][j], G[piv][j]);
        const double d = G[c2][c2];
        for (int j = 0; j < 12; ++j) G[c2][j] /= d;
        for (int r = 0; r < 6; ++r) {
            if (r == c2) continue;
            const double m = G[r][c2];
            for (int j = 0; j < 12; ++j) G[r][j] -= m * G[c2][j];
        }
    }
    // sop[r][q] = sum_c inv[r][c] M[k][c] / sqrt(w) = sum_c inv[r][c] B[q][c] / w
    pt.sop.assign((size_t)6 * Q, 0.0);
    for (int r = 0; r < 6; ++r)
        for (int q : known) {
            double acc = 0;
            for (int c2 = 0; c2 < 6; ++c2) acc += G[r][6 + c2] * stress_basis(L, q, c2);
            pt.sop[(size_t)r * Q + q] = acc / L.w[q];
        }
    return true;
}

void regularized_apply(const orc_problem& o, const Port& p, const double* f, double* out) {
    const Lattice& L = o.L;
    const int Q = L.Q;
    double tgt[27], rho, j[3], u[3], eq[27], stress[6] = {0, 0, 0, 0, 0, 0};
    reconstruct(o, p, f, tgt);
    moments(L, tgt, rho, j);
    for (int d = 0; d < 3; ++d) u[d] = j[d] / rho;
    const double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    for (int q = 0; q < Q; ++q) {
        const double cu = dotc(L, q, u);
        eq[q] = rho * L.w[q] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * u2);
    }
    for (int r = 0; r < 6; ++r)
        for (int q = 0; q < Q; ++q) stress[r] += (f[q] - eq[q]) * p.sop[(size_t)r * Q + q];
    for (int q = 0; q < Q; ++q) {
        double acc = eq[q];
        for (int r = 0; r < 6; ++r) acc += stress[r] * stress_basis(L, q, r);
        out[q] = acc;
    }
}

// Transpose of regularized_apply at a streamed state whose rebuilt
// populations are `post`: the map depends on the streamed populations
// nonlinearly only through the density and velocity of the legacy target,
// and the rebuilt cell carries exactly those (the stress basis has no mass
// or momentum), so post's moments fix the linearisation.
void regularized_vjp(const orc_problem& o, const Port& p, const double* post, const double* g, double* fb) {
    const Lattice& L = o.L;
    const int Q = L.Q;
    double rho, j[3], u[3];
    moments(L, post, rho, j);
    for (int d = 0; d < 3; ++d) u[d] = j[d] / rho;
    double sb[6] = {0, 0, 0, 0, 0, 0}, direct[27], eqb[27];
    for (int r = 0; r < 6; ++r)
        for (int q = 0; q < Q; ++q) sb[r] += g[q] * stress_basis(L, q, r);
    for (int q = 0; q < Q; ++q) {
        double acc = 0;
        for (int r = 0; r < 6; ++r) acc += sb[r] * p.sop[(size_t)r * Q + q];
        direct[q] = acc;
        eqb[q] = g[q] - acc;
    }
    double rb = 0, ub[3] = {0, 0, 0};
    eq_vjp(o, rho, u, eqb, 1.0, rb, ub);
    double jb[3];
    for (int d = 0; d < 3; ++d) {
        jb[d] = ub[d] / rho;
        rb -= ub[d] * u[d] / rho;
    }
    double tb[27];
    for (int q = 0; q < Q; ++q) tb[q] = rb + jb[0] * L.c[q][0] + jb[1] * L.c[q][1] + jb[2] * L.c[q][2];
    // the legacy target is affine: its Jacobian p.jac (rows r, columns k)
    for (int k = 0; k < Q; ++k) {
        double acc = direct[k];
        for (int r = 0; r < Q; ++r) acc += p.jac[(size_t)r * Q + k] * tb[r];
        fb[k] = acc;
    }
}

void set_port_time(const orc_problem& o, int64_t t_index) {
    const double t = (double)t_index * o.dt;
    for (Port& p : o.ports) {
        if (!p.pulsatile) continue;
        double ramp, wave;
        signal_factors(p, t, ramp, wave);
        if (p.pressure) p.density = 1.0 + ramp * (wave * p.amp_p + p.mean_p) * o.pressure_unit;
        for (int d = 0; d < 3; ++d) p.vel[d] = ramp * (wave * p.amp_vel[d] + p.mean_vel[d]);
        port_jacobian(o, p);
    }
}

inline double resistance(const orc_problem& o, double phi) {
    return o.dt * o.drag_max * o.drag_shape * (1.0 - phi) / (o.drag_shape + phi);
}
inline double resistance_derivative(const orc_problem& o, double phi) {
    double q = o.drag_shape, d = q + phi;
    return o.dt * o.drag_max * q * (-d - (1.0 - phi)) / (d * d);
}

// ---------------------------------------------------------------- collision
// Macroscopic state with the implicit half-step Brinkman velocity
// (solver.rs:190-196; moving/psm.rs:213-226 with zero solid velocity).
inline void macroscopic(const orc_problem& o, const double* f, double alpha, double& rho, double u[3],
                        double F[3]) {
    double m[3];
    moments(o.L, f, rho, m);
    double s = alpha * 0.5 + 1.0;
    for (int d = 0; d < 3; ++d) u[d] = (m[d] / rho + 0.5 * o.a[d]) / s;
    for (int d = 0; d < 3; ++d) F[d] = rho * (o.a[d] - alpha * u[d]);
}

// Static-provider BGK (solver.rs:298-322).
void collide_bgk(const orc_problem& o, const double* f, double alpha, double* out, double tau) {
    const Lattice& L = o.L;
    double rho, u[3], F[3];
    macroscopic(o, f, alpha, rho, u, F);
    double uf = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double k = 1.0 - 0.5 / tau;
    for (int q = 0; q < L.Q; ++q) {
        double cu = dotc(L, q, u), cf = dotc(L, q, F);
        double eq = rho * L.w[q] * (1.0 + cu * 3.0 + cu * cu * 4.5 - usq * 1.5);
        double src = k * L.w[q] * (cf * 3.0 - uf * 3.0 + cu * cf * 9.0);
        out[q] = f[q] - (f[q] - eq) / tau + src;
    }
}

// The relaxation time of cell x (Tau::at, solver.rs:180-186).
inline double tau_at(const orc_problem& o, int64_t x) { return o.tau_cell.empty() ? o.tau : o.tau_cell[x]; }

// collide_cell_vjp, solver.rs:214-285 (returns f_bar, alpha_bar and tau_bar).
void collide_bgk_vjp(const orc_problem& o, const double* f, double alpha, const double* g, double* f_bar,
                     double& alpha_bar, double tau, double& tau_bar) {
    const Lattice& L = o.L;
    const int Q = L.Q;
    double rho, m[3];
    moments(L, f, rho, m);
    double s = 1.0 + 0.5 * alpha;
    double u[3], F[3];
    for (int d = 0; d < 3; ++d) u[d] = (m[d] / rho + 0.5 * o.a[d]) / s;
    for (int d = 0; d < 3; ++d) F[d] = rho * (o.a[d] - alpha * u[d]);
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double uf = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
    double k = 1.0 - 0.5 / tau;
    double rho_bar = 0, uf_bar = 0, usq_bar = 0;
    tau_bar = 0;
    double u_bar[3] = {0, 0, 0}, F_bar[3] = {0, 0, 0};
    for (int q = 0; q < Q; ++q) f_bar[q] = 0;
    for (int q = 0; q < Q; ++q) {
        double gq = g[q];
        if (gq == 0.0) continue;
        double cu = dotc(L, q, u), cf = dotc(L, q, F);
        double poly = 1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq;
        f_bar[q] += gq * (1.0 - 1.0 / tau);
        double eq_bar = gq / tau;
        double eq = rho * L.w[q] * poly;
        tau_bar += gq * (f[q] - eq) / (tau * tau) +
                   gq * L.w[q] * (0.5 / (tau * tau)) * (3.0 * cf - 3.0 * uf + 9.0 * cu * cf);
        double h = gq * L.w[q] * k;
        double cf_bar = h * (3.0 + 9.0 * cu);
        double cu_bar = h * 9.0 * cf;
        uf_bar -= 3.0 * h;
        rho_bar += eq_bar * L.w[q] * poly;
        double e = eq_bar * rho * L.w[q];
        cu_bar += e * (3.0 + 9.0 * cu);
        usq_bar -= 1.5 * e;
        for (int d = 0; d < 3; ++d) {
            u_bar[d] += cu_bar * L.c[q][d];
            F_bar[d] += cf_bar * L.c[q][d];
        }
    }
    for (int d = 0; d < 3; ++d) {
        u_bar[d] += usq_bar * 2.0 * u[d] + uf_bar * F[d];
        F_bar[d] += uf_bar * u[d];
    }
    double a_bar = 0;
    for (int d = 0; d < 3; ++d) {
        rho_bar += F_bar[d] * (o.a[d] - alpha * u[d]);
        a_bar -= F_bar[d] * rho * u[d];
        u_bar[d] -= F_bar[d] * rho * alpha;
    }
    double m_bar[3], s_bar = 0;
    for (int d = 0; d < 3; ++d) {
        m_bar[d] = u_bar[d] / (s * rho);
        rho_bar -= u_bar[d] * m[d] / (s * rho * rho);
        s_bar -= u_bar[d] * u[d] / s;
    }
    a_bar += 0.5 * s_bar;
    for (int q = 0; q < Q; ++q) {
        double v = f_bar[q] + rho_bar;
        for (int d = 0; d < 3; ++d) v += m_bar[d] * L.c[q][d];
        f_bar[q] = v;
    }
    alpha_bar = a_bar;
}

// TRT collide_pairs, moving/collision.rs:457-488.
void collide_pairs(const orc_problem& o, const double* f, double rho, const double u[3], const double F[3],
                   double* out) {
    const Lattice& L = o.L;
    double omega = o.omega, om = o.om;
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double uf = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
    double base = 1.0 - usq * 1.5;
    double kp = 1.0 - omega * 0.5, km = 1.0 - om * 0.5;
    double w0 = L.w[0];
    double eq0 = rho * w0 * base;
    out[0] = f[0] - omega * (f[0] - eq0) - kp * uf * (3.0 * w0);
    for (int i = 1; i < L.Q; ++i) {
        int oi = L.opp[i];
        if (oi < i) continue;
        double w = L.w[i];
        double cu = dotc(L, i, u), cf = dotc(L, i, F);
        double wr = rho * w;
        double eqp = wr * (base + cu * cu * 4.5);
        double eqm = wr * cu * 3.0;
        double sp = (cu * cf * 9.0 - uf * 3.0) * w;
        double sm = cf * (3.0 * w);
        double fp = (f[i] + f[oi]) * 0.5, fm = (f[i] - f[oi]) * 0.5;
        double A = kp * sp - omega * (fp - eqp);
        double Bv = km * sm - om * (fm - eqm);
        out[i] = f[i] + A + Bv;
        out[oi] = f[oi] + A - Bv;
    }
}

// collide_pairs_vjp, moving/collision.rs:492-570 (omega is fixed: no rate cotangent).
void collide_pairs_vjp(const orc_problem& o, const double* f, double rho, const double u[3], const double F[3],
                       const double* g, double* f_bar, double& rho_bar, double u_bar[3], double F_bar[3]) {
    const Lattice& L = o.L;
    (void)f;
    double omega = o.omega, om = o.om;
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double base = 1.0 - usq * 1.5;
    double kp = 1.0 - omega * 0.5, km = 1.0 - om * 0.5;
    rho_bar = 0;
    double usq_bar = 0, uf_bar = 0;
    for (int d = 0; d < 3; ++d) u_bar[d] = F_bar[d] = 0;
    double w0 = L.w[0];
    double g0 = g[0];
    f_bar[0] = g0 * (1.0 - omega);
    rho_bar += g0 * omega * w0 * base;
    usq_bar -= g0 * omega * rho * (1.5 * w0);
    uf_bar -= g0 * kp * (3.0 * w0);
    for (int i = 1; i < L.Q; ++i) {
        int oi = L.opp[i];
        if (oi < i) continue;
        double w = L.w[i];
        double cu = dotc(L, i, u), cf = dotc(L, i, F);
        double wr = rho * w;
        double a_bar = g[i] + g[oi];
        double b_bar = g[i] - g[oi];
        double fp_bar = -omega * a_bar, fm_bar = -om * b_bar;
        double eqp_bar = omega * a_bar, eqm_bar = om * b_bar;
        double sp_bar = kp * a_bar, sm_bar = km * b_bar;
        f_bar[i] = g[i] + (fp_bar + fm_bar) * 0.5;
        f_bar[oi] = g[oi] + (fp_bar - fm_bar) * 0.5;
        rho_bar += eqp_bar * w * (base + cu * cu * 4.5) + eqm_bar * cu * (3.0 * w);
        usq_bar -= eqp_bar * wr * 1.5;
        double cu_bar = eqp_bar * wr * cu * 9.0 + eqm_bar * wr * 3.0 + sp_bar * cf * (9.0 * w);
        double cf_bar = sp_bar * cu * (9.0 * w) + sm_bar * (3.0 * w);
        uf_bar -= sp_bar * (3.0 * w);
        for (int d = 0; d < 3; ++d) {
            if (L.c[i][d] != 0) {
                u_bar[d] += cu_bar * L.c[i][d];
                F_bar[d] += cf_bar * L.c[i][d];
            }
        }
    }
    for (int d = 0; d < 3; ++d) {
        u_bar[d] += usq_bar * u[d] * 2.0 + uf_bar * F[d];
        F_bar[d] += uf_bar * u[d];
    }
}

inline void equilibrium(const Lattice& L, double rho, const double u[3], double* eq) {
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double base = 1.0 - usq * 1.5;
    for (int i = 0; i < L.Q; ++i) {
        double cu = dotc(L, i, u);
        eq[i] = rho * L.w[i] * (base + cu * 3.0 + cu * cu * 4.5);
    }
}

// equilibrium_vjp, moving/lattice.rs:194-221
void equilibrium_vjp(const Lattice& L, double rho, const double u[3], const double* g, double& rho_bar,
                     double u_bar[3]) {
    double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    double base = 1.0 - usq * 1.5;
    double usq_bar = 0;
    for (int i = 0; i < L.Q; ++i) {
        double cu = dotc(L, i, u);
        double poly = base + cu * 3.0 + cu * cu * 4.5;
        double gw = g[i] * L.w[i];
        rho_bar += gw * poly;
        double e = gw * rho;
        double cu_bar = e * (cu * 9.0 + 3.0);
        for (int d = 0; d < 3; ++d)
            if (L.c[i][d] != 0) u_bar[d] += cu_bar * L.c[i][d];
        usq_bar -= e * 1.5;
    }
    for (int d = 0; d < 3; ++d) u_bar[d] += usq_bar * u[d] * 2.0;
}

inline double group_rate(const orc_problem& o, int g) {
    switch (g) {
        case G_MASS:
        case G_SHEAR: return o.omega;
        case G_MOMENTUM:
        case G_ODD: return o.om;
        case G_BULK: return std::isnan(o.bulk_rate) ? o.omega : o.bulk_rate;
        default: return std::isnan(o.even_rate) ? o.omega : o.even_rate;
    }
}

// MRT relax / relax_transpose, moving/collision.rs:349-375, 409-425.
void mrt_relax(const orc_problem& o, const double* y, double* r) {
    const int Q = o.Q;
    const Basis& B = o.basis;
    double rm[27];
    for (int k = 0; k < Q; ++k) {
        double acc = 0;
        for (int i = 0; i < Q; ++i) acc += y[i] * B.rows[k * Q + i];
        rm[k] = acc * group_rate(o, B.groups[k]) / B.norms[k];
    }
    for (int i = 0; i < Q; ++i) {
        double acc = 0;
        for (int k = 0; k < Q; ++k) acc += rm[k] * B.rows[k * Q + i];
        r[i] = acc * o.L.w[i];
    }
}
void mrt_relax_transpose(const orc_problem& o, const double* g, double* r) {
    const int Q = o.Q;
    const Basis& B = o.basis;
    double sc[27];
    for (int k = 0; k < Q; ++k) {
        double acc = 0;
        for (int i = 0; i < Q; ++i) acc += g[i] * o.L.w[i] * B.rows[k * Q + i];
        sc[k] = acc * group_rate(o, B.groups[k]) / B.norms[k];
    }
    for (int i = 0; i < Q; ++i) {
        double acc = 0;
        for (int k = 0; k < Q; ++k) acc += sc[k] * B.rows[k * Q + i];
        r[i] = acc;
    }
}

inline void source_terms(const Lattice& L, const double u[3], const double F[3], double* src) {
    double uf = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
    for (int i = 0; i < L.Q; ++i) {
        double cu = dotc(L, i, u), cf = dotc(L, i, F);
        src[i] = (cf * 3.0 + cu * cf * 9.0 - uf * 3.0) * L.w[i];
    }
}

// Generic collide, moving/collision.rs:438-454 (MRT branch).
void collide_mrt(const orc_problem& o, const double* f, double rho, const double u[3], const double F[3],
                 double* out) {
    const int Q = o.Q;
    double eq[27], src[27], y[27], r[27];
    equilibrium(o.L, rho, u, eq);
    source_terms(o.L, u, F, src);
    for (int i = 0; i < Q; ++i) y[i] = f[i] - eq[i] + src[i] * 0.5;
    mrt_relax(o, y, r);
    for (int i = 0; i < Q; ++i) out[i] = f[i] - r[i] + src[i];
}

// Generic collide_vjp, moving/collision.rs:574-634 (no rate cotangent).
void collide_mrt_vjp(const orc_problem& o, const double* f, double rho, const double u[3], const double F[3],
                     const double* g, double* f_bar, double& rho_bar, double u_bar[3], double F_bar[3]) {
    const Lattice& L = o.L;
    const int Q = L.Q;
    (void)f;
    double rt[27];
    mrt_relax_transpose(o, g, rt);
    double src_bar[27];
    for (int i = 0; i < Q; ++i) {
        f_bar[i] = g[i] - rt[i];
        src_bar[i] = g[i] - rt[i] * 0.5;
    }
    rho_bar = 0;
    for (int d = 0; d < 3; ++d) u_bar[d] = F_bar[d] = 0;
    equilibrium_vjp(L, rho, u, rt, rho_bar, u_bar);
    double uf_bar = 0;
    for (int i = 0; i < Q; ++i) {
        double h = src_bar[i] * L.w[i];
        double cu = dotc(L, i, u), cf = dotc(L, i, F);
        double cf_bar = h * (cu * 9.0 + 3.0);
        double cu_bar = h * cf * 9.0;
        uf_bar -= h * 3.0;
        for (int d = 0; d < 3; ++d)
            if (L.c[i][d] != 0) {
                F_bar[d] += cf_bar * L.c[i][d];
                u_bar[d] += cu_bar * L.c[i][d];
            }
    }
    for (int d = 0; d < 3; ++d) {
        u_bar[d] += uf_bar * F[d];
        F_bar[d] += uf_bar * u[d];
    }
}

// One cell update: collide of the selected operator.
void collide_cell(const orc_problem& o, const double* f, double alpha, double* out, double tau) {
    if (o.coll == LBM_BGK) {
        collide_bgk(o, f, alpha, out, tau);
        return;
    }
    double rho, u[3], F[3];
    macroscopic(o, f, alpha, rho, u, F);
    if (o.coll == LBM_TRT) collide_pairs(o, f, rho, u, F, out);
    else collide_mrt(o, f, rho, u, F, out);
}

// Collision VJP with the Brinkman chain of moving/psm.rs cell_update_vjp
// (Brinkman branch, zero solid velocity, :402-486).
void collide_cell_vjp(const orc_problem& o, const double* f, double alpha, const double* g, double* f_bar,
                      double& alpha_bar, double tau, double& tau_bar) {
    tau_bar = 0;
    if (o.coll == LBM_BGK) {
        collide_bgk_vjp(o, f, alpha, g, f_bar, alpha_bar, tau, tau_bar);
        return;
    }
    const Lattice& L = o.L;
    const int Q = L.Q;
    double rho, j[3];
    moments(L, f, rho, j);
    double den = 1.0 + alpha * 0.5;
    double sv[3], u[3], F[3], z[3];
    for (int d = 0; d < 3; ++d) {
        sv[d] = j[d] / rho + o.a[d] * 0.5;
        u[d] = sv[d] / den;
    }
    for (int d = 0; d < 3; ++d) {
        z[d] = -alpha * u[d];
        F[d] = rho * (o.a[d] + z[d]);
    }
    double rho_bar, u_bar[3], F_bar[3];
    if (o.coll == LBM_TRT) collide_pairs_vjp(o, f, rho, u, F, g, f_bar, rho_bar, u_bar, F_bar);
    else collide_mrt_vjp(o, f, rho, u, F, g, f_bar, rho_bar, u_bar, F_bar);
    double a_bar = 0;
    for (int d = 0; d < 3; ++d) {
        rho_bar += F_bar[d] * (o.a[d] + z[d]);
        double zb = F_bar[d] * rho;
        a_bar -= zb * u[d];
        u_bar[d] -= zb * alpha;
    }
    double j_bar[3];
    for (int d = 0; d < 3; ++d) {
        double s_bar = u_bar[d] / den;
        a_bar -= u_bar[d] * sv[d] / (den * den) * 0.5;
        j_bar[d] = s_bar / rho;
        rho_bar -= s_bar * j[d] / (rho * rho);
    }
    for (int i = 0; i < Q; ++i) {
        double v = f_bar[i] + rho_bar;
        for (int d = 0; d < 3; ++d) v += j_bar[d] * L.c[i][d];
        f_bar[i] = v;
    }
    alpha_bar = a_bar;
}

// ---------------------------------------------------------------- stepping
// collide (solver.rs:324-328) + Streaming::stream (:131-136) + ports (ports.rs:560-579)
double interval(const orc_problem& o, const double* before, const double* alpha, double* after,
                std::vector<double>& post) {
    const int Q = o.Q;
    const int64_t N = o.N;
    post.resize((size_t)N * Q);
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < N; ++x) collide_cell(o, before + x * Q, alpha[x], post.data() + x * Q, tau_at(o, x));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N * Q; ++i) {
        uint32_t s = o.source[i];
        after[i] = s == NONE ? before[i] : post[s];
    }
    double exch = 0;
    for (const Port& p : o.ports) {
        for (int64_t cell : p.cells) {
            double vals[27];
            if (p.recon == 3) regularized_apply(o, p, after + cell * Q, vals);
            else if (p.recon) nee_apply(o, p, after + (cell + p.nb_off) * Q, vals);
            else reconstruct(o, p, after + cell * Q, vals);
            for (int q = 0; q < Q; ++q) {
                exch += vals[q] - after[cell * Q + q];
                after[cell * Q + q] = vals[q];
            }
        }
    }
    return exch;
}

// interval_vjp, solver.rs:642-674, with apply_ports_vjp (ports.rs:582-621)
// and Streaming::stream_vjp (solver.rs:138-157).
void interval_vjp(const orc_problem& o, const double* before, const double* alpha, const double* after_bar,
                  double* f_bar, double* alpha_bar, double* tau_bar = nullptr) {
    const int Q = o.Q;
    const int64_t N = o.N;
    std::vector<double> refl(after_bar, after_bar + N * Q);
    for (const Port& p : o.ports)
        for (int64_t cell : p.cells)
            for (int q = 0; q < Q; ++q) refl[cell * Q + q] = 0.0;
    // the extrapolating ports linearise at the neighbours' streamed
    // populations of the next state (reflected_cells, solver.rs:617-639)
    std::vector<double> streamed, post_tmp;
    bool any_nee = false;
    for (const Port& p : o.ports) any_nee = any_nee || p.recon != 0;
    if (any_nee) {
        streamed.resize((size_t)N * Q);
        interval(o, before, alpha, streamed.data(), post_tmp);
    }
    for (const Port& p : o.ports)
        for (int64_t cell : p.cells) {
            const double* g = after_bar + cell * Q;
            bool any = false;
            for (int r = 0; r < Q; ++r) any |= g[r] != 0.0;
            if (!any) continue;
            if (p.recon == 3) {
                double fb[27];
                regularized_vjp(o, p, streamed.data() + cell * Q, g, fb);
                for (int k = 0; k < Q; ++k) refl[cell * Q + k] += fb[k];
                continue;
            }
            if (p.recon) {
                double nb_bar[27];
                nee_vjp(o, p, streamed.data() + (cell + p.nb_off) * Q, g, nb_bar);
                for (int k = 0; k < Q; ++k) refl[(cell + p.nb_off) * Q + k] += nb_bar[k];
                continue;
            }
            for (int r = 0; r < Q; ++r) {
                if (g[r] == 0.0) continue;
                for (int k = 0; k < Q; ++k) refl[cell * Q + k] += p.jac[r * Q + k] * g[r];
            }
        }
    std::vector<double> post_bar((size_t)N * Q);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N * Q; ++i) {
        double acc = 0;
        uint32_t r0 = o.readers[2 * i], r1 = o.readers[2 * i + 1];
        if (r0 != NONE) acc += refl[r0];
        if (r1 != NONE) acc += refl[r1];
        post_bar[i] = acc;
    }
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < N; ++x) {
        double* fb = f_bar + x * Q;
        const double* g = post_bar.data() + x * Q;
        bool any = false;
        for (int q = 0; q < Q; ++q) any |= g[q] != 0.0;
        double ab = 0, tb = 0;
        if (any) {
            collide_cell_vjp(o, before + x * Q, alpha[x], g, fb, ab, tau_at(o, x), tb);
        } else {
            for (int q = 0; q < Q; ++q) fb[q] = 0.0;
        }
        if (o.solid[x])
            for (int q = 0; q < Q; ++q) fb[q] += refl[x * Q + q];
        if (alpha_bar) alpha_bar[x] = ab;
        if (tau_bar) tau_bar[x] = o.solid[x] ? 0.0 : tb;
    }
}

// ---------------------------------------------------------------- responses
struct Scales {
    double vel, dens, dt, dv, nfluid, visc;
};
inline Scales scales(const orc_problem& o) {
    Scales s;
    s.vel = o.dx / o.dt;
    s.dens = o.density;
    s.dt = o.dt;
    s.dv = o.dx * o.dx * o.dx;
    s.nfluid = (double)o.fluid_cells;
    s.visc = o.density * std::pow(o.dx, 5) / std::pow(o.dt, 3);
    return s;
}

// Viscous dissipation per cell in lattice units and its pieces.
struct Visc {
    double sigma[3][3];
    double phi;
};
inline Visc viscous(const orc_problem& o, const double* f, double rho, const double u[3], const double F[3]) {
    const Lattice& L = o.L;
    double M2[3][3] = {};
    for (int q = 0; q < L.Q; ++q)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) M2[a][b] += f[q] * L.c[q][a] * L.c[q][b];
    double k = 1.0 - 0.5 / o.tau;
    double nu = (o.tau - 0.5) / 3.0;
    Visc v;
    double ss = 0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double pi = M2[a][b] - rho * ((a == b ? 1.0 / 3.0 : 0.0) + u[a] * u[b]);
            double t = 0.5 * (u[a] * F[b] + u[b] * F[a]);
            v.sigma[a][b] = -k * (pi + t);
            ss += v.sigma[a][b] * v.sigma[a][b];
        }
    v.phi = ss / (2.0 * rho * nu);
    return v;
}

// vector_cell (solver.rs:835-856) extended with the pressure-drop and
// viscous-dissipation contributions; returns per-cell summands.
void vector_cell(const orc_problem& o, const Scales& s, int64_t x, const double* f, double alpha, double phi,
                 double c[8]) {
    for (int k = 0; k < 8; ++k) c[k] = 0;
    c[5] = phi;
    if (o.solid[x]) return;
    double rho, u[3], F[3];
    macroscopic(o, f, alpha, rho, u, F);
    double U[3] = {u[0] * s.vel, u[1] * s.vel, u[2] * s.vel};
    double R = rho * s.dens;
    double usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
    c[0] = U[0];
    c[1] = U[1];
    c[2] = U[2];
    c[3] = R * usq;
    c[4] = R * alpha / s.dt * usq;
    int role = o.port_role[x];
    if (role != 0) {
        double p = s.dens * (rho - 1.0) * s.vel * s.vel / 3.0;
        c[6] = role > 0 ? p / (double)o.n_inlet : -p / (double)o.n_outlet;
    }
    c[7] = viscous(o, f, rho, u, F).phi;
}

void vector(const orc_problem& o, const double* phi, const double* alpha, const double* f, double out[8]) {
    Scales s = scales(o);
    double sums[8] = {};
    for (int64_t x = 0; x < o.N; ++x) {
        double c[8];
        vector_cell(o, s, x, f + x * o.Q, alpha[x], phi[x], c);
        for (int k = 0; k < 8; ++k) sums[k] += c[k];
    }
    out[0] = sums[0] / s.nfluid;
    out[1] = sums[1] / s.nfluid;
    out[2] = sums[2] / s.nfluid;
    out[3] = 0.5 * sums[3] * s.dv;
    out[4] = sums[4] * s.dv;
    out[5] = sums[5] * s.dv;
    out[6] = (o.n_inlet > 0 && o.n_outlet > 0) ? sums[6] : 0.0;
    out[7] = sums[7] * s.visc;
}

// vector_vjp (solver.rs:896-947) by hand instead of forward-mode duals.
void vector_vjp(const orc_problem& o, const double* phi, const double* alpha, const double* f, const double w[8],
                double* f_bar, double* alpha_bar, double* phi_bar) {
    const Lattice& L = o.L;
    const int Q = L.Q;
    Scales s = scales(o);
    double W[8] = {w[0] / s.nfluid, w[1] / s.nfluid, w[2] / s.nfluid, 0.5 * w[3] * s.dv, w[4] * s.dv,
                   w[5] * s.dv,     (o.n_inlet > 0 && o.n_outlet > 0) ? w[6] : 0.0, w[7] * s.visc};
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < o.N; ++x) {
        double* fb = f_bar + x * Q;
        for (int q = 0; q < Q; ++q) fb[q] = 0;
        alpha_bar[x] = 0;
        phi_bar[x] = W[5];
        if (o.solid[x]) continue;
        const double* fx = f + x * Q;
        double al = alpha[x];
        double rho, m[3];
        moments(L, fx, rho, m);
        double sden = 1.0 + 0.5 * al;
        double u[3], F[3];
        for (int d = 0; d < 3; ++d) u[d] = (m[d] / rho + 0.5 * o.a[d]) / sden;
        for (int d = 0; d < 3; ++d) F[d] = rho * (o.a[d] - al * u[d]);
        double U[3] = {u[0] * s.vel, u[1] * s.vel, u[2] * s.vel};
        double usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
        double R = rho * s.dens;
        double rho_bar = 0, a_bar = 0, u_bar[3] = {0, 0, 0}, F_bar[3] = {0, 0, 0}, M2_bar[3][3] = {};
        for (int d = 0; d < 3; ++d) u_bar[d] += W[d] * s.vel;
        double kin = W[3] + W[4] * al / s.dt;
        for (int d = 0; d < 3; ++d) u_bar[d] += kin * R * 2.0 * U[d] * s.vel;
        rho_bar += kin * s.dens * usq;
        a_bar += W[4] * R / s.dt * usq;
        int role = o.port_role[x];
        if (role != 0 && W[6] != 0.0) {
            double dp = s.dens * s.vel * s.vel / 3.0;
            rho_bar += W[6] * (role > 0 ? dp / (double)o.n_inlet : -dp / (double)o.n_outlet);
        }
        if (W[7] != 0.0) {
            Visc v = viscous(o, fx, rho, u, F);
            double k = 1.0 - 0.5 / o.tau;
            double nu = (o.tau - 0.5) / 3.0;
            double ss = 0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) ss += v.sigma[a][b] * v.sigma[a][b];
            rho_bar += -W[7] * ss / (2.0 * rho * rho * nu);
            double sb[3][3];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) sb[a][b] = W[7] * v.sigma[a][b] / (rho * nu);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    double pb = -k * sb[a][b];  // Pi_bar == T_bar
                    M2_bar[a][b] += pb;
                    rho_bar -= pb * ((a == b ? 1.0 / 3.0 : 0.0) + u[a] * u[b]);
                    u_bar[a] -= rho * pb * u[b];
                    u_bar[b] -= rho * pb * u[a];
                    u_bar[a] += 0.5 * pb * F[b];
                    u_bar[b] += 0.5 * pb * F[a];
                    F_bar[b] += 0.5 * pb * u[a];
                    F_bar[a] += 0.5 * pb * u[b];
                }
        }
        for (int d = 0; d < 3; ++d) {
            rho_bar += F_bar[d] * (o.a[d] - al * u[d]);
            a_bar -= F_bar[d] * rho * u[d];
            u_bar[d] -= F_bar[d] * rho * al;
        }
        double m_bar[3], s_bar = 0;
        for (int d = 0; d < 3; ++d) {
            m_bar[d] = u_bar[d] / (sden * rho);
            rho_bar -= u_bar[d] * m[d] / (sden * rho * rho);
            s_bar -= u_bar[d] * u[d] / sden;
        }
        a_bar += 0.5 * s_bar;
        for (int q = 0; q < Q; ++q) {
            double v = rho_bar;
            for (int d = 0; d < 3; ++d) v += m_bar[d] * L.c[q][d];
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) v += M2_bar[a][b] * L.c[q][a] * L.c[q][b];
            fb[q] = v;
        }
        alpha_bar[x] = a_bar;
    }
}

// ---------------------------------------------------------------- design map
double filtered(const orc_problem& o, const double* raw, int64_t x) {
    if (!o.filtered) return raw[x];
    double num = 0;
    for (auto& t : o.rows[x].terms) num += t.second * raw[t.first];
    return num / o.den[x];
}

void design_map(const orc_problem& o, const double* raw, double* phi) {
    bool proj = o.beta > 0;
    double pa = 0, pden = 1;
    if (proj) {
        pa = std::tanh(o.beta * o.eta);
        pden = pa + std::tanh(o.beta * (1.0 - o.eta));
    }
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < o.N; ++x) {
        if (o.solid[x]) phi[x] = 0.0;
        else if (o.editable[x]) {
            double f = filtered(o, raw, x);
            phi[x] = proj ? (pa + std::tanh(o.beta * (f - o.eta))) / pden : f;
        } else phi[x] = o.fixed[x];
    }
}

// DesignMap::vjp, design.rs:219-243
void design_vjp(const orc_problem& o, const double* raw, const double* phi_bar, double* out) {
    bool proj = o.beta > 0;
    double pden = 1;
    if (proj) pden = std::tanh(o.beta * o.eta) + std::tanh(o.beta * (1.0 - o.eta));
    for (int64_t x = 0; x < o.N; ++x) out[x] = 0;
    for (int64_t x = 0; x < o.N; ++x) {
        if (!o.editable[x] || phi_bar[x] == 0.0) continue;
        double g = phi_bar[x];
        if (proj) {
            double t = std::tanh(o.beta * (filtered(o, raw, x) - o.eta));
            g *= o.beta * (1.0 - t * t) / pden;
        }
        if (!o.filtered) out[x] += g;
        else {
            double scale = g / o.den[x];
            for (auto& t : o.rows[x].terms) out[t.first] += t.second * scale;
        }
    }
}

void initial(const orc_problem& o, double* f) {
    const Lattice& L = o.L;
    double fluid[27];
    for (int q = 0; q < L.Q; ++q) fluid[q] = L.w[q] - 1.5 * L.w[q] * dotc(L, q, o.a);
    for (int64_t x = 0; x < o.N; ++x)
        for (int q = 0; q < L.Q; ++q) f[x * L.Q + q] = o.solid[x] ? L.w[q] : fluid[q];
}

// Per-state admission quantities (solver.rs:714-755).
void state_stats(const orc_problem& o, const double* f, const double* alpha, double& mass, double& minimum,
                 double& worst, bool& finite) {
    const int Q = o.Q;
    double m = 0, mn = INFINITY, wv = 0;
    bool fin = true;
#pragma omp parallel for reduction(+ : m) reduction(min : mn) reduction(max : wv) reduction(&& : fin)
    for (int64_t x = 0; x < o.N; ++x) {
        const double* fx = f + x * Q;
        for (int q = 0; q < Q; ++q) fin = fin && std::isfinite(fx[q]);
        if (o.solid[x]) continue;
        for (int q = 0; q < Q; ++q) mn = std::min(mn, fx[q]);
        double rho, u[3], F[3];
        macroscopic(o, fx, alpha[x], rho, u, F);
        wv = std::max(wv, std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        m += rho;
    }
    mass = m;
    minimum = mn;
    worst = wv;
    finite = fin;
}

}  // namespace

// ==================================================================== C ABI
extern "C" {

const char* orc_error(void) { return g_error.c_str(); }
void orc_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
}
int orc_threads(void) { return omp_get_max_threads(); }

int orc_mrt_basis(int q, double* rows, double* norms, int32_t* groups) {
    Lattice L = make_lattice(q);
    Basis B;
    if (!make_basis(L, B)) return 1;
    for (int i = 0; i < q * q; ++i) rows[i] = B.rows[i];
    for (int i = 0; i < q; ++i) {
        norms[i] = B.norms[i];
        groups[i] = B.groups[i];
    }
    return 0;
}

int orc_create(const lbm_problem_t* p, orc_problem** out) {
    *out = nullptr;
    if (p->lattice != 19 && p->lattice != 27) {
        g_error = "lattice must be 19 or 27";
        return 1;
    }
    auto* o = new orc_problem();
    o->L = make_lattice(p->lattice);
    o->Q = p->lattice;
    o->coll = p->collision;
    for (int a = 0; a < 3; ++a) {
        o->shape[a] = p->shape[a];
        o->periodic[a] = p->periodic_axes[a] != 0;
    }
    o->N = o->shape[0] * o->shape[1] * o->shape[2];
    o->dx = p->spacing_m;
    o->dt = p->step_s;
    o->density = p->density_kg_m3;
    o->nu = p->kinematic_viscosity_m2_s;
    o->tau = 0.5 + 3.0 * o->nu * o->dt / (o->dx * o->dx);  // solver.rs:490
    for (int d = 0; d < 3; ++d) o->a[d] = p->acceleration_m_s2[d] * o->dt * o->dt / o->dx;
    o->drag_max = p->drag_max_per_s;
    o->drag_shape = p->drag_shape;
    o->mach_limit = p->mach_limit;
    const int64_t N = o->N;
    o->solid.assign(p->solid_mask, p->solid_mask + N);
    o->editable.resize(N);
    for (int64_t x = 0; x < N; ++x) o->editable[x] = p->design_region[x] && !p->solid_mask[x];
    o->fixed.assign(p->fixed_design, p->fixed_design + N);
    o->fluid_cells = 0;
    for (int64_t x = 0; x < N; ++x) o->fluid_cells += o->solid[x] ? 0 : 1;
    // DesignMap::new (design.rs:109-171), box filter as the documented extension
    o->beta = p->projection_beta;
    o->eta = p->projection_eta;
    o->den.assign(N, 1.0);
    std::vector<std::pair<std::array<int64_t, 3>, double>> offsets;
    if (p->filter_kind == LBM_FILTER_BOX) {
        int h = p->box_half_width;
        if (h > 0)
            for (int a = -h; a <= h; ++a)
                for (int b = -h; b <= h; ++b)
                    for (int c = -h; c <= h; ++c) offsets.push_back({{a, b, c}, 1.0});
    } else {
        double radius = p->filter_radius_m / o->dx;
        if (radius > 0) {
            int64_t reach = (int64_t)std::ceil(radius);
            for (int64_t a = -reach; a <= reach; ++a)
                for (int64_t b = -reach; b <= reach; ++b)
                    for (int64_t c = -reach; c <= reach; ++c) {
                        double norm = std::sqrt((double)(a * a + b * b + c * c));
                        double wgt = std::max(radius - norm, 0.0);
                        if (wgt != 0.0) offsets.push_back({{a, b, c}, wgt});
                    }
        }
    }
    if (!offsets.empty()) {
        o->filtered = true;
        o->rows.resize(N);
        for (int64_t x = 0; x < N; ++x) {
            double den = 0;
            for (auto& of : offsets) {
                int64_t back[3] = {-of.first[0], -of.first[1], -of.first[2]};
                if (!inside(*o, x, back)) continue;
                int64_t src = wrap(*o, x, back);
                if (!o->editable[src]) continue;
                o->rows[x].terms.push_back({src, of.second});
                den += of.second;
            }
            o->den[x] = den > 0 ? den : 1.0;
        }
    }
    // Streaming::new (solver.rs:84-119)
    const int Q = o->Q;
    o->blocked.assign(N * Q, 0);
    for (int64_t x = 0; x < N; ++x)
        for (int q = 0; q < Q; ++q) {
            int64_t back[3] = {-o->L.c[q][0], -o->L.c[q][1], -o->L.c[q][2]};
            o->blocked[x * Q + q] = o->solid[wrap(*o, x, back)] || !inside(*o, x, back);
        }
    o->source.assign(N * Q, NONE);
    o->readers.assign(N * Q * 2, NONE);
    for (int64_t x = 0; x < N; ++x) {
        if (o->solid[x]) continue;
        for (int q = 0; q < Q; ++q) {
            int64_t from;
            if (o->blocked[x * Q + q]) from = x * Q + o->L.opp[q];
            else {
                int64_t back[3] = {-o->L.c[q][0], -o->L.c[q][1], -o->L.c[q][2]};
                from = wrap(*o, x, back) * Q + q;
            }
            o->source[x * Q + q] = (uint32_t)from;
            uint32_t* slot = &o->readers[2 * from];
            if (slot[0] == NONE) slot[0] = (uint32_t)(x * Q + q);
            else slot[1] = (uint32_t)(x * Q + q);
        }
    }
    // collision rates (moving/collision.rs:302-305)
    o->omega = 1.0 / o->tau;
    double magic = p->collision == LBM_MRT ? p->mrt_odd_magic : p->trt_magic;
    if (std::isnan(magic)) magic = 3.0 / 16.0;
    double tp = 1.0 / o->omega - 0.5;
    o->om = p->collision == LBM_BGK ? o->omega : 1.0 / (0.5 + magic / tp);
    o->bulk_rate = p->mrt_bulk_rate;
    o->even_rate = p->mrt_even_rate;
    if (p->collision == LBM_MRT && !make_basis(o->L, o->basis)) {
        g_error = "MRT moment basis incomplete";
        delete o;
        return 1;
    }
    // ports (ports.rs:106-272 normalisation, CompiledPort::new :509-521)
    o->port_role.assign(N, 0);
    double unit = o->dx / o->dt;
    o->pressure_unit = 3.0 / (o->density * unit * unit);
    for (int k = 0; k < p->n_ports; ++k) {
        const lbm_port_t& src = p->ports[k];
        Port pt;
        pt.pressure = src.kind == LBM_PORT_PRESSURE;
        pt.axis = src.face / 2;
        pt.sign = (src.face % 2 == 0) ? 1 : -1;
        for (int d = 0; d < 3; ++d) pt.vel[d] = src.velocity_m_s[d] * o->dt / o->dx;
        if (pt.pressure) pt.density = 1.0 + src.gauge_pressure_Pa * 3.0 / (o->density * unit * unit);
        for (int d = 0; d < 3; ++d) {
            pt.mean_vel[d] = pt.vel[d];
            pt.amp_vel[d] = pt.pressure ? 0.0 : src.amplitude_m_s[d] * o->dt / o->dx;
        }
        pt.mean_p = pt.pressure ? src.gauge_pressure_Pa : 0.0;
        pt.amp_p = pt.pressure ? src.amplitude_Pa : 0.0;
        pt.freq = src.frequency_hz;
        pt.phase = src.phase_rad;
        pt.ramp = src.ramp_s;
        pt.pulsatile = pt.freq != 0.0 || pt.ramp != 0.0;
        for (int64_t x = 0; x < N; ++x)
            if (src.mask[x]) pt.cells.push_back(x);
        pt.recon = src.reconstruction;
        const int64_t stride[3] = {o->shape[1] * o->shape[2], o->shape[2], 1};
        pt.nb_off = pt.sign * stride[pt.axis];
        port_jacobian(*o, pt);
        if (pt.recon == 3 && !regularized_operator(o->L, pt)) {
            g_error = "Regularized port stress fit is rank deficient or ill conditioned";
            delete o;
            return 1;
        }
        for (int64_t x : pt.cells) o->port_role[x] = pt.pressure ? -1 : 1;
        if (pt.pressure) o->n_outlet += (int64_t)pt.cells.size();
        else o->n_inlet += (int64_t)pt.cells.size();
        o->ports.push_back(std::move(pt));
    }
    *out = o;
    return 0;
}

void orc_destroy(orc_problem* o) { delete o; }

void orc_info(const orc_problem* o, int64_t* cells, int32_t* q, double* tau, double* a_lattice,
              int64_t* fluid_cells) {
    if (cells) *cells = o->N;
    if (q) *q = o->Q;
    if (tau) *tau = o->tau;
    if (a_lattice)
        for (int d = 0; d < 3; ++d) a_lattice[d] = o->a[d];
    if (fluid_cells) *fluid_cells = o->fluid_cells;
}

void orc_design(const orc_problem* o, const double* raw, double* phi, double* alpha) {
    std::vector<double> tmp;
    double* ph = phi;
    if (!ph) {
        tmp.resize(o->N);
        ph = tmp.data();
    }
    design_map(*o, raw, ph);
    if (alpha)
        for (int64_t x = 0; x < o->N; ++x) alpha[x] = resistance(*o, ph[x]);
}

void orc_design_vjp(const orc_problem* o, const double* raw, const double* phi_bar, double* out) {
    design_vjp(*o, raw, phi_bar, out);
}

void orc_resistance_derivative(const orc_problem* o, const double* phi, double* out) {
    for (int64_t x = 0; x < o->N; ++x) out[x] = resistance_derivative(*o, phi[x]);
}

void orc_initial(const orc_problem* o, double* f) { initial(*o, f); }

double orc_interval(const orc_problem* o, const double* before, const double* alpha, double* after) {
    std::vector<double> post;
    return interval(*o, before, alpha, after, post);
}

void orc_history_trace(const orc_problem* o, const double* alpha, int64_t steps, double* final_state,
                       orc_diag_t* diag, double* mass_out, double* exch_out);

void orc_history(const orc_problem* o, const double* alpha, int64_t steps, double* final_state,
                 orc_diag_t* diag) {
    orc_history_trace(o, alpha, steps, final_state, diag, nullptr, nullptr);
}

void orc_history_trace(const orc_problem* o, const double* alpha, int64_t steps, double* final_state,
                       orc_diag_t* diag, double* mass_out, double* exch_out) {
    const int64_t NQ = o->N * o->Q;
    std::vector<double> a(NQ), b(NQ), post;
    initial(*o, a.data());
    std::vector<double> mass((size_t)steps + 1), changes((size_t)steps);
    double minimum = INFINITY, mach = 0;
    bool finite = true;
    for (int64_t t = 0; t <= steps; ++t) {
        double m, mn, wv;
        bool fin;
        state_stats(*o, a.data(), alpha, m, mn, wv, fin);
        mass[t] = m;
        minimum = std::min(minimum, mn);
        mach = std::max(mach, wv);
        finite = finite && fin;
        if (t == steps) break;
        set_port_time(*o, t + 1);
        changes[t] = interval(*o, a.data(), alpha, b.data(), post);
        std::swap(a, b);
    }
    mach *= std::sqrt(3.0);
    bool use_changes = !o->ports.empty();
    double err = 0, cum = 0, total = 0;
    for (int64_t t = 0; t <= steps; ++t) {
        if (t > 0 && use_changes) cum += changes[t - 1];
        err = std::max(err, std::fabs(mass[t] - (mass[0] + cum)));
    }
    for (int64_t t = 0; t < steps; ++t) total += changes[t];
    err /= mass[0];
    if (diag) {
        diag->maximum_mach = mach;
        diag->relative_mass_drift = err;
        diag->minimum_population = minimum;
        diag->boundary_exchange_total = use_changes ? total : 0.0;
        diag->nonfinite = finite ? 0 : 1;
        diag->admitted = (finite && minimum > 0 && mach <= o->mach_limit && err <= 1e-6) ? 1 : 0;
    }
    if (final_state) std::memcpy(final_state, a.data(), sizeof(double) * NQ);
    for (int64_t t = 0; t <= steps; ++t) {
        if (mass_out) mass_out[t] = mass[t];
        if (exch_out) exch_out[t] = t == 0 ? 0.0 : changes[t - 1];
    }
}

void orc_vector(const orc_problem* o, const double* phi, const double* alpha, const double* f, double* out8) {
    vector(*o, phi, alpha, f, out8);
}

void orc_vector_vjp(const orc_problem* o, const double* phi, const double* alpha, const double* f,
                    const double* w8, double* f_bar, double* alpha_bar, double* phi_bar) {
    vector_vjp(*o, phi, alpha, f, w8, f_bar, alpha_bar, phi_bar);
}

void orc_interval_vjp(const orc_problem* o, const double* before, const double* alpha,
                      const double* after_bar, double* f_bar, double* alpha_bar) {
    interval_vjp(*o, before, alpha, after_bar, f_bar, alpha_bar);
}

void orc_interval_vjp_tau(const orc_problem* o, const double* before, const double* alpha,
                          const double* after_bar, double* f_bar, double* alpha_bar, double* tau_bar) {
    interval_vjp(*o, before, alpha, after_bar, f_bar, alpha_bar, tau_bar);
}

int orc_set_tau(orc_problem* o, const double* tau) {
    if (!tau) {
        o->tau_cell.clear();
        return 0;
    }
    if (o->coll != LBM_BGK) return 1;
    o->tau_cell.assign(tau, tau + o->N);
    return 0;
}

void orc_set_time(const orc_problem* o, int64_t t_index) { set_port_time(*o, t_index); }

// ---------------------------------------------------------------- cell ranges
// The pieces of interval (solver.rs:604-614) and interval_vjp (:642-674)
// restricted to the cells [c0, c1), for x-slab domain decomposition checks:
// each call reads only the slots the restricted computation needs, so
// arrays that hold NaN outside a slab and its exchanged halo show every slot
// the decomposition fails to provide.
void orc_collide_range(const orc_problem* o, const double* before, const double* alpha, double* post, int64_t c0,
                       int64_t c1) {
    const int Q = o->Q;
#pragma omp parallel for schedule(static)
    for (int64_t x = c0; x < c1; ++x) collide_cell(*o, before + x * Q, alpha[x], post + x * Q, tau_at(*o, x));
}

void orc_stream_range(const orc_problem* o, const double* post, const double* before, double* after, int64_t c0,
                      int64_t c1) {
    const int Q = o->Q;
#pragma omp parallel for schedule(static)
    for (int64_t i = c0 * Q; i < c1 * Q; ++i) {
        const uint32_t s = o->source[i];
        after[i] = s == NONE ? before[i] : post[s];
    }
}

double orc_ports_range(const orc_problem* o, double* after, int64_t c0, int64_t c1) {
    const int Q = o->Q;
    double exch = 0;
    for (const Port& p : o->ports)
        for (int64_t cell : p.cells) {
            if (cell < c0 || cell >= c1) continue;
            double vals[27];
            reconstruct(*o, p, after + cell * Q, vals);
            for (int q = 0; q < Q; ++q) {
                exch += vals[q] - after[cell * Q + q];
                after[cell * Q + q] = vals[q];
            }
        }
    return exch;
}

// refl = apply_ports_vjp of after_bar on the cells [c0, c1)
void orc_ports_vjp_range(const orc_problem* o, const double* after_bar, double* refl, int64_t c0, int64_t c1) {
    const int Q = o->Q;
    for (int64_t i = c0 * Q; i < c1 * Q; ++i) refl[i] = after_bar[i];
    for (const Port& p : o->ports)
        for (int64_t cell : p.cells)
            if (cell >= c0 && cell < c1)
                for (int q = 0; q < Q; ++q) refl[cell * Q + q] = 0.0;
    for (const Port& p : o->ports)
        for (int64_t cell : p.cells) {
            if (cell < c0 || cell >= c1) continue;
            const double* g = after_bar + cell * Q;
            for (int r = 0; r < Q; ++r) {
                if (g[r] == 0.0) continue;
                for (int k = 0; k < Q; ++k) refl[cell * Q + k] += p.jac[r * Q + k] * g[r];
            }
        }
}

// post_bar of the slots of the cells [c0, c1): Streaming::stream_vjp (solver.rs:138-157)
void orc_stream_vjp_range(const orc_problem* o, const double* refl, double* post_bar, int64_t c0, int64_t c1) {
    const int Q = o->Q;
#pragma omp parallel for schedule(static)
    for (int64_t i = c0 * Q; i < c1 * Q; ++i) {
        double acc = 0;
        const uint32_t r0 = o->readers[2 * i], r1 = o->readers[2 * i + 1];
        if (r0 != NONE) acc += refl[r0];
        if (r1 != NONE) acc += refl[r1];
        post_bar[i] = acc;
    }
}

// f_bar and alpha_bar of the cells [c0, c1) from post_bar (collide_vjp) plus the
// pass-through of solid cells' own slots (previous_bar)
void orc_collide_vjp_range(const orc_problem* o, const double* before, const double* alpha, const double* post_bar,
                           const double* refl, double* f_bar, double* alpha_bar, int64_t c0, int64_t c1) {
    const int Q = o->Q;
#pragma omp parallel for schedule(static)
    for (int64_t x = c0; x < c1; ++x) {
        double* fb = f_bar + x * Q;
        const double* g = post_bar + x * Q;
        bool any = false;
        for (int q = 0; q < Q; ++q) any |= g[q] != 0.0;
        double ab = 0, tb = 0;
        if (any) collide_cell_vjp(*o, before + x * Q, alpha[x], g, fb, ab, tau_at(*o, x), tb);
        else
            for (int q = 0; q < Q; ++q) fb[q] = 0.0;
        if (o->solid[x])
            for (int q = 0; q < Q; ++q) fb[q] += refl[x * Q + q];
        alpha_bar[x] = ab;
    }
}

// Fixed-wall momentum-exchange loads (wall_exchange.rs: layout :44-70, loads
// :79-84, loads_from_post :86-100): `before` is collided with the Guo-BGK
// collision; for every blocked pull link q of a fluid cell (cells, then
// links, in order) that is not a port cell's link along its port's inward
// normal, force = -2 c_q (post_opp(q) - w_q + w_q datum / unit) scale.
// Returns the number of links; forces (3 per link) when not NULL.
int64_t orc_wall_loads(const orc_problem* o, const double* before, const double* alpha, double datum_pa,
                       double* forces) {
    const int Q = o->Q;
    const Lattice& L = o->L;
    std::vector<int> port_of(o->N, -1);
    for (size_t k = 0; k < o->ports.size(); ++k)
        for (int64_t x : o->ports[k].cells) port_of[x] = (int)k;
    const double scale = o->density * std::pow(o->dx, 4) / (o->dt * o->dt);
    const double unit = o->density * (o->dx / o->dt) * (o->dx / o->dt) / 3.0;
    int64_t n = 0;
    std::vector<double> post(Q);
    for (int64_t x = 0; x < o->N; ++x) {
        if (o->solid[x]) continue;
        bool collided = false;
        for (int q = 0; q < Q; ++q) {
            if (!o->blocked[x * Q + q]) continue;
            const int k = port_of[x];
            if (k >= 0 && L.c[q][o->ports[k].axis] == o->ports[k].sign) continue;
            if (forces) {
                if (!collided) {
                    collide_bgk(*o, before + x * Q, alpha[x], post.data(), tau_at(*o, x));
                    collided = true;
                }
                const double mag = post[L.opp[q]] - L.w[q] + L.w[q] * datum_pa / unit;
                for (int a = 0; a < 3; ++a) forces[3 * n + a] = -2.0 * L.c[q][a] * mag * scale;
            }
            ++n;
        }
    }
    return n;
}

void orc_port_apply(const orc_problem* o, int port, const double* f_in, double* f_out) {
    // the extrapolating reconstructions read the inward neighbour's populations
    if (o->ports[port].recon == 3) regularized_apply(*o, o->ports[port], f_in, f_out);
    else if (o->ports[port].recon) nee_apply(*o, o->ports[port], f_in, f_out);
    else reconstruct(*o, o->ports[port], f_in, f_out);
}

int orc_gradient(const orc_problem* o, const double* raw, const double* w8, int64_t steps, int mode, int64_t K,
                 double tol, int64_t max_iter, double* grad, double* responses8, orc_grad_report_t* report) {
    const int64_t N = o->N;
    const int64_t NQ = N * o->Q;
    std::vector<double> phi(N), alpha(N), dres(N);
    design_map(*o, raw, phi.data());
    for (int64_t x = 0; x < N; ++x) {
        alpha[x] = resistance(*o, phi[x]);
        dres[x] = resistance_derivative(*o, phi[x]);
    }
    if (K <= 0 || K > steps) K = steps > 0 ? steps : 1;
    // forward with Every(K) checkpoints (scan.rs:181-196)
    std::vector<std::pair<int64_t, std::vector<double>>> ckpt;
    std::vector<double> x(NQ), nx(NQ), post;
    initial(*o, x.data());
    ckpt.push_back({0, x});
    int64_t evals = 0;
    // mode 2: the weighted responses averaged over the states 1..steps (a
    // stage objective: every state seeds the adjoint with weights w/steps)
    const bool stage = mode == 2;
    double ws[8], avg[8] = {0, 0, 0, 0, 0, 0, 0, 0}, r8[8];
    for (int k = 0; k < 8; ++k) ws[k] = stage ? w8[k] / (double)steps : w8[k];
    for (int64_t t = 0; t < steps; ++t) {
        set_port_time(*o, t + 1);
        interval(*o, x.data(), alpha.data(), nx.data(), post);
        ++evals;
        std::swap(x, nx);
        if ((t + 1) % K == 0 && t + 1 < steps) ckpt.push_back({t + 1, x});
        if (stage) {
            vector(*o, phi.data(), alpha.data(), x.data(), r8);
            for (int k = 0; k < 8; ++k) avg[k] += r8[k] / (double)steps;
        }
    }
    if (stage) std::memcpy(responses8, avg, sizeof(avg));
    else vector(*o, phi.data(), alpha.data(), x.data(), responses8);
    std::vector<double> lam(NQ), abar_final(N), phibar(N), abar(N, 0.0), fb(NQ), ab(N);
    vector_vjp(*o, phi.data(), alpha.data(), x.data(), ws, lam.data(), abar_final.data(), phibar.data());
    std::vector<double> sf(NQ), sa(N), sp(N);
    int status = 0;
    int64_t iters = 0;
    double resid = 0;
    if (mode == 0 || mode == 2) {
        while (!ckpt.empty()) {
            auto [start, xs] = std::move(ckpt.back());
            ckpt.pop_back();
            int64_t end = std::min(start + K, steps);
            std::vector<std::vector<double>> states;
            states.push_back(std::move(xs));
            for (int64_t t = start; t + 1 < end; ++t) {
                std::vector<double> nxt(NQ);
                set_port_time(*o, t + 1);
                interval(*o, states.back().data(), alpha.data(), nxt.data(), post);
                ++evals;
                states.push_back(std::move(nxt));
            }
            for (int64_t t = end - 1; t >= start; --t) {
                set_port_time(*o, t + 1);
                interval_vjp(*o, states[t - start].data(), alpha.data(), lam.data(), fb.data(), ab.data());
                for (int64_t c = 0; c < N; ++c) abar[c] += ab[c];
                std::swap(lam, fb);
                ++iters;
                if (stage && t >= 1) {
                    // the stage seed of state t
                    vector_vjp(*o, phi.data(), alpha.data(), states[t - start].data(), ws, sf.data(), sa.data(),
                               sp.data());
                    for (int64_t i = 0; i < NQ; ++i) lam[i] += sf[i];
                    for (int64_t c = 0; c < N; ++c) {
                        abar[c] += sa[c];
                        phibar[c] += sp[c];
                    }
                }
            }
        }
    } else {
        auto norm = [&](const std::vector<double>& v) {
            double s = 0;
            for (double e : v) s += e * e;
            return std::sqrt(s);
        };
        set_port_time(*o, steps);
        double n0 = norm(lam);
        status = 2;
        if (n0 == 0) status = 0;
        while (status != 0 && iters < max_iter) {
            interval_vjp(*o, x.data(), alpha.data(), lam.data(), fb.data(), ab.data());
            for (int64_t c = 0; c < N; ++c) abar[c] += ab[c];
            std::swap(lam, fb);
            ++iters;
            resid = norm(lam) / n0;
            if (resid <= tol) status = 0;
        }
    }
    for (int64_t c = 0; c < N; ++c) phibar[c] += (abar[c] + abar_final[c]) * dres[c];
    design_vjp(*o, raw, phibar.data(), grad);
    if (report) {
        report->iterations = iters;
        report->forward_evaluations = evals;
        report->residual = resid;
    }
    return status;
}

}  // extern "C"
