// mma_cpu.cpp -- Method of Moving Asymptotes on the host CPU (include/mma_cpu.h).
//
// Restates MmaOptimizer::step of the reference optimiser (crates/
// implexity-optim/src/mma.rs) for large design vectors: the n-sized work of
// every interior-point Newton step runs as a few fused OpenMP passes (the
// per-variable terms are recomputed from x, the asymptotes and the p/q
// coefficients instead of being stored), and only the (m+1)-sized reduced
// system is dense.  Variables and formulas follow the reference names
// (xsi, eta, mu, zet, s, epsi, ...).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mma_cpu.h"

namespace {

thread_local std::string g_err;

struct ContractError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct RuntimeError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

using Vec = std::vector<double>;

// Dense solve with partial pivoting (the reduced Newton system, m+1 sized).
Vec dense_solve(Vec a, int dim, Vec b) {
    for (int k = 0; k < dim; ++k) {
        int piv = k;
        for (int r = k + 1; r < dim; ++r)
            if (std::fabs(a[(size_t)r * dim + k]) > std::fabs(a[(size_t)piv * dim + k])) piv = r;
        if (!(std::fabs(a[(size_t)piv * dim + k]) > 0.0)) throw RuntimeError("Singular matrix: zero pivot");
        if (piv != k) {
            for (int c = 0; c < dim; ++c) std::swap(a[(size_t)k * dim + c], a[(size_t)piv * dim + c]);
            std::swap(b[k], b[piv]);
        }
        for (int r = k + 1; r < dim; ++r) {
            const double f = a[(size_t)r * dim + k] / a[(size_t)k * dim + k];
            if (f == 0.0) continue;
            for (int c = k; c < dim; ++c) a[(size_t)r * dim + c] -= f * a[(size_t)k * dim + c];
            b[r] -= f * b[k];
        }
    }
    Vec x(dim);
    for (int k = dim - 1; k >= 0; --k) {
        double s = b[k];
        for (int c = k + 1; c < dim; ++c) s -= a[(size_t)k * dim + c] * x[c];
        x[k] = s / a[(size_t)k * dim + k];
    }
    return x;
}

bool all_finite(const double* v, size_t n) {
    bool ok = true;
#pragma omp parallel for reduction(&& : ok) schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) ok = ok && std::isfinite(v[i]);
    return ok;
}

}  // namespace

struct mma_handle {
    int64_t n = 0, m = 0;
    mma_options_t o{};
    Vec a, c, d, x_min, x_max, xmami;
    Vec low, upp;  // asymptotes L, U (empty until the first step)
    int64_t iter = 0;
    double last_kkt = std::numeric_limits<double>::infinity();
    Vec lam, y;
    double z = 0.0;
    bool ip_converged = true;
    double ip_last_residual = 0.0;
    int64_t newton_steps = 0;
    std::string err;
    // --- GCMMA (MmaOptimizer::gcmma, mma.rs:339-355; GcmmaState :242-248)
    bool gcmma = false;
    mma_gcmma_options_t g{};
    int64_t nonfinite_trials = 0;
    Vec rho_last;  // rho0 then rho of the last step

    // --- subproblem data (Sub, mma.rs:180-188)
    Vec p0, q0, P, Q, alpha, beta, b;
    // --- interior-point variables (Vars, mma.rs:190-201) and work arrays
    Vec x, xsi, eta, mu, s;
    double zv = 1.0, zet = 1.0;
    Vec ox, oxsi, oeta, dx, dxsi, deta, delx, diagx;

    double natural_residual(const double* xx, const double* yy, double zz, const double* ll, const double* grad,
                            const double* g, const double* lo, const double* hi) const;
    void asymptote_update(const double* xk, const double* xkm1, const double* xkm2);
    void ip_residual(double epsi, double& norm, double& maxabs) const;
    void solve_subproblem();
    double sub_kkt() const;
};

// natural_residual (mma.rs:443-476): the max-norm of the projected-gradient
// residuals of x, y, z and lambda.
double mma_handle::natural_residual(const double* xx, const double* yy, double zz, const double* ll,
                                    const double* grad, const double* g, const double* lo, const double* hi) const {
    double rx = 0.0;
#pragma omp parallel for reduction(max : rx) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double r = xx[i] - std::min(std::max(xx[i] - grad[i], lo[i]), hi[i]);
        rx = std::max(rx, std::fabs(r));
    }
    double al = 0.0;
    for (int64_t j = 0; j < m; ++j) al += a[j] * ll[j];
    double out = std::max(rx, std::fabs(zz - std::max(0.0, zz - (o.a0 - al))));
    for (int64_t j = 0; j < m; ++j) {
        out = std::max(out, std::fabs(yy[j] - std::max(0.0, yy[j] - (c[j] + d[j] * yy[j] - ll[j]))));
        out = std::max(out, std::fabs(ll[j] - std::max(0.0, ll[j] + g[j])));
    }
    return out;
}

// asymptote_update (mma.rs:522-553).
void mma_handle::asymptote_update(const double* xk, const double* xkm1, const double* xkm2) {
    if (iter < 2 || low.empty()) {
        low.resize(n);
        upp.resize(n);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            const double span = x_max[i] - x_min[i];
            low[i] = xk[i] - o.asymptote_init * span;
            upp[i] = xk[i] + o.asymptote_init * span;
        }
        return;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double span = x_max[i] - x_min[i];
        const double zzz = (xk[i] - xkm1[i]) * (xkm1[i] - xkm2[i]);
        const double f = zzz > 0.0 ? o.asymptote_expand : zzz < 0.0 ? o.asymptote_contract : 1.0;
        double lo = xk[i] - f * (xkm1[i] - low[i]);
        double up = xk[i] + f * (upp[i] - xkm1[i]);
        lo = std::max(lo, xk[i] - o.asymptote_hi * span);
        lo = std::min(lo, xk[i] - o.asymptote_lo * span);
        up = std::min(up, xk[i] + o.asymptote_hi * span);
        up = std::max(up, xk[i] + o.asymptote_lo * span);
        low[i] = lo;
        upp[i] = up;
    }
}

// ip_residual (mma.rs:862-903): 2-norm and max-norm of the perturbed KKT
// residual of the subproblem at barrier epsi.
void mma_handle::ip_residual(double epsi, double& norm, double& maxabs) const {
    double s2 = 0.0, mx = 0.0;
    Vec a1(m, 0.0), a2(m, 0.0);
    bool finite = true;
#pragma omp parallel
    {
        Vec la1(m, 0.0), la2(m, 0.0);
        double ls2 = 0.0, lmx = 0.0;
        bool lf = true;
#pragma omp for schedule(static) nowait
        for (int64_t i = 0; i < n; ++i) {
            const double ux = upp[i] - x[i], xl = x[i] - low[i];
            double plam = p0[i], qlam = q0[i];
            for (int64_t j = 0; j < m; ++j) {
                plam += lam[j] * P[(size_t)j * n + i];
                qlam += lam[j] * Q[(size_t)j * n + i];
                la1[j] += P[(size_t)j * n + i] / ux;
                la2[j] += Q[(size_t)j * n + i] / xl;
            }
            const double r1 = plam / (ux * ux) - qlam / (xl * xl) - xsi[i] + eta[i];
            const double r2 = xsi[i] * (x[i] - alpha[i]) - epsi;
            const double r3 = eta[i] * (beta[i] - x[i]) - epsi;
            lf = lf && std::isfinite(r1) && std::isfinite(r2) && std::isfinite(r3);
            ls2 += r1 * r1 + r2 * r2 + r3 * r3;
            lmx = std::max(lmx, std::max(std::fabs(r1), std::max(std::fabs(r2), std::fabs(r3))));
        }
#pragma omp critical
        {
            s2 += ls2;
            mx = std::max(mx, lmx);
            finite = finite && lf;
            for (int64_t j = 0; j < m; ++j) {
                a1[j] += la1[j];
                a2[j] += la2[j];
            }
        }
    }
    double al = 0.0;
    for (int64_t j = 0; j < m; ++j) al += a[j] * lam[j];
    auto add = [&](double r) {
        finite = finite && std::isfinite(r);
        s2 += r * r;
        mx = std::max(mx, std::fabs(r));
    };
    for (int64_t j = 0; j < m; ++j) add(c[j] + d[j] * y[j] - mu[j] - lam[j]);
    add(o.a0 - zet - al);
    for (int64_t j = 0; j < m; ++j) add(a1[j] + a2[j] - a[j] * zv - y[j] + s[j] - b[j]);
    for (int64_t j = 0; j < m; ++j) add(mu[j] * y[j] - epsi);
    add(zet * zv - epsi);
    for (int64_t j = 0; j < m; ++j) add(lam[j] * s[j] - epsi);
    if (!finite) throw RuntimeError("MMA: non-finite values in interior-point residual");
    norm = std::sqrt(s2);
    maxabs = mx;
}

// solve_subproblem (mma.rs:906-1131): primal-dual interior point with the
// barrier epsi reduced tenfold from 1 to epsimin.
void mma_handle::solve_subproblem() {
    for (int64_t i = 0; i < n; ++i) {
        if (!(beta[i] > alpha[i])) throw ContractError("MMA: move-limit box has beta <= alpha");
        if (!(alpha[i] > low[i]) || !(beta[i] < upp[i]))
            throw ContractError("MMA: move-limit box must lie strictly inside (L, U)");
    }
    x.resize(n);
    xsi.resize(n);
    eta.resize(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        x[i] = 0.5 * (alpha[i] + beta[i]);
        xsi[i] = std::max(1.0 / (x[i] - alpha[i]), 1.0);
        eta[i] = std::max(1.0 / (beta[i] - x[i]), 1.0);
    }
    y.assign(m, 1.0);
    zv = 1.0;
    lam.assign(m, 1.0);
    mu.resize(m);
    for (int64_t j = 0; j < m; ++j) mu[j] = std::max(1.0, 0.5 * c[j]);
    zet = 1.0;
    s.assign(m, 1.0);
    ox.resize(n);
    oxsi.resize(n);
    oeta.resize(n);
    dx.resize(n);
    dxsi.resize(n);
    deta.resize(n);
    delx.resize(n);
    diagx.resize(n);
    double epsi = 1.0;
    bool converged = true;
    double residumax = std::numeric_limits<double>::infinity();
    newton_steps = 0;
    if (m >= n && m > 0) throw ContractError("MMA: this solver needs fewer constraints than design variables");
    const int dim = (int)m + 1;
    while (epsi > o.epsimin) {
        double residunorm;
        ip_residual(epsi, residunorm, residumax);
        int64_t ittt = 0;
        while (residumax > 0.9 * epsi) {
            if (ittt >= o.max_inner) {
                if (o.strict_subproblem)
                    throw RuntimeError("MMA subproblem: interior-point iteration did not reach tolerance at barrier epsi=" +
                                       std::to_string(epsi) + " within " + std::to_string(o.max_inner) +
                                       " Newton steps (max|r|=" + std::to_string(residumax) + ")");
                converged = false;
                break;
            }
            ++ittt;
            ++newton_steps;
            // pass A: delx, diagx per variable; gvec = P/ux + Q/xl, the reduced
            // matrix sum_i GG_r GG_c / diagx and GG (delx / diagx), with
            // GG_ji = P_ji/ux^2 - Q_ji/xl^2
            Vec gvec(m, 0.0), ggdx(m, 0.0), AA((size_t)dim * dim, 0.0);
#pragma omp parallel
            {
                Vec lg(m, 0.0), lgg(m, 0.0), laa((size_t)m * m, 0.0), gg(m);
#pragma omp for schedule(static) nowait
                for (int64_t i = 0; i < n; ++i) {
                    const double ux1 = upp[i] - x[i], xl1 = x[i] - low[i];
                    const double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
                    double plam = p0[i], qlam = q0[i];
                    for (int64_t j = 0; j < m; ++j) {
                        const double pj = P[(size_t)j * n + i], qj = Q[(size_t)j * n + i];
                        plam += lam[j] * pj;
                        qlam += lam[j] * qj;
                        lg[j] += pj / ux1 + qj / xl1;
                        gg[j] = pj / ux2 - qj / xl2;
                    }
                    const double dpsidx = plam / ux2 - qlam / xl2;
                    const double xa = x[i] - alpha[i], bx = beta[i] - x[i];
                    const double dl = dpsidx - epsi / xa + epsi / bx;
                    const double dg = 2.0 * (plam / (ux2 * ux1) + qlam / (xl2 * xl1)) + xsi[i] / xa + eta[i] / bx;
                    delx[i] = dl;
                    diagx[i] = dg;
                    for (int64_t r = 0; r < m; ++r) {
                        lgg[r] += gg[r] * (dl / dg);
                        for (int64_t cc = 0; cc < m; ++cc) laa[(size_t)r * m + cc] += gg[r] / dg * gg[cc];
                    }
                }
#pragma omp critical
                {
                    for (int64_t j = 0; j < m; ++j) {
                        gvec[j] += lg[j];
                        ggdx[j] += lgg[j];
                    }
                    for (int64_t r = 0; r < m; ++r)
                        for (int64_t cc = 0; cc < m; ++cc) AA[(size_t)r * dim + cc] += laa[(size_t)r * m + cc];
                }
            }
            double al = 0.0;
            for (int64_t j = 0; j < m; ++j) al += a[j] * lam[j];
            Vec dely(m), dellam(m), diagy(m), diaglamyi(m), bb(dim);
            for (int64_t j = 0; j < m; ++j) {
                dely[j] = c[j] + d[j] * y[j] - lam[j] - epsi / y[j];
                dellam[j] = gvec[j] - a[j] * zv - y[j] - b[j] + epsi / lam[j];
                diagy[j] = d[j] + mu[j] / y[j];
                diaglamyi[j] = s[j] / lam[j] + 1.0 / diagy[j];
            }
            const double delz = o.a0 - al - epsi / zv;
            for (int64_t r = 0; r < m; ++r) {
                bb[r] = dellam[r] + dely[r] / diagy[r] - ggdx[r];
                AA[(size_t)r * dim + r] += diaglamyi[r];
                AA[(size_t)r * dim + m] = a[r];
                AA[(size_t)m * dim + r] = a[r];
            }
            bb[m] = delz;
            AA[(size_t)m * dim + m] = -zet / zv;
            const Vec sol = dense_solve(AA, dim, bb);
            const Vec dlam(sol.begin(), sol.begin() + m);
            const double dz = sol[m];
            Vec dy(m), dmu(m), ds(m);
            for (int64_t j = 0; j < m; ++j) {
                dy[j] = -dely[j] / diagy[j] + dlam[j] / diagy[j];
                dmu[j] = -mu[j] + epsi / y[j] - (mu[j] * dy[j]) / y[j];
                ds[j] = -s[j] + epsi / lam[j] - (s[j] * dlam[j]) / lam[j];
            }
            const double dzet = -zet + epsi / zv - zet * dz / zv;
            // pass B: dx, dxsi, deta and the largest feasible step
            double stm = 1.0;
            bool finite = true;
#pragma omp parallel for reduction(max : stm) reduction(&& : finite) schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                const double ux1 = upp[i] - x[i], xl1 = x[i] - low[i];
                double gtl = 0.0;
                for (int64_t j = 0; j < m; ++j)
                    gtl += (P[(size_t)j * n + i] / (ux1 * ux1) - Q[(size_t)j * n + i] / (xl1 * xl1)) * dlam[j];
                const double ddx = -delx[i] / diagx[i] - gtl / diagx[i];
                const double xa = x[i] - alpha[i], bx = beta[i] - x[i];
                const double dxs = -xsi[i] + epsi / xa - (xsi[i] * ddx) / xa;
                const double det = -eta[i] + epsi / bx + (eta[i] * ddx) / bx;
                dx[i] = ddx;
                dxsi[i] = dxs;
                deta[i] = det;
                finite = finite && std::isfinite(ddx) && std::isfinite(dxs) && std::isfinite(det);
                stm = std::max(stm, std::max(-1.01 * ddx / xa, 1.01 * ddx / bx));
                stm = std::max(stm, std::max(-1.01 * dxs / xsi[i], -1.01 * det / eta[i]));
            }
            auto chk = [&](double v) { finite = finite && std::isfinite(v); };
            for (int64_t j = 0; j < m; ++j) {
                chk(dy[j]);
                chk(dlam[j]);
                chk(dmu[j]);
                chk(ds[j]);
                stm = std::max(stm, -1.01 * dy[j] / y[j]);
                stm = std::max(stm, -1.01 * dlam[j] / lam[j]);
                stm = std::max(stm, -1.01 * dmu[j] / mu[j]);
                stm = std::max(stm, -1.01 * ds[j] / s[j]);
            }
            chk(dz);
            chk(dzet);
            if (!finite) throw RuntimeError("MMA: non-finite values in Newton direction");
            stm = std::max(stm, -1.01 * dz / zv);
            stm = std::max(stm, -1.01 * dzet / zet);
            double steg = 1.0 / stm;
            // line search on the residual norm (at most 50 halvings)
            std::memcpy(ox.data(), x.data(), n * sizeof(double));
            std::memcpy(oxsi.data(), xsi.data(), n * sizeof(double));
            std::memcpy(oeta.data(), eta.data(), n * sizeof(double));
            const Vec oy = y, olam = lam, omu = mu, os = s;
            const double oz = zv, ozet = zet;
            int itto = 0;
            double resinew = 2.0 * residunorm;
            while (resinew > residunorm && itto < 50) {
                ++itto;
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < n; ++i) {
                    x[i] = ox[i] + steg * dx[i];
                    xsi[i] = oxsi[i] + steg * dxsi[i];
                    eta[i] = oeta[i] + steg * deta[i];
                }
                for (int64_t j = 0; j < m; ++j) {
                    y[j] = oy[j] + steg * dy[j];
                    lam[j] = olam[j] + steg * dlam[j];
                    mu[j] = omu[j] + steg * dmu[j];
                    s[j] = os[j] + steg * ds[j];
                }
                zv = oz + steg * dz;
                zet = ozet + steg * dzet;
                double rn, rm;
                ip_residual(epsi, rn, rm);
                resinew = rn;
                residumax = rm;
                steg *= 0.5;
            }
            residunorm = resinew;
        }
        epsi *= 0.1;
    }
    ip_converged = converged;
    ip_last_residual = residumax;
}

// sub_kkt (mma.rs:1133-1148).
double mma_handle::sub_kkt() const {
    Vec grad(n), psi(m, 0.0), g(m);
#pragma omp parallel
    {
        Vec lp(m, 0.0);
#pragma omp for schedule(static) nowait
        for (int64_t i = 0; i < n; ++i) {
            const double ux = upp[i] - x[i], xl = x[i] - low[i];
            double pt = p0[i], qt = q0[i];
            for (int64_t j = 0; j < m; ++j) {
                pt += lam[j] * P[(size_t)j * n + i];
                qt += lam[j] * Q[(size_t)j * n + i];
                lp[j] += P[(size_t)j * n + i] / ux + Q[(size_t)j * n + i] / xl;
            }
            grad[i] = pt / (ux * ux) - qt / (xl * xl);
        }
#pragma omp critical
        for (int64_t j = 0; j < m; ++j) psi[j] += lp[j];
    }
    for (int64_t j = 0; j < m; ++j) g[j] = psi[j] - a[j] * zv - y[j] - b[j];
    return natural_residual(x.data(), y.data(), zv, lam.data(), grad.data(), g.data(), alpha.data(), beta.data());
}

// ------------------------------------------------------------------ C-ABI
extern "C" {

void mma_default_options(mma_options_t* o) {
    if (!o) return;
    o->move_limit = 0.2;
    o->asymptote_init = 0.5;
    o->asymptote_expand = 1.2;
    o->asymptote_contract = 0.7;
    o->asymptote_lo = 0.01;
    o->asymptote_hi = 10.0;
    o->a0 = 1.0;
    o->raa0 = 1e-5;
    o->albefa = 0.1;
    o->epsimin = 1e-7;
    o->max_inner = 200;
    o->strict_subproblem = 0;
}

const char* mma_last_error(const mma_handle* h) { return h ? h->err.c_str() : g_err.c_str(); }

static mma_status fail(mma_handle* h, mma_status st, const std::string& msg) {
    g_err = msg;
    if (h) h->err = msg;
    return st;
}

mma_status mma_create(int64_t n, int64_t m, const mma_options_t* opts, const double* a, const double* c,
                      const double* d, const double* x_min, const double* x_max, int64_t n_bounds,
                      mma_handle** out) {
    if (!out) return fail(nullptr, MMA_E_CONTRACT, "MMA: out must not be NULL");
    *out = nullptr;
    try {
        if (n < 1) throw ContractError("MMA: design_dim must be >= 1");
        if (m < 0) throw ContractError("MMA: n_constraints must be >= 0");
        mma_options_t o;
        mma_default_options(&o);
        if (opts) o = *opts;
        if (!(0.0 < o.move_limit && o.move_limit <= 1.0)) throw ContractError("MMA: move_limit must lie in (0, 1]");
        if (!(0.0 < o.asymptote_lo && o.asymptote_lo < o.asymptote_init && o.asymptote_init <= o.asymptote_hi))
            throw ContractError("MMA: require 0 < asymptote_lo < asymptote_init <= asymptote_hi");
        if (!(0.0 < o.albefa && o.albefa < 1.0)) throw ContractError("MMA: albefa must lie in (0, 1)");
        if (o.epsimin <= 0.0 || o.max_inner < 1) throw ContractError("MMA: epsimin must be > 0 and max_inner >= 1");
        auto h = new mma_handle();
        h->n = n;
        h->m = m;
        h->o = o;
        auto coef = [&](const double* v, double def, const char* name) {
            Vec r(m, def);
            if (v)
                for (int64_t j = 0; j < m; ++j) {
                    if (!std::isfinite(v[j])) {
                        delete h;
                        throw ContractError(std::string("MMA: coefficient '") + name + "' must be finite");
                    }
                    r[j] = v[j];
                }
            return r;
        };
        h->a = coef(a, 0.0, "a");
        h->c = coef(c, 1000.0, "c");
        h->d = coef(d, 1.0, "d");
        if (!x_min || !x_max || (n_bounds != 1 && n_bounds != n)) {
            delete h;
            throw ContractError("MMA: x_min is not broadcastable to (" + std::to_string(n) + ",)");
        }
        h->x_min.resize(n);
        h->x_max.resize(n);
        h->xmami.resize(n);
        bool ordered = true;
        for (int64_t i = 0; i < n; ++i) {
            h->x_min[i] = x_min[n_bounds == 1 ? 0 : i];
            h->x_max[i] = x_max[n_bounds == 1 ? 0 : i];
            ordered = ordered && h->x_max[i] > h->x_min[i];
            h->xmami[i] = std::max(h->x_max[i] - h->x_min[i], 1e-5);
        }
        if (!ordered) {
            delete h;
            throw ContractError("MMA: x_max must exceed x_min in every coordinate");
        }
        h->lam.assign(m, 0.0);
        h->y.assign(m, 0.0);
        *out = h;
        return MMA_OK;
    } catch (const ContractError& e) {
        return fail(nullptr, MMA_E_CONTRACT, e.what());
    } catch (const std::exception& e) {
        return fail(nullptr, MMA_E_RUNTIME, e.what());
    }
}

void mma_destroy(mma_handle* h) { delete h; }

double mma_kkt_residual(const mma_handle* h, const double* x, const double* df0dx, const double* fs,
                        const double* dfsdx) {
    if (!h || h->iter == 0) return std::numeric_limits<double>::infinity();
    const int64_t n = h->n, m = h->m;
    Vec grad(df0dx, df0dx + n);
    for (int64_t j = 0; j < m; ++j)
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) grad[i] += dfsdx[(size_t)j * n + i] * h->lam[j];
    Vec g(m);
    for (int64_t j = 0; j < m; ++j) g[j] = fs[j] - h->a[j] * h->z - h->y[j];
    return h->natural_residual(x, h->y.data(), h->z, h->lam.data(), grad.data(), g.data(), h->x_min.data(),
                               h->x_max.data());
}

// coerce (mma.rs:478-520), the KKT residual of the incoming iterate,
// asymptote_update (:522-553) and trust_box (:555-571): the part of a step
// before the subproblem's coefficients.  Returns the coerced iterate.
static Vec begin_step(mma_handle* h, const double* x_k, const double* x_km1, const double* x_km2, double f0,
                      const double* df0dx, const double* fs, const double* dfsdx, const double* x_new) {
    const int64_t n = h->n, m = h->m;
    if (!x_k || !x_km1 || !x_km2 || !df0dx || !x_new || (m > 0 && (!fs || !dfsdx)))
        throw ContractError("MMA: input shapes must be x:(N,), df0dx:(N,), fs:(m,), dfsdx:(m,N) with N=" +
                            std::to_string(n) + ", m=" + std::to_string(m) + ": cannot reshape");
    const struct {
        const char* name;
        const double* v;
        size_t len;
    } arrs[] = {{"x_k", x_k, (size_t)n},      {"x_km1", x_km1, (size_t)n}, {"x_km2", x_km2, (size_t)n},
                {"df0dx", df0dx, (size_t)n},  {"fs", fs, (size_t)m},       {"dfsdx", dfsdx, (size_t)(m * n)}};
    for (const auto& a : arrs)
        if (a.len && !all_finite(a.v, a.len)) throw ContractError(std::string("MMA: non-finite entries in ") + a.name);
    if (!std::isfinite(f0)) throw ContractError("MMA: objective value f0 is not finite");
    Vec xk(n);
    bool inside = true;
#pragma omp parallel for reduction(&& : inside) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        inside = inside && x_k[i] >= h->x_min[i] - 1e-12 && x_k[i] <= h->x_max[i] + 1e-12;
        xk[i] = std::min(std::max(x_k[i], h->x_min[i]), h->x_max[i]);
    }
    if (!inside) throw ContractError("MMA: x_k lies outside [x_min, x_max]");
    h->last_kkt = mma_kkt_residual(h, xk.data(), df0dx, fs, dfsdx);
    h->asymptote_update(xk.data(), x_km1, x_km2);
    h->alpha.resize(n);
    h->beta.resize(n);
    const mma_options_t& o = h->o;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        const double l = h->low[i], u = h->upp[i], x = xk[i];
        const double span = h->x_max[i] - h->x_min[i];
        h->alpha[i] = std::max(std::max(l + o.albefa * (x - l), x - o.move_limit * span), h->x_min[i]);
        h->beta[i] = std::min(std::min(u - o.albefa * (u - x), x + o.move_limit * span), h->x_max[i]);
    }
    return xk;
}

// pq / big_pq (mma.rs:573-615) with the objective's rho0 and the
// constraints' rho (raa0 for every one in a plain step), and rhs (:617-622).
static void build_sub(mma_handle* h, const Vec& xk, const double* df0dx, const double* fs, const double* dfsdx,
                      double rho0, const Vec& rho) {
    const int64_t n = h->n, m = h->m;
    h->p0.resize(n);
    h->q0.resize(n);
    h->P.resize((size_t)m * n);
    h->Q.resize((size_t)m * n);
    Vec bsum(m, 0.0);
#pragma omp parallel
    {
        Vec lb(m, 0.0);
#pragma omp for schedule(static) nowait
        for (int64_t i = 0; i < n; ++i) {
            const double l = h->low[i], u = h->upp[i], x = xk[i];
            const double ux2 = (u - x) * (u - x), xl2 = (x - l) * (x - l);
            auto pq = [&](double df, double r, double& p, double& q) {
                const double dfp = std::max(df, 0.0), dfm = std::max(-df, 0.0);
                const double t = 0.001 * (dfp + dfm) + r / h->xmami[i];
                p = (dfp + t) * ux2;
                q = (dfm + t) * xl2;
            };
            pq(df0dx[i], rho0, h->p0[i], h->q0[i]);
            for (int64_t j = 0; j < m; ++j) {
                double& p = h->P[(size_t)j * n + i];
                double& q = h->Q[(size_t)j * n + i];
                pq(dfsdx[(size_t)j * n + i], rho[j], p, q);
                lb[j] += p / (u - x) + q / (x - l);
            }
        }
#pragma omp critical
        for (int64_t j = 0; j < m; ++j) bsum[j] += lb[j];
    }
    h->b.resize(m);
    for (int64_t j = 0; j < m; ++j) h->b[j] = bsum[j] - fs[j];
}

// record (mma.rs:771-797) and the step's diagnostics.
static void finish_step(mma_handle* h, double* x_new, mma_info_t* info, std::chrono::steady_clock::time_point t0,
                        int64_t inner, bool conservative) {
    const double skkt = h->sub_kkt();
    h->z = h->zv;
    ++h->iter;
    std::memcpy(x_new, h->x.data(), h->n * sizeof(double));
    if (info) {
        info->iteration = h->iter;
        info->kkt_residual = h->last_kkt;
        info->subproblem_kkt = skkt;
        info->subproblem_converged = h->ip_converged ? 1 : 0;
        info->subproblem_ip_residual = h->ip_last_residual;
        info->z = h->z;
        info->newton_steps = h->newton_steps;
        info->wallclock_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        info->inner_iterations = inner;
        info->conservative = conservative ? 1 : 0;
    }
}

mma_status mma_step(mma_handle* h, const double* x_k, const double* x_km1, const double* x_km2, double f0,
                    const double* df0dx, const double* fs, const double* dfsdx, double* x_new, mma_info_t* info) {
    if (!h) return fail(nullptr, MMA_E_CONTRACT, "MMA: handle is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    try {
        if (h->gcmma)
            throw ContractError("GCMMA.step requires eval_true(x) -> (f0, fs) to test conservativeness of the "
                                "approximation at the trial point");
        const Vec xk = begin_step(h, x_k, x_km1, x_km2, f0, df0dx, fs, dfsdx, x_new);
        build_sub(h, xk, df0dx, fs, dfsdx, h->o.raa0, Vec(h->m, h->o.raa0));
        h->solve_subproblem();
        finish_step(h, x_new, info, t0, 0, true);
        return MMA_OK;
    } catch (const ContractError& e) {
        return fail(h, MMA_E_CONTRACT, e.what());
    } catch (const std::exception& e) {
        return fail(h, MMA_E_RUNTIME, e.what());
    }
}

void mma_gcmma_default_options(mma_gcmma_options_t* g) {
    if (!g) return;
    g->rho_min = 1e-6;
    g->rho_init = 0.1;
    g->rho_growth = 10.0;
    g->max_conservative = 15;
}

mma_status mma_enable_gcmma(mma_handle* h, const mma_gcmma_options_t* g) {
    if (!h) return fail(nullptr, MMA_E_CONTRACT, "MMA: handle is NULL");
    mma_gcmma_options_t o;
    mma_gcmma_default_options(&o);
    if (g) o = *g;
    if (!(o.rho_min > 0.0 && o.rho_init > 0.0 && o.rho_growth > 1.0))
        return fail(h, MMA_E_CONTRACT, "GCMMA: require rho_min > 0, rho_init > 0, rho_growth > 1");
    if (o.max_conservative < 0) return fail(h, MMA_E_CONTRACT, "GCMMA: max_conservative must be >= 0");
    h->gcmma = true;
    h->g = o;
    h->nonfinite_trials = 0;
    h->rho_last.clear();
    return MMA_OK;
}

// step_gcmma (mma.rs:666-769): the conservative inner loop.  The subproblem
// is solved with rho0 (objective) and rho (constraints) raised until the
// approximations at the trial point bound the true values from above
// (within epsimin), or max_conservative inner iterations have run.
mma_status mma_step_gcmma(mma_handle* h, const double* x_k, const double* x_km1, const double* x_km2, double f0,
                          const double* df0dx, const double* fs, const double* dfsdx, mma_eval_fn eval_true,
                          void* ctx, double* x_new, mma_info_t* info) {
    if (!h) return fail(nullptr, MMA_E_CONTRACT, "MMA: handle is NULL");
    const auto t0 = std::chrono::steady_clock::now();
    try {
        if (!h->gcmma) return mma_step(h, x_k, x_km1, x_km2, f0, df0dx, fs, dfsdx, x_new, info);
        if (!eval_true) throw ContractError("GCMMA: eval_true must not be NULL");
        const mma_gcmma_options_t& g = h->g;
        const int64_t n = h->n, m = h->m;
        const Vec xk = begin_step(h, x_k, x_km1, x_km2, f0, df0dx, fs, dfsdx, x_new);
        // initial rho from the spans of the gradients (mma.rs:688-695)
        double s0 = 0.0;
        Vec sr(m, 0.0);
        for (int64_t i = 0; i < n; ++i) {
            const double span = h->x_max[i] - h->x_min[i];
            s0 += std::fabs(df0dx[i]) * span;
            for (int64_t j = 0; j < m; ++j) sr[j] += std::fabs(dfsdx[(size_t)j * n + i]) * span;
        }
        double rho0 = std::max(g.rho_min, g.rho_init * s0 / (double)n);
        Vec rho(m);
        for (int64_t j = 0; j < m; ++j) rho[j] = std::max(g.rho_min, g.rho_init * sr[j] / (double)n);
        // psi of rows (p, q) at x (psi_rows, mma.rs:624-629)
        auto psi = [&](const double* p, const double* q, const double* xx) {
            double acc = 0.0;
#pragma omp parallel for reduction(+ : acc) schedule(static)
            for (int64_t i = 0; i < n; ++i) acc += p[i] / (h->upp[i] - xx[i]) + q[i] / (xx[i] - h->low[i]);
            return acc;
        };
        int64_t inner = 0, nonfinite = 0;
        bool conservative = false;
        Vec fnew(m);
        for (;;) {
            build_sub(h, xk, df0dx, fs, dfsdx, rho0, rho);
            h->solve_subproblem();
            const double r0 = f0 - psi(h->p0.data(), h->q0.data(), xk.data());
            const double f0app = r0 + psi(h->p0.data(), h->q0.data(), h->x.data());
            Vec fapp(m);
            for (int64_t j = 0; j < m; ++j)
                fapp[j] = psi(&h->P[(size_t)j * n], &h->Q[(size_t)j * n], h->x.data()) - h->b[j];
            double f0new = 0.0;
            if (eval_true(h->x.data(), &f0new, fnew.data(), ctx) != 0)
                throw RuntimeError("GCMMA: eval_true reported a failure");
            bool finite = std::isfinite(f0new);
            for (int64_t j = 0; j < m; ++j) finite = finite && std::isfinite(fnew[j]);
            if (!finite) {
                ++nonfinite;
                if (inner >= g.max_conservative) break;
                ++inner;
                rho0 *= g.rho_growth;
                for (double& r : rho) r *= g.rho_growth;
                continue;
            }
            const bool bad0 = f0app + h->o.epsimin < f0new;
            std::vector<char> bad(m);
            bool any = bad0;
            for (int64_t j = 0; j < m; ++j) {
                bad[j] = fapp[j] + h->o.epsimin < fnew[j];
                any = any || bad[j];
            }
            if (!any) {
                conservative = true;
                break;
            }
            if (inner >= g.max_conservative) break;
            ++inner;
            double w = 0.0;
#pragma omp parallel for reduction(+ : w) schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                const double xv = h->x[i], l = h->low[i], u = h->upp[i];
                const double xxux = (xv - xk[i]) / (u - xv), xxxl = (xv - xk[i]) / (xv - l);
                w += (xxux * xxxl) * ((u - l) / h->xmami[i]);
            }
            w = std::max(w, 1e-12);
            if (bad0) rho0 = std::min(1.1 * (rho0 + (f0new - f0app) / w), g.rho_growth * rho0);
            for (int64_t j = 0; j < m; ++j)
                if (bad[j]) rho[j] = std::min(1.1 * (rho[j] + (fnew[j] - fapp[j]) / w), g.rho_growth * rho[j]);
        }
        h->nonfinite_trials += nonfinite;
        h->rho_last.assign(1, rho0);
        h->rho_last.insert(h->rho_last.end(), rho.begin(), rho.end());
        finish_step(h, x_new, info, t0, inner, conservative);
        return MMA_OK;
    } catch (const ContractError& e) {
        return fail(h, MMA_E_CONTRACT, e.what());
    } catch (const std::exception& e) {
        return fail(h, MMA_E_RUNTIME, e.what());
    }
}

int64_t mma_gcmma_state(const mma_handle* h, double* rho, int64_t* nonfinite_trials) {
    if (!h || !h->gcmma) return -1;
    if (rho) std::copy(h->rho_last.begin(), h->rho_last.end(), rho);
    if (nonfinite_trials) *nonfinite_trials = h->nonfinite_trials;
    return (int64_t)h->rho_last.size();
}

int64_t mma_state(const mma_handle* h, double* lam, double* y, double* z, double* low, double* upp) {
    if (!h) return -1;
    if (lam) std::copy(h->lam.begin(), h->lam.end(), lam);
    if (y) std::copy(h->y.begin(), h->y.end(), y);
    if (z) *z = h->z;
    if (low && !h->low.empty()) std::copy(h->low.begin(), h->low.end(), low);
    if (upp && !h->upp.empty()) std::copy(h->upp.begin(), h->upp.end(), upp);
    return h->iter;
}

}  // extern "C"
