// lbm_misc.cu -- one-off kernels around the stepping: initial state,
// responses and their VJP (the adjoint seed), state/adjoint layout
// conversions, the design map and its transpose.  Streamed states are read
// through the pull of the stepping kernels and written through its inverse
// scatter (pull_index, lbm_device.cuh).
#include <algorithm>

#include "lbm_device.cuh"

namespace lbm {
namespace {

// ------------------------------------------------------------------ kernels
// Initial streamed state (initial_populations, solver.rs:593-601): fluid
// w(1 - 1.5 c.a), solid w.  Fluid cells scatter through the inverse pull,
// solid cells fill their own slots.
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_init(Geometry G, Physics P, T* A, const uint32_t* __restrict__ mask,
                                                uint32_t c_begin, uint32_t c_end) {
    using L = Lat<Q>;
    // an x-slab initialises its owned cells only: they also fill the ghost
    // slots they pull from, which the ghost cells must not overwrite
    for (uint32_t x = c_begin + blockIdx.x * BLOCK + threadIdx.x; x < c_end; x += gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
        const bool solid = m & MASK_SOLID;
        const uint32_t n = (uint32_t)G.n;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float ca = L::cx(q) * P.a[0] + L::cy(q) * P.a[1] + L::cz(q) * P.a[2];
            const float g = solid ? 0.f : -1.5f * L::w(q) * ca;
            A[solid ? q * n + x : pull_index<Q>(G, x, m, q)] = penc<Q, T>(g, q);
        }
    }
}

// Responses of one state (mode 0) or their VJP seeding the adjoint (mode 1).
// vector_cell / vector_vjp, solver.rs:835-947, plus the pressure drop and the
// viscous dissipation sigma:sigma / (2 rho nu) with the Guo-corrected
// non-equilibrium stress sigma = -(1 - omega/2) (Pi_neq + (uF + Fu)/2).
template <int Q, typename T, typename TL, int MODE>
__global__ void __launch_bounds__(BLOCK) k_objective(ObjArgs a) {
    using L = Lat<Q>;
    const T* A = static_cast<const T*>(a.pop);
    const int64_t n = a.G.n;
    Sums<8> acc;
    acc.init();
    double nsum = 0.0;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < (uint32_t)n; x += gridDim.x * BLOCK) {
        if (x < a.c_begin || x >= a.c_end) continue;  // ghost planes of an x-slab belong to other ranks
        const uint32_t m = a.mask[x];
        if (m & MASK_SOLID) {
            if constexpr (MODE == 0) acc.add(5, (double)a.phi[x]);
            else {
                a.phibar[x] = (float)a.w[5];
                a.abar_final[x] = 0.f;
            }
            continue;
        }
        float g[Q];
        load_pop<Q, T>(A, a.G, x, m, g);
        const PortMap* pm = (m & MASK_PORT) ? &a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1] : nullptr;
        const float alpha = a.alpha[x];
        if constexpr (MODE == 0) {
            // Responses in FP64 from the stored populations: the viscous
            // stress is a small difference of second moments, which FP32
            // arithmetic would resolve to only ~1e-4 per cell.
            double gd[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) gd[q] = g[q];
            if (a.apply_ports && pm && pm->recon == 3) {
                float gp[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) gp[q] = g[q];
                regularized_apply<Q>(*pm, gp);
#pragma unroll
                for (int q = 0; q < Q; ++q) gd[q] = gp[q];
            } else if (a.apply_ports && pm && pm->recon) {
                // extrapolation from the inward neighbour's streamed populations
                const uint32_t xn = (uint32_t)((int64_t)x + pm->nb_off);
                float gnf[Q];
                load_pop<Q, T>(A, a.G, xn, a.mask[xn], gnf);
                double gn[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) gn[q] = gnf[q];
                nee_apply<Q, double>(*pm, gn, gd);
            } else if (a.apply_ports && pm) {
                double in[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) in[q] = gd[q];
#pragma unroll
                for (int r = 0; r < Q; ++r) {
                    if (pm->unknown_mask & (1u << r)) {
                        double acc_r = pm->bias[r];
#pragma unroll
                        for (int kk = 0; kk < Q; ++kk) acc_r = fma((double)pm->jac[r][kk], in[kk], acc_r);
                        gd[r] = acc_r;
                    }
                }
            }
            double rp = 0.0, j[3] = {0.0, 0.0, 0.0}, S2[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
                rp += gd[q];
                if (c0) { j[0] += c0 * gd[q]; S2[0] += gd[q]; }
                if (c1) { j[1] += c1 * gd[q]; S2[1] += gd[q]; }
                if (c2) { j[2] += c2 * gd[q]; S2[2] += gd[q]; }
                if (c0 && c1) S2[3] += c0 * c1 * gd[q];
                if (c0 && c2) S2[4] += c0 * c2 * gd[q];
                if (c1 && c2) S2[5] += c1 * c2 * gd[q];
            }
            const double rho = 1.0 + rp, sd = 1.0 + 0.5 * (double)alpha;
            double ud[3], Fd[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ud[d] = (j[d] / rho + 0.5 * (double)a.P.a[d]) / sd;
                Fd[d] = rho * ((double)a.P.a[d] - (double)alpha * ud[d]);
            }
            const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
            const double kd = 1.0 - 0.5 / (double)a.tau, nud = ((double)a.tau - 0.5) / 3.0;
            double ss = 0.0;
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                const double pi = S2[e] - (e < 3 ? rp / 3.0 : 0.0) - rho * ud[ia[e]] * ud[ib[e]];
                const double t = 0.5 * (ud[ia[e]] * Fd[ib[e]] + ud[ib[e]] * Fd[ia[e]]);
                const double sg = -kd * (pi + t);
                ss += (e < 3 ? 1.0 : 2.0) * sg * sg;
            }
            const double V = a.vel;
            const double U[3] = {ud[0] * V, ud[1] * V, ud[2] * V};
            const double R = rho * a.dens;
            const double usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
            acc.add(0, U[0]);
            acc.add(1, U[1]);
            acc.add(2, U[2]);
            acc.add(3, R * usq);
            acc.add(4, R * (double)alpha / a.dt_s * usq);
            acc.add(5, (double)a.phi[x]);
            if (pm) acc.add(6, (double)pm->dp_weight * a.dens * rp * V * V / 3.0);
            acc.add(7, ss / (2.0 * rho * nud));
            if (a.fields) {
                a.fields[x] = (float)rp;
                a.fields[n + x] = (float)ud[0];
                a.fields[2 * n + x] = (float)ud[1];
                a.fields[3 * n + x] = (float)ud[2];
            }
            continue;
        }
        // the (rho - 1, j / rho) a nonlinear port's transpose is linearised at
        float rpn = 0.f, un[3] = {0.f, 0.f, 0.f};
        if (pm && pm->recon && (a.apply_ports || a.port_transpose)) {
            float gp[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) gp[q] = g[q];
            port_state<Q, T>(*pm, A, a.G, a.mask, x, gp, &rpn, un);
            if (a.apply_ports) {
#pragma unroll
                for (int q = 0; q < Q; ++q) g[q] = gp[q];
            }
        } else if (a.apply_ports && pm) {
            apply_port<Q>(*pm, g);
        }
        Macro M = macroscopic<Q>(g, alpha, a.P);
        float S[6];
        second_moments<Q>(g, S);
        SeedParams sp;
#pragma unroll
        for (int r = 0; r < 8; ++r) sp.w[r] = (float)a.w[r];
        sp.vel = a.vel;
        sp.dens = a.dens;
        sp.dt_s = a.dt_s;
        sp.tau = a.tau;
        const float* u = M.u;
        {
            float fb[Q];
            const float abar = response_vjp<Q>(M.rp, M.u, S, alpha, pm ? pm->dp_weight : 0.f, pm != nullptr, sp, a.P, fb);
            a.abar_final[x] = abar;
            a.phibar[x] = (float)a.w[5];
            if (a.record) {
                a.record[x] = M.rp;
                a.record[n + x] = u[0];
                a.record[2 * n + x] = u[1];
                a.record[3 * n + x] = u[2];
            }
            // (an extrapolating port cell keeps its neighbour's share in its own
            // slots for launch_nee_move)
            if (a.port_transpose && pm) port_vjp<Q>(*pm, rpn, un, fb);
            if (a.write_lambda) {
                TL* B = static_cast<TL*>(a.lam);
#pragma unroll
                for (int q = 0; q < Q; ++q) B[q * n + x] = Cvt<TL>::from(fb[q] * a.lam_scale);
            }
            if (a.norm2) {
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const float sv = fb[q] * a.lam_scale;
                    nsum += (double)sv * (double)sv;
                }
            }
        }
    }
    if constexpr (MODE == 0) {
        finish_sums<8>(acc, a.sums, a.red);
    } else {
        if (a.norm2) {
            Sums<1> s;
            s.init();
            s.h[0] = nsum;
            finish_sums<1>(s, a.norm2, a.red);
        }
    }
}

// Streamed state (with the pending port reconstruction) in natural planes.
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_canon_pop(Geometry G, const T* A, const uint32_t* __restrict__ mask,
                                                     const PortMap* ports, int apply_ports, float* out) {
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < (uint32_t)G.n; x += gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
        float g[Q];
        if (m & MASK_SOLID) {
#pragma unroll
            for (int q = 0; q < Q; ++q) g[q] = pdec<Q, T>(A[(int64_t)q * G.n + x], q);
        } else {
            load_pop<Q, T>(A, G, x, m, g);
            if (apply_ports && (m & MASK_PORT)) port_state<Q, T>(ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], A, G, mask, x, g);
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) out[(int64_t)q * G.n + x] = g[q];
    }
}

// A given streamed state (natural planes, g = f - w) -> stored layout: the
// inverse of the pull for fluid cells, own slots for solid cells.
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_upload_pop(Geometry G, T* A, const uint32_t* __restrict__ mask,
                                                      const float* in) {
    const uint32_t n = (uint32_t)G.n;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < n; x += gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
#pragma unroll
        for (int q = 0; q < Q; ++q)
            A[(m & MASK_SOLID) ? q * n + x : pull_index<Q>(G, x, m, q)] = penc<Q, T>(in[(size_t)q * n + x], q);
    }
}

// Natural-order lambda after a transposed step (own slots; zero at solids).
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_canon_lam(Geometry G, const T* B, const uint32_t* __restrict__ mask,
                                                     float inv_scale, float* out) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
        const bool solid = mask[x] & MASK_SOLID;
#pragma unroll
        for (int q = 0; q < Q; ++q)
            out[(int64_t)q * G.n + x] = solid ? 0.f : Cvt<T>::to(B[(int64_t)q * G.n + x]) * inv_scale;
    }
}

// Natural lambda (cotangent of the post-port state) -> stored seed layout.
// Nonlinear port cells take the (rho - 1, u) they are linearised at from
// rec_next, the record of the state lambda belongs to; extrapolating ones
// keep the neighbour's share in their own slots for launch_nee_move.
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_seed_lam(Geometry G, T* B, const uint32_t* __restrict__ mask,
                                                    const PortMap* ports, const float* in, float scale,
                                                    int port_transpose_on, const float* rec_next,
                                                    const float* __restrict__ alpha) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
        if (m & MASK_SOLID) continue;
        float v[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] = in[(int64_t)q * G.n + x];
        if (port_transpose_on && (m & MASK_PORT)) {
            const PortMap& pm = ports[((m >> MASK_PORT_SHIFT) & 7u) - 1];
            if (!pm.recon) {
                port_transpose<Q>(pm, v);
            } else {
                const int64_t xm = port_lin_cell(pm, x);
                const float sc = 1.f + 0.5f * alpha[xm];
                const float um[3] = {rec_next[G.n + xm] * sc, rec_next[2 * G.n + xm] * sc, rec_next[3 * G.n + xm] * sc};
                port_vjp<Q>(pm, rec_next[xm], um, v);
            }
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) B[q * G.n + x] = Cvt<T>::from(v[q] * scale);
    }
}

// Second half of an extrapolating port's transpose: the neighbour's share,
// which the transposed step (or seed) left in the port cell's own slots, is
// added to the neighbour's slots and the port cell's slots are cleared
// (its populations are rebuilt from the neighbour, so nothing flows back
// through them).  The cells of one port have distinct neighbours; ports are
// moved one launch after another.
template <typename TL>
__global__ void __launch_bounds__(BLOCK) k_nee_move(TL* B, int64_t n, int Q, const uint32_t* __restrict__ cells,
                                                   int64_t count, int64_t nb_off) {
    for (int64_t i = (int64_t)blockIdx.x * BLOCK + threadIdx.x; i < count; i += (int64_t)gridDim.x * BLOCK) {
        const int64_t x = cells[i], xn = x + nb_off;
        for (int q = 0; q < Q; ++q) {
            const float v = Cvt<TL>::to(B[q * n + x]);
            B[q * n + xn] = Cvt<TL>::from(Cvt<TL>::to(B[q * n + xn]) + v);
            B[q * n + x] = Cvt<TL>::from(0.f);
        }
    }
}

// ------------------------------------------------------------------ wall loads
// Fixed-wall momentum exchange of the last interval (wall_exchange.rs:79-100):
// the state before the last step is pulled again from the previous array
// (with its port reconstruction), collided with the Guo-BGK collision that
// the reference's loads use whatever the problem's collision
// (solver::collide), and each listed blocked link (cell, q) gets the
// outgoing population g*_opp(q) = f*_opp(q) - w_opp(q).
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_wall_loads(Geometry G, Physics P, const T* A, const uint32_t* __restrict__ mask,
                                                      const float* __restrict__ alpha, const PortMap* ports,
                                                      int apply_ports, const uint32_t* cells, const uint8_t* links,
                                                      int64_t n_links, double* out, const float* omega_cell) {
    for (int64_t i = (int64_t)blockIdx.x * BLOCK + threadIdx.x; i < n_links; i += (int64_t)gridDim.x * BLOCK) {
        const uint32_t x = cells[i];
        const int q = links[i];
        const uint32_t m = mask[x];
        float g[Q];
        load_pop<Q, T>(A, G, x, m, g);
        if (apply_ports && (m & MASK_PORT)) port_state<Q, T>(ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], A, G, mask, x, g);
        const float om = omega_cell ? omega_cell[x] : P.omega;  // BGK: both pair rates
        collide_fused<Q, CK_PAIRS, 0>(g, alpha[x], P, true, om, om);
        float o = 0.f;
#pragma unroll
        for (int r = 0; r < Q; ++r)
            if (r == opp<Q>(q)) o = g[r];
        out[i] = (double)o;
    }
}

// ------------------------------------------------------------------ relaxation-time cotangent
// tau_bar of interval_vjp with Tau::PerCell (collide_cell_vjp, solver.rs:
// 214-285): with post_bar the cotangent of the cell's post-collision
// populations (gathered from the stored next-state cotangent like the
// transposed step), tau_bar = sum_q post_bar_q [(f_q - eq_q) + w_q (3 c.F -
// 3 u.F + 9 (c.u)(c.F)) / 2] / tau^2 at the state f.  FP64 arithmetic; one
// thread per cell (a per-step call, not a stepping kernel).
template <int Q>
__global__ void __launch_bounds__(BLOCK) k_tau_bar(Geometry G, Physics P, const float* __restrict__ g,
                                                   const float* __restrict__ lam, const uint32_t* __restrict__ mask,
                                                   const float* __restrict__ alpha,
                                                   const float* __restrict__ omega_cell, double* out) {
    using L = Lat<Q>;
    const uint32_t n = (uint32_t)G.n;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < n; x += gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
        if (m & MASK_SOLID) {
            out[x] = 0.0;
            continue;
        }
        double f[Q], rho = 0.0, j[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            f[q] = L::wd(q) + (double)g[(size_t)q * n + x];
            rho += f[q];
            j[0] += L::cx(q) * f[q];
            j[1] += L::cy(q) * f[q];
            j[2] += L::cz(q) * f[q];
        }
        const double al = alpha[x], s = 1.0 + 0.5 * al;
        double u[3], F[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            u[d] = (j[d] / rho + 0.5 * (double)P.a[d]) / s;
            F[d] = rho * ((double)P.a[d] - al * u[d]);
        }
        const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const double uf = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
        const double tau = 1.0 / (double)(omega_cell ? omega_cell[x] : P.omega);
        double tb = 0.0;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const double pb = (double)lam[pull_adj_index<Q>(G, x, m, q)];
            const double cu = dotc_d<Q>(q, u), cf = dotc_d<Q>(q, F);
            const double eq = rho * L::wd(q) * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq);
            tb += pb * ((f[q] - eq) + 0.5 * L::wd(q) * (3.0 * cf - 3.0 * uf + 9.0 * cu * cf));
        }
        out[x] = tb / (tau * tau);
    }
}

// ------------------------------------------------------------------ slab halos
// x-slab decomposition: the face-crossing directions of one x plane of a
// stored array (state or adjoint) to or from a contiguous buffer laid out
// [direction][cell of the plane].  Plain coalesced copies.
struct HaloDirs {
    int32_t q[9];
    int32_t n;
};
template <typename T>
__global__ void __launch_bounds__(BLOCK) k_halo_copy(T* arr, uint32_t n, uint32_t plane0, uint32_t sx, HaloDirs d,
                                                     T* buf, int unpack) {
    const uint32_t total = sx * (uint32_t)d.n;
    for (uint32_t i = blockIdx.x * BLOCK + threadIdx.x; i < total; i += gridDim.x * BLOCK) {
        const uint32_t k = i / sx, j = i - k * sx;
        T* slot = arr + (size_t)d.q[k] * n + plane0 + j;
        if (unpack) *slot = buf[i];
        else buf[i] = *slot;
    }
}

// ------------------------------------------------------------------ bounded-wait probe
// One thread waits on an mbarrier that nothing arrives at, with the stepping
// kernels' bounded wait and a short limit: the wait must give up, set the
// error flag and return, leaving the context usable.
__global__ void k_wait_probe(int* err, uint64_t limit_ns, unsigned long long* waited_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint64_t t0 = global_ns();
        mbar_wait(&bar, 0, err, limit_ns);
        *waited_ns = global_ns() - t0;
    }
}

// ------------------------------------------------------------------ design
__device__ __forceinline__ bool shifted(const Geometry& G, int64_t x, int dx, int dy, int dz, int64_t& out) {
    int64_t i, j, k;
    coords(G, x, i, j, k);
    i += dx;
    j += dy;
    k += dz;
    if (i < 0 || i >= G.nx) {
        if (!(G.periodic & 1)) return false;
        i = (i % G.nx + G.nx) % G.nx;
    }
    if (j < 0 || j >= G.ny) {
        if (!(G.periodic & 2)) return false;
        j = (j % G.ny + G.ny) % G.ny;
    }
    if (k < 0 || k >= G.nz) {
        if (!(G.periodic & 4)) return false;
        k = (k % G.nz + G.nz) % G.nz;
    }
    out = (i * G.ny + j) * G.nz + k;
    return true;
}

// DesignMap::map + resistance (design.rs:199-216, 284-286).
__global__ void __launch_bounds__(BLOCK) k_design_map(DesignArgs a) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < a.G.n; x += (int64_t)gridDim.x * BLOCK) {
        const uint8_t c = a.cls[x];
        float phi, den = 1.f, slope = 0.f;
        if (c == 0) phi = 0.f;
        else if (c == 2) phi = a.fixed[x];
        else {
            float f;
            if (a.n_offsets == 0) f = a.raw[x];
            else {
                float num = 0.f, dsum = 0.f;
                for (int o = 0; o < a.n_offsets; ++o) {
                    const int4 off = a.offsets[o];
                    int64_t src;
                    if (!shifted(a.G, x, -off.x, -off.y, -off.z, src)) continue;
                    if (a.cls[src] != 1) continue;
                    const float wgt = __int_as_float(off.w);
                    num = fmaf(wgt, a.raw[src], num);
                    dsum += wgt;
                }
                den = dsum > 0.f ? dsum : 1.f;
                f = num / den;
            }
            if (a.beta > 0.f) {
                const float t = tanhf(a.beta * (f - a.eta));
                phi = (a.proj_a + t) / a.proj_den;
                slope = a.beta * (1.f - t * t) / a.proj_den;
            } else {
                phi = f;
                slope = 1.f;
            }
        }
        a.phi[x] = phi;
        a.alpha[x] = a.ramp_c * (1.f - phi) / (a.ramp_q + phi);
        a.den[x] = den;
        a.slope[x] = slope;
    }
}

// phi_bar += (abar + abar_final) d alpha / d phi; then the projection slope
// and the filter normalisation (provider.rs:352-354, design.rs:219-243).
__global__ void __launch_bounds__(BLOCK) k_sens_scale(DesignArgs a) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < a.G.n; x += (int64_t)gridDim.x * BLOCK) {
        float v = 0.f;
        if (a.cls[x] == 1) {
            const float phi = a.phi[x];
            const float d = a.ramp_q + phi;
            const float dres = a.ramp_c * (-d - (1.f - phi)) / (d * d);
            float ab = 0.f;
            if (a.abar) ab += a.abar[x] * a.abar_scale;
            if (a.abar_final) ab += a.abar_final[x];
            const float pb = a.phibar[x] + ab * dres;
            v = pb * a.slope[x] / a.den[x];
        }
        a.scale[x] = v;
    }
}

__global__ void __launch_bounds__(BLOCK) k_filter_transpose(DesignArgs a) {
    for (int64_t s = (int64_t)blockIdx.x * BLOCK + threadIdx.x; s < a.G.n; s += (int64_t)gridDim.x * BLOCK) {
        float g = 0.f;
        if (a.cls[s] == 1) {
            if (a.n_offsets == 0) g = a.scale[s];
            else {
                for (int o = 0; o < a.n_offsets; ++o) {
                    const int4 off = a.offsets[o];
                    int64_t x;
                    if (!shifted(a.G, s, off.x, off.y, off.z, x)) continue;
                    g = fmaf(__int_as_float(off.w), a.scale[x], g);
                }
            }
        }
        a.grad[s] = g;
    }
}


}  // namespace

cudaError_t launch_init(int Q, int storage, const Geometry& G, const Physics& P, void* pop, const uint32_t* mask,
                        int64_t c_begin, int64_t c_end, cudaStream_t s) {
    const int grid = blocks_for(c_end - c_begin, 0);
    const uint32_t b = (uint32_t)c_begin, e = (uint32_t)c_end;
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T, k_init<19, T><<<grid, BLOCK, 0, s>>>(G, P, static_cast<T*>(pop), mask, b, e))
    } else {
        LBM_STORAGE_DISPATCH(storage, T, k_init<27, T><<<grid, BLOCK, 0, s>>>(G, P, static_cast<T*>(pop), mask, b, e))
    }
    return cudaGetLastError();
}

template <int Q, typename T>
static void objective_dispatch(int lstorage, int mode, const ObjArgs& a, int grid, cudaStream_t s) {
    if (mode == 0) {
        k_objective<Q, T, float, 0><<<persistent_grid((const void*)k_objective<Q, T, float, 0>, a.G.n), BLOCK, 0, s>>>(a);
    } else {
        LBM_STORAGE_DISPATCH(lstorage, TL, k_objective<Q, T, TL, 1><<<persistent_grid((const void*)k_objective<Q, T, TL, 1>, a.G.n), BLOCK, 0, s>>>(a))
    }
}

cudaError_t launch_wait_probe(int* err, uint64_t limit_ns, unsigned long long* waited_ns, cudaStream_t s) {
    k_wait_probe<<<1, 32, 0, s>>>(err, limit_ns, waited_ns);
    return cudaGetLastError();
}

cudaError_t launch_objective(int Q, int storage, int lstorage, int mode, const ObjArgs& a, int grid,
                             cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T, objective_dispatch<19, T>(lstorage, mode, a, grid, s))
    } else {
        LBM_STORAGE_DISPATCH(storage, T, objective_dispatch<27, T>(lstorage, mode, a, grid, s))
    }
    return cudaGetLastError();
}

cudaError_t launch_canon_pop(int Q, int storage, const Geometry& G, const void* pop, const uint32_t* mask,
                             const PortMap* ports, int apply_ports, float* out, int grid, cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_canon_pop<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(pop), mask, ports,
                                                                        apply_ports, out))
    } else {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_canon_pop<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(pop), mask, ports,
                                                                        apply_ports, out))
    }
    return cudaGetLastError();
}

cudaError_t launch_upload_pop(int Q, int storage, const Geometry& G, void* pop, const uint32_t* mask,
                              const float* in, int grid, cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_upload_pop<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(pop), mask, in))
    } else {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_upload_pop<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(pop), mask, in))
    }
    return cudaGetLastError();
}

cudaError_t launch_wall_loads(int Q, int storage, const Geometry& G, const Physics& P, const void* A,
                              const uint32_t* mask, const float* alpha, const PortMap* ports, int apply_ports,
                              const uint32_t* cells, const uint8_t* links, int64_t n_links, double* out,
                              const float* omega_cell, cudaStream_t s) {
    if (n_links <= 0) return cudaSuccess;
    const int grid = (int)std::min<int64_t>((n_links + BLOCK - 1) / BLOCK, 4096);
    Physics B = P;
    B.om = B.omega;  // BGK: both pair rates equal the shear rate
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_wall_loads<19, T><<<grid, BLOCK, 0, s>>>(G, B, static_cast<const T*>(A), mask, alpha,
                                                                         ports, apply_ports, cells, links, n_links,
                                                                         out, omega_cell))
    } else {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_wall_loads<27, T><<<grid, BLOCK, 0, s>>>(G, B, static_cast<const T*>(A), mask, alpha,
                                                                         ports, apply_ports, cells, links, n_links,
                                                                         out, omega_cell))
    }
    return cudaGetLastError();
}

cudaError_t launch_tau_bar(int Q, const Geometry& G, const Physics& P, const float* g, const float* lam,
                           const uint32_t* mask, const float* alpha, const float* omega_cell, double* out, int grid,
                           cudaStream_t s) {
    if (Q == 19) k_tau_bar<19><<<grid, BLOCK, 0, s>>>(G, P, g, lam, mask, alpha, omega_cell, out);
    else k_tau_bar<27><<<grid, BLOCK, 0, s>>>(G, P, g, lam, mask, alpha, omega_cell, out);
    return cudaGetLastError();
}

cudaError_t launch_halo_copy(int storage, void* arr, int64_t n, int64_t plane0, int64_t sx, const int32_t* dirs,
                             int ndir, void* buf, int unpack, cudaStream_t s) {
    if (ndir < 1 || ndir > 9) return cudaErrorInvalidValue;
    HaloDirs d{};
    for (int k = 0; k < ndir; ++k) d.q[k] = dirs[k];
    d.n = ndir;
    const int grid = (int)std::min<int64_t>((sx * ndir + BLOCK - 1) / BLOCK, 1024);
    LBM_STORAGE_DISPATCH(storage, T,
                         k_halo_copy<T><<<grid, BLOCK, 0, s>>>(static_cast<T*>(arr), (uint32_t)n, (uint32_t)plane0,
                                                               (uint32_t)sx, d, static_cast<T*>(buf), unpack))
    return cudaGetLastError();
}

cudaError_t launch_canon_lam(int Q, int lstorage, const Geometry& G, const void* lam, const uint32_t* mask,
                             float inv_scale, float* out, int grid, cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_canon_lam<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(lam), mask,
                                                                        inv_scale, out))
    } else {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_canon_lam<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(lam), mask,
                                                                        inv_scale, out))
    }
    return cudaGetLastError();
}

cudaError_t launch_seed_lam(int Q, int lstorage, const Geometry& G, void* lam, const uint32_t* mask,
                            const PortMap* ports, const float* in, float scale, int port_transpose_on,
                            const float* rec_next, const float* alpha, int grid, cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_seed_lam<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(lam), mask, ports, in,
                                                                       scale, port_transpose_on, rec_next, alpha))
    } else {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_seed_lam<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(lam), mask, ports, in,
                                                                       scale, port_transpose_on, rec_next, alpha))
    }
    return cudaGetLastError();
}

cudaError_t launch_nee_move(int lstorage, void* lam, int64_t n, int Q, const uint32_t* cells, int64_t count,
                            int64_t nb_off, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int grid = (int)std::min<int64_t>((count + BLOCK - 1) / BLOCK, 1024);
    LBM_STORAGE_DISPATCH(lstorage, T,
                         k_nee_move<T><<<grid, BLOCK, 0, s>>>(static_cast<T*>(lam), n, Q, cells, count, nb_off))
    return cudaGetLastError();
}

cudaError_t launch_design_map(const DesignArgs& a, int grid, cudaStream_t s) {
    k_design_map<<<grid, BLOCK, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_sens_scale(const DesignArgs& a, int grid, cudaStream_t s) {
    k_sens_scale<<<grid, BLOCK, 0, s>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_filter_transpose(const DesignArgs& a, int grid, cudaStream_t s) {
    k_filter_transpose<<<grid, BLOCK, 0, s>>>(a);
    return cudaGetLastError();
}



}  // namespace lbm
