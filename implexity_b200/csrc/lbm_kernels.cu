// lbm_kernels.cu -- sm_100a kernels of the differentiable lattice-Boltzmann
// density-design solver.
//
// Memory layout (all on one GPU):
//   populations  Q planes of n cells, plane q at pop + q*n; cells in the
//                reference Grid order (i*ny + j)*nz + k, so axis 2 is the
//                contiguous one.  FP32 stores g = f - w; FP16/BF16 store g/w.
//   mask         one uint32 per cell (lbm_common.cuh)
//   alpha, phi   FP32 per cell
//   lambda       Q planes, adjoint populations (FP32/FP16/BF16, global scale)
//   record       4 FP32 planes (rho-1, u) of the forward state the adjoint
//                linearises at
//
// Streaming is the AA pattern: one population array updated in place.  A step
// of parity 0 reads a cell's own slots and writes its post-collision values
// into the opposite slots of the same cell; a step of parity 1 reads the
// neighbours' opposite slots (the post-collision values streaming in) and
// writes to the neighbours' slots.  A blocked link (halfway bounce-back,
// Streaming::new solver.rs:84-119) reads/writes the cell's own slot instead.
// Every slot is read and written by exactly one thread per step, so the
// update is race free without a second buffer.
//
// The adjoint transposes the same pattern: it is the AA scheme run with the
// velocities reversed (pull from x + c_q), linearised at a recorded (rho, u).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbm_launch.h"

namespace lbm {
namespace {

constexpr int BLOCK = 256;
constexpr unsigned FULL = 0xffffffffu;

// ------------------------------------------------------------------ storage
template <typename T>
struct Cvt;
template <>
struct Cvt<float> {
    static constexpr bool scaled = false;
    __device__ __forceinline__ static float to(float v) { return v; }
    __device__ __forceinline__ static float from(float v) { return v; }
};
template <>
struct Cvt<__half> {
    static constexpr bool scaled = true;
    __device__ __forceinline__ static float to(__half v) { return __half2float(v); }
    __device__ __forceinline__ static __half from(float v) { return __float2half_rn(v); }
};
template <>
struct Cvt<__nv_bfloat16> {
    static constexpr bool scaled = true;
    __device__ __forceinline__ static float to(__nv_bfloat16 v) { return __bfloat162float(v); }
    __device__ __forceinline__ static __nv_bfloat16 from(float v) { return __float2bfloat16_rn(v); }
};

// population value of direction q (g = f - w) <-> stored element
template <int Q, typename T>
__device__ __forceinline__ float pdec(T v, int q) {
    if constexpr (Cvt<T>::scaled) return Cvt<T>::to(v) * Lat<Q>::w(q);
    else return Cvt<T>::to(v);
}
template <int Q, typename T>
__device__ __forceinline__ T penc(float g, int q) {
    if constexpr (Cvt<T>::scaled) return Cvt<T>::from(g * (float)(1.0 / Lat<Q>::wd(q)));
    else return Cvt<T>::from(g);
}

// ------------------------------------------------------------------ indexing
__device__ __forceinline__ int64_t neighbor(const Geometry& G, int64_t x, uint32_t m, int dx, int dy, int dz) {
    if (!(m & MASK_WRAP)) return x + (int64_t)dx * G.sx + (int64_t)dy * G.sy + dz;
    int64_t k = x % G.nz;
    int64_t ij = x / G.nz;
    int64_t j = ij % G.ny;
    int64_t i = ij / G.ny;
    i += dx;
    j += dy;
    k += dz;
    if (i < 0) i += G.nx;
    else if (i >= G.nx) i -= G.nx;
    if (j < 0) j += G.ny;
    else if (j >= G.ny) j -= G.ny;
    if (k < 0) k += G.nz;
    else if (k >= G.nz) k -= G.nz;
    return (i * G.ny + j) * G.nz + k;
}

__device__ __forceinline__ void coords(const Geometry& G, int64_t x, int64_t& i, int64_t& j, int64_t& k) {
    k = x % G.nz;
    int64_t ij = x / G.nz;
    j = ij % G.ny;
    i = ij / G.ny;
}

// Forward AA access.  parity 0 reads own slots; parity 1 gathers the
// neighbours' opposite slots (own slot when the link is blocked).
template <int Q, typename T>
__device__ __forceinline__ void load_pop(const T* __restrict__ A, const Geometry& G, int64_t x, uint32_t m,
                                         int parity, float (&g)[Q]) {
    using L = Lat<Q>;
    const int64_t n = G.n;
    if (parity == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] = pdec<Q, T>(A[q * n + x], q);
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int64_t idx;
            if (m & (1u << q)) idx = q * n + x;
            else idx = opp<Q>(q) * n + neighbor(G, x, m, -L::cx(q), -L::cy(q), -L::cz(q));
            g[q] = pdec<Q, T>(A[idx], q);
        }
    }
}

template <int Q, typename T>
__device__ __forceinline__ void store_pop(T* A, const Geometry& G, int64_t x, uint32_t m, int parity,
                                          const float (&g)[Q]) {
    using L = Lat<Q>;
    const int64_t n = G.n;
    if (parity == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) A[opp<Q>(q) * n + x] = penc<Q, T>(g[q], q);
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            int64_t idx;
            if (m & (1u << opp<Q>(q))) idx = opp<Q>(q) * n + x;  // x + c_q is a wall: bounce back
            else idx = q * n + neighbor(G, x, m, L::cx(q), L::cy(q), L::cz(q));
            A[idx] = penc<Q, T>(g[q], q);
        }
    }
}

// Adjoint AA access (velocities reversed).
template <int Q, typename T>
__device__ __forceinline__ void load_lam(const T* __restrict__ B, const Geometry& G, int64_t x, uint32_t m,
                                         int parity, float scale, float (&v)[Q]) {
    using L = Lat<Q>;
    const int64_t n = G.n;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int64_t idx;
        if (parity == 0 || (m & (1u << opp<Q>(q)))) idx = (int64_t)q * n + x;
        else idx = opp<Q>(q) * n + neighbor(G, x, m, L::cx(q), L::cy(q), L::cz(q));
        v[q] = Cvt<T>::to(B[idx]) * scale;
    }
}

template <int Q, typename T>
__device__ __forceinline__ void store_lam(T* B, const Geometry& G, int64_t x, uint32_t m, int parity, float scale,
                                          const float (&v)[Q]) {
    using L = Lat<Q>;
    const int64_t n = G.n;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        int64_t idx;
        if (parity == 0 || (m & (1u << q))) idx = opp<Q>(q) * n + x;
        else idx = (int64_t)q * n + neighbor(G, x, m, -L::cx(q), -L::cy(q), -L::cz(q));
        B[idx] = Cvt<T>::from(v[q] * scale);
    }
}

// ------------------------------------------------------------------ ports
// Applies the affine port map to a port cell's streamed populations; returns
// the exchanged mass (ports.rs:560-579).
template <int Q>
__device__ __forceinline__ float apply_port(const PortMap& P, float (&g)[Q]) {
    float in[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) in[q] = g[q];
    float exch = 0.f;
    const uint32_t um = P.unknown_mask;
#pragma unroll
    for (int r = 0; r < Q; ++r) {
        if (um & (1u << r)) {
            float acc = P.bias[r];
#pragma unroll
            for (int k = 0; k < Q; ++k) acc = fmaf(P.jac[r][k], in[k], acc);
            exch += acc - in[r];
            g[r] = acc;
        }
    }
    return exch;
}

// lambda <- J^T lambda for a port cell (apply_ports_vjp, ports.rs:582-621).
template <int Q>
__device__ __forceinline__ void port_transpose(const PortMap& P, float (&v)[Q]) {
    float in[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) in[q] = v[q];
    const uint32_t um = P.unknown_mask;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
        float acc = (um & (1u << k)) ? 0.f : in[k];
#pragma unroll
        for (int r = 0; r < Q; ++r)
            if (um & (1u << r)) acc = fmaf(P.jac[r][k], in[r], acc);
        v[k] = acc;
    }
}

// ------------------------------------------------------------------ physics
struct Macro {
    float rp, rho, u[3], F[3];
};

// Implicit half-step Brinkman velocity and Guo force (solver.rs:190-196,
// moving/psm.rs:213-226 with zero solid velocity).
template <int Q>
__device__ __forceinline__ Macro macroscopic(const float (&g)[Q], float alpha, const Physics& P) {
    using L = Lat<Q>;
    Macro M;
    float rp = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        rp += g[q];
        if (L::cx(q)) jx += L::cx(q) * g[q];
        if (L::cy(q)) jy += L::cy(q) * g[q];
        if (L::cz(q)) jz += L::cz(q) * g[q];
    }
    M.rp = rp;
    M.rho = 1.f + rp;
    const float inv_s = 1.f / (1.f + 0.5f * alpha);
    const float inv_rho = 1.f / M.rho;
    M.u[0] = (jx * inv_rho + 0.5f * P.a[0]) * inv_s;
    M.u[1] = (jy * inv_rho + 0.5f * P.a[1]) * inv_s;
    M.u[2] = (jz * inv_rho + 0.5f * P.a[2]) * inv_s;
#pragma unroll
    for (int d = 0; d < 3; ++d) M.F[d] = M.rho * (P.a[d] - alpha * M.u[d]);
    return M;
}

template <int Q>
__device__ __forceinline__ float dotc(int q, const float (&v)[3]) {
    using L = Lat<Q>;
    float s = 0.f;
    if (L::cx(q)) s += L::cx(q) * v[0];
    if (L::cy(q)) s += L::cy(q) * v[1];
    if (L::cz(q)) s += L::cz(q) * v[2];
    return s;
}

// TRT collision in pair form (moving/collision.rs:457-488), in shifted
// variables g = f - w; BGK is the case om == omega.  MRT adds the rank-one
// corrections of the moments whose rate differs from the shear rate: the
// odd moments of the Gram-Schmidt basis span exactly the antisymmetric
// subspace, so MRT with all even rates equal to omega is TRT.
template <int Q, int COLL>
__device__ __forceinline__ void collide(float (&g)[Q], const Macro& M, const Physics& P) {
    using L = Lat<Q>;
    const float om = P.omega, omm = P.om;
    const float kp = 1.f - 0.5f * om, km = 1.f - 0.5f * omm;
    const float* u = M.u;
    const float* F = M.F;
    const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const float uf = u[0] * F[0] + u[1] * F[1] + u[2] * F[2];
    const float rho = M.rho, rp = M.rp;
    float dproj[MAX_PROJ];
    if constexpr (COLL == CK_MRT) {
#pragma unroll
        for (int p = 0; p < MAX_PROJ; ++p) dproj[p] = 0.f;
    }
    {
        const float w0 = L::w(0);
        const float geq = w0 * (rp - 1.5f * rho * usq);
        const float src = -3.f * w0 * uf;
        if constexpr (COLL == CK_MRT) {
            const float y0 = g[0] - geq + 0.5f * src;
#pragma unroll
            for (int p = 0; p < MAX_PROJ; ++p)
                if (p < P.n_proj) dproj[p] = fmaf(P.proj_right[p][0], y0, dproj[p]);
        }
        g[0] = g[0] - om * (g[0] - geq) + kp * src;
    }
#pragma unroll
    for (int i = 1; i <= L::NPAIR; ++i) {
        const int o = opp<Q>(i);
        const float w = L::w(i);
        const float cu = dotc<Q>(i, M.u);
        const float cf = dotc<Q>(i, M.F);
        const float geqp = w * (rp + rho * (4.5f * cu * cu - 1.5f * usq));
        const float eqm = 3.f * rho * w * cu;
        const float sp = w * (9.f * cu * cf - 3.f * uf);
        const float sm = 3.f * w * cf;
        const float gp = 0.5f * (g[i] + g[o]);
        const float gm = 0.5f * (g[i] - g[o]);
        if constexpr (COLL == CK_MRT) {
            const float yp = gp - geqp + 0.5f * sp;
#pragma unroll
            for (int p = 0; p < MAX_PROJ; ++p)
                if (p < P.n_proj) dproj[p] = fmaf(2.f * P.proj_right[p][i], yp, dproj[p]);
        }
        const float A = kp * sp - om * (gp - geqp);
        const float Bv = km * sm - omm * (gm - eqm);
        g[i] = g[i] + A + Bv;
        g[o] = g[o] + A - Bv;
    }
    if constexpr (COLL == CK_MRT) {
#pragma unroll
        for (int p = 0; p < MAX_PROJ; ++p) {
            if (p < P.n_proj) {
                const float c = P.proj_rate[p] * dproj[p];
#pragma unroll
                for (int i = 0; i < Q; ++i) g[i] = fmaf(-c, P.proj_left[p][i], g[i]);
            }
        }
    }
}

// Collision transpose at the recorded (rho, u): given gb = d(loss)/d(post),
// returns d(loss)/d(f) in gb and d(loss)/d(alpha).  Derivation: post = f - R y
// + src, y = f - eq(rho, u) + src(u, F)/2; the cotangents of eq and src only
// need the weighted zeroth, first and second moments of R^T gb, then the
// Brinkman chain F = rho (a - alpha u), u = (m/rho + a/2)/(1 + alpha/2).
template <int Q, int COLL>
__device__ __forceinline__ float collide_vjp(float (&gb)[Q], float rp, const float (&u)[3], float alpha,
                                             const Physics& P) {
    using L = Lat<Q>;
    const float om = P.omega, omm = P.om;
    const float rho = 1.f + rp;
    const float s = 1.f + 0.5f * alpha;
    float F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d] = rho * (P.a[d] - alpha * u[d]);
    // z = R^T gb
    float z[Q];
    z[0] = om * gb[0];
#pragma unroll
    for (int i = 1; i <= L::NPAIR; ++i) {
        const int o = opp<Q>(i);
        const float p = 0.5f * (gb[i] + gb[o]), mm = 0.5f * (gb[i] - gb[o]);
        z[i] = om * p + omm * mm;
        z[o] = om * p - omm * mm;
    }
    if constexpr (COLL == CK_MRT) {
#pragma unroll
        for (int p = 0; p < MAX_PROJ; ++p) {
            if (p < P.n_proj) {
                float e = 0.f;
#pragma unroll
                for (int i = 0; i < Q; ++i) e = fmaf(P.proj_left[p][i], gb[i], e);
                const float c = P.proj_rate[p] * e;
#pragma unroll
                for (int i = 0; i < Q; ++i) z[i] = fmaf(c, P.proj_right[p][i], z[i]);
            }
        }
    }
    // weighted moments of z and of h = gb - z/2
    float Z0 = 0.f, Z1[3] = {0.f, 0.f, 0.f}, Z2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float H0 = 0.f, H1[3] = {0.f, 0.f, 0.f}, H2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const float w = L::w(i);
        const float zw = w * z[i];
        const float hw = w * (gb[i] - 0.5f * z[i]);
        const int c0 = L::cx(i), c1 = L::cy(i), c2 = L::cz(i);
        Z0 += zw;
        H0 += hw;
        if (c0) { Z1[0] += c0 * zw; H1[0] += c0 * hw; }
        if (c1) { Z1[1] += c1 * zw; H1[1] += c1 * hw; }
        if (c2) { Z1[2] += c2 * zw; H1[2] += c2 * hw; }
        if (c0) { Z2[0] += zw; H2[0] += hw; }
        if (c1) { Z2[1] += zw; H2[1] += hw; }
        if (c2) { Z2[2] += zw; H2[2] += hw; }
        if (c0 && c1) { Z2[3] += c0 * c1 * zw; H2[3] += c0 * c1 * hw; }
        if (c0 && c2) { Z2[4] += c0 * c2 * zw; H2[4] += c0 * c2 * hw; }
        if (c1 && c2) { Z2[5] += c1 * c2 * zw; H2[5] += c1 * c2 * hw; }
    }
    // Z2 u, H2 u, H2 F (symmetric 3x3 stored xx yy zz xy xz yz)
    auto mul = [](const float (&S)[6], const float* v, float* out) {
        out[0] = S[0] * v[0] + S[3] * v[1] + S[4] * v[2];
        out[1] = S[3] * v[0] + S[1] * v[1] + S[5] * v[2];
        out[2] = S[4] * v[0] + S[5] * v[1] + S[2] * v[2];
    };
    float Z2u[3], H2u[3], H2F[3];
    mul(Z2, u, Z2u);
    mul(H2, u, H2u);
    mul(H2, F, H2F);
    const float usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    float rho_bar = Z0 * (1.f - 1.5f * usq) + 3.f * (u[0] * Z1[0] + u[1] * Z1[1] + u[2] * Z1[2]) +
                    4.5f * (u[0] * Z2u[0] + u[1] * Z2u[1] + u[2] * Z2u[2]);
    float ub[3], Fb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ub[d] = rho * (3.f * Z1[d] + 9.f * Z2u[d] - 3.f * u[d] * Z0) + 9.f * H2F[d] - 3.f * F[d] * H0;
        Fb[d] = 3.f * H1[d] + 9.f * H2u[d] - 3.f * u[d] * H0;
    }
    float abar = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        rho_bar += Fb[d] * (P.a[d] - alpha * u[d]);
        abar -= rho * Fb[d] * u[d];
        ub[d] -= rho * alpha * Fb[d];
    }
    const float inv = 1.f / (s * rho);
    float mb[3];
    float sbar = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mb[d] = ub[d] * inv;
        rho_bar -= ub[d] * (s * u[d] - 0.5f * P.a[d]) * inv;
        sbar -= ub[d] * u[d] / s;
    }
    abar += 0.5f * sbar;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        float v = gb[i] - z[i] + rho_bar;
        if (L::cx(i)) v += L::cx(i) * mb[0];
        if (L::cy(i)) v += L::cy(i) * mb[1];
        if (L::cz(i)) v += L::cz(i) * mb[2];
        gb[i] = v;
    }
    return abar;
}

// ------------------------------------------------------------------ reductions
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}
// (h, l) += (h2, l2), compensated
__device__ __forceinline__ void dd_add(double& h, double& l, double h2, double l2) {
    double s, e;
    two_sum(h, h2, s, e);
    e += l + l2;
    h = s + e;
    l = e - (h - s);
}

struct DiagAcc {
    double mh, ml, eh, el;
    float minf, maxu2;
    int nf;
    __device__ void init() {
        mh = ml = eh = el = 0.0;
        minf = INFINITY;
        maxu2 = 0.f;
        nf = 0;
    }
    __device__ void merge(const DiagAcc& o) {
        dd_add(mh, ml, o.mh, o.ml);
        dd_add(eh, el, o.eh, o.el);
        minf = fminf(minf, o.minf);
        maxu2 = fmaxf(maxu2, o.maxu2);
        nf |= o.nf;
    }
    __device__ void shfl_merge(int off) {
        DiagAcc o;
        o.mh = __shfl_down_sync(FULL, mh, off);
        o.ml = __shfl_down_sync(FULL, ml, off);
        o.eh = __shfl_down_sync(FULL, eh, off);
        o.el = __shfl_down_sync(FULL, el, off);
        o.minf = __shfl_down_sync(FULL, minf, off);
        o.maxu2 = __shfl_down_sync(FULL, maxu2, off);
        o.nf = __shfl_down_sync(FULL, nf, off);
        merge(o);
    }
};

__device__ DiagAcc block_reduce(DiagAcc v) {
    __shared__ DiagAcc sh[BLOCK / 32];
    for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        if (lane < BLOCK / 32) v = sh[lane];
        else v.init();
        for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    }
    return v;
}

// Writes one block's partial, and lets the last block to finish combine all
// partials in a fixed order (deterministic) into *out.  No block waits.
__device__ void finish_diag(DiagAcc v, StepDiag* out, const Reduce& red) {
    __shared__ bool last;
    v = block_reduce(v);
    if (threadIdx.x == 0) {
        double* p = red.partial + (size_t)blockIdx.x * 8;
        p[0] = v.mh;
        p[1] = v.ml;
        p[2] = v.eh;
        p[3] = v.el;
        p[4] = v.minf;
        p[5] = v.maxu2;
        p[6] = v.nf;
        __threadfence();
        unsigned t = atomicAdd(red.counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    DiagAcc acc;
    acc.init();
    for (unsigned b = threadIdx.x; b < gridDim.x; b += BLOCK) {
        const double* p = red.partial + (size_t)b * 8;
        DiagAcc o;
        o.mh = __ldcg(p + 0);
        o.ml = __ldcg(p + 1);
        o.eh = __ldcg(p + 2);
        o.el = __ldcg(p + 3);
        o.minf = (float)__ldcg(p + 4);
        o.maxu2 = (float)__ldcg(p + 5);
        o.nf = (int)__ldcg(p + 6);
        acc.merge(o);
    }
    acc = block_reduce(acc);
    if (threadIdx.x == 0) {
        out->mass_hi = acc.mh;
        out->mass_lo = acc.ml;
        out->exch_hi = acc.eh;
        out->exch_lo = acc.el;
        out->min_f = acc.minf;
        out->max_u2 = acc.maxu2;
        out->nonfinite = acc.nf;
        *red.counter = 0;
        __threadfence();
    }
}

// NS compensated double sums.
template <int NS>
struct Sums {
    double h[NS], l[NS];
    __device__ void init() {
#pragma unroll
        for (int k = 0; k < NS; ++k) h[k] = l[k] = 0.0;
    }
    __device__ void add(int k, double v) { dd_add(h[k], l[k], v, 0.0); }
    __device__ void merge(const Sums& o) {
#pragma unroll
        for (int k = 0; k < NS; ++k) dd_add(h[k], l[k], o.h[k], o.l[k]);
    }
    __device__ void shfl_merge(int off) {
        Sums o;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            o.h[k] = __shfl_down_sync(FULL, h[k], off);
            o.l[k] = __shfl_down_sync(FULL, l[k], off);
        }
        merge(o);
    }
};

template <int NS>
__device__ Sums<NS> block_reduce_sums(Sums<NS> v) {
    __shared__ Sums<NS> sh[BLOCK / 32];
    for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        if (lane < BLOCK / 32) v = sh[lane];
        else v.init();
        for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    }
    return v;
}

template <int NS>
__device__ void finish_sums(Sums<NS> v, double* out, const Reduce& red) {
    __shared__ bool last;
    v = block_reduce_sums<NS>(v);
    if (threadIdx.x == 0) {
        double* p = red.partial + (size_t)blockIdx.x * 2 * NS;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            p[2 * k] = v.h[k];
            p[2 * k + 1] = v.l[k];
        }
        __threadfence();
        unsigned t = atomicAdd(red.counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    Sums<NS> acc;
    acc.init();
    for (unsigned b = threadIdx.x; b < gridDim.x; b += BLOCK) {
        const double* p = red.partial + (size_t)b * 2 * NS;
        Sums<NS> o;
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            o.h[k] = __ldcg(p + 2 * k);
            o.l[k] = __ldcg(p + 2 * k + 1);
        }
        acc.merge(o);
    }
    acc = block_reduce_sums<NS>(acc);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            out[2 * k] = acc.h[k];
            out[2 * k + 1] = acc.l[k];
        }
        *red.counter = 0;
        __threadfence();
    }
}

// ------------------------------------------------------------------ kernels
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_init(Geometry G, Physics P, T* A, const uint32_t* __restrict__ mask) {
    using L = Lat<Q>;
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
        const bool solid = mask[x] & MASK_SOLID;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            // initial_populations, solver.rs:593-601: fluid w(1 - 1.5 c.a), solid w
            const float ca = L::cx(q) * P.a[0] + L::cy(q) * P.a[1] + L::cz(q) * P.a[2];
            const float g = solid ? 0.f : -1.5f * L::w(q) * ca;
            A[(int64_t)q * G.n + x] = penc<Q, T>(g, q);
        }
    }
}

// One fused step: load (AA parity) -> port reconstruction -> admission
// reductions of the loaded state -> collision -> AA store.
template <int Q, int COLL, typename T>
__global__ void __launch_bounds__(BLOCK) k_forward(FwdArgs a) {
    using L = Lat<Q>;
    T* A = static_cast<T*>(a.pop);
    DiagAcc acc;
    acc.init();
    const int64_t n = a.G.n;
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < n; x += (int64_t)gridDim.x * BLOCK) {
        const uint32_t m = a.mask[x];
        if (m & MASK_SOLID) continue;
        float g[Q];
        load_pop<Q, T>(A, a.G, x, m, a.parity, g);
        float exch = 0.f;
        if (a.apply_ports && (m & MASK_PORT)) exch = apply_port<Q>(a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], g);
        const float alpha = a.alpha[x];
        Macro M = macroscopic<Q>(g, alpha, a.P);
        if (a.diag) {
            acc.mh += (double)M.rp;
            acc.eh += (double)exch;
            float mn = INFINITY;
            bool fin = true;
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float f = L::w(q) + g[q];
                mn = fminf(mn, f);
                fin = fin && isfinite(g[q]);
            }
            acc.minf = fminf(acc.minf, mn);
            acc.maxu2 = fmaxf(acc.maxu2, M.u[0] * M.u[0] + M.u[1] * M.u[1] + M.u[2] * M.u[2]);
            if (!fin) acc.nf = 1;
        }
        if (a.record) {
            a.record[x] = M.rp;
            a.record[n + x] = M.u[0];
            a.record[2 * n + x] = M.u[1];
            a.record[3 * n + x] = M.u[2];
        }
        if (a.collide) {
            collide<Q, COLL>(g, M, a.P);
            store_pop<Q, T>(A, a.G, x, m, a.parity, g);
        }
    }
    if (a.diag) finish_diag(acc, a.diag, a.red);
}

template <int Q, int COLL, typename T>
__global__ void __launch_bounds__(BLOCK) k_adjoint(AdjArgs a) {
    T* B = static_cast<T*>(a.lam);
    const int64_t n = a.G.n;
    double nsum = 0.0;
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < n; x += (int64_t)gridDim.x * BLOCK) {
        const uint32_t m = a.mask[x];
        if (m & MASK_SOLID) continue;
        float v[Q];
        load_lam<Q, T>(B, a.G, x, m, a.parity, a.in_scale_inv, v);
        const float rp = a.record[x];
        const float u[3] = {a.record[n + x], a.record[2 * n + x], a.record[3 * n + x]};
        const float alpha = a.alpha[x];
        const float ab = collide_vjp<Q, COLL>(v, rp, u, alpha, a.P);
        if (a.overwrite_abar) a.abar[x] = ab * a.abar_factor;
        else a.abar[x] = fmaf(ab, a.abar_factor, a.abar[x]);
        if (a.port_transpose && (m & MASK_PORT)) port_transpose<Q>(a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], v);
        store_lam<Q, T>(B, a.G, x, m, a.parity, a.out_scale, v);
        if (a.norm2) {
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float s = v[q] * a.out_scale;
                nsum += (double)s * (double)s;
            }
        }
    }
    if (a.norm2) {
        Sums<1> s;
        s.init();
        s.h[0] = nsum;
        finish_sums<1>(s, a.norm2, a.red);
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
    const float k = 1.f - 0.5f / a.tau;
    const float nu = (a.tau - 0.5f) / 3.f;
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < n; x += (int64_t)gridDim.x * BLOCK) {
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
        load_pop<Q, T>(A, a.G, x, m, a.parity, g);
        const PortMap* pm = (m & MASK_PORT) ? &a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1] : nullptr;
        if (a.apply_ports && pm) apply_port<Q>(*pm, g);
        const float alpha = a.alpha[x];
        Macro M = macroscopic<Q>(g, alpha, a.P);
        // second moments of g: M2_ab = sum c_a c_b g (f adds delta/3)
        float S[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
            if (c0) S[0] += g[q];
            if (c1) S[1] += g[q];
            if (c2) S[2] += g[q];
            if (c0 && c1) S[3] += c0 * c1 * g[q];
            if (c0 && c2) S[4] += c0 * c2 * g[q];
            if (c1 && c2) S[5] += c1 * c2 * g[q];
        }
        const float* u = M.u;
        const float* F = M.F;
        const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
        float sig[6];
        float ss = 0.f;
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const float pi = S[e] - (e < 3 ? M.rp / 3.f : 0.f) - M.rho * u[ia[e]] * u[ib[e]];
            const float t = 0.5f * (u[ia[e]] * F[ib[e]] + u[ib[e]] * F[ia[e]]);
            sig[e] = -k * (pi + t);
            ss += (e < 3 ? 1.f : 2.f) * sig[e] * sig[e];
        }
        const float dpw = pm ? pm->dp_weight : 0.f;
        if constexpr (MODE == 0) {
            const float U[3] = {u[0] * a.vel, u[1] * a.vel, u[2] * a.vel};
            const double R = (double)M.rho * a.dens;
            const double usq = (double)U[0] * U[0] + (double)U[1] * U[1] + (double)U[2] * U[2];
            acc.add(0, U[0]);
            acc.add(1, U[1]);
            acc.add(2, U[2]);
            acc.add(3, R * usq);
            acc.add(4, R * alpha / a.dt_s * usq);
            acc.add(5, (double)a.phi[x]);
            if (pm) acc.add(6, (double)dpw * a.dens * (double)M.rp * a.vel * a.vel / 3.0);
            acc.add(7, (double)ss / (2.0 * M.rho * nu));
            if (a.fields) {
                a.fields[x] = M.rp;
                a.fields[n + x] = u[0];
                a.fields[2 * n + x] = u[1];
                a.fields[3 * n + x] = u[2];
            }
        } else {
            // cotangents of rho, u, F, M2 (all lattice units)
            const float V = a.vel;
            const float U[3] = {u[0] * V, u[1] * V, u[2] * V};
            const float usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
            const float R = M.rho * a.dens;
            const float W3 = (float)a.w[3], W4 = (float)a.w[4], W7 = (float)a.w[7];
            float rb = 0.f, abar = 0.f, ub[3], Fb[3] = {0.f, 0.f, 0.f}, Sb[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            const float kin = W3 + W4 * alpha / a.dt_s;
#pragma unroll
            for (int d = 0; d < 3; ++d) ub[d] = (float)a.w[d] * V + kin * R * 2.f * U[d] * V;
            rb += kin * a.dens * usq;
            abar += W4 * R / a.dt_s * usq;
            if (pm) rb += (float)a.w[6] * dpw * a.dens * V * V / 3.f;
            if (W7 != 0.f) {
                rb += -W7 * ss / (2.f * M.rho * M.rho * nu);
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    const float mult = (e < 3 ? 1.f : 2.f);  // off-diagonals appear twice
                    const float pb = -k * W7 * sig[e] / (M.rho * nu) * mult;
                    const int i0 = ia[e], i1 = ib[e];
                    Sb[e] += pb;
                    rb -= pb * ((e < 3 ? 1.f / 3.f : 0.f) + u[i0] * u[i1]);
                    if (e < 3) {
                        ub[i0] -= 2.f * M.rho * pb * u[i0];
                        ub[i0] += pb * F[i0];
                        Fb[i0] += pb * u[i0];
                    } else {
                        ub[i0] -= M.rho * pb * u[i1];
                        ub[i1] -= M.rho * pb * u[i0];
                        ub[i0] += 0.5f * pb * F[i1];
                        ub[i1] += 0.5f * pb * F[i0];
                        Fb[i1] += 0.5f * pb * u[i0];
                        Fb[i0] += 0.5f * pb * u[i1];
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                rb += Fb[d] * (a.P.a[d] - alpha * u[d]);
                abar -= Fb[d] * M.rho * u[d];
                ub[d] -= Fb[d] * M.rho * alpha;
            }
            const float s = 1.f + 0.5f * alpha;
            const float inv = 1.f / (s * M.rho);
            float mb[3], sbar = 0.f;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                mb[d] = ub[d] * inv;
                rb -= ub[d] * (s * u[d] - 0.5f * a.P.a[d]) * inv;
                sbar -= ub[d] * u[d] / s;
            }
            abar += 0.5f * sbar;
            float fb[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int c0 = L::cx(q), c1 = L::cy(q), c2 = L::cz(q);
                float v = rb;
                if (c0) v += c0 * mb[0] + Sb[0];
                if (c1) v += c1 * mb[1] + Sb[1];
                if (c2) v += c2 * mb[2] + Sb[2];
                if (c0 && c1) v += c0 * c1 * Sb[3];
                if (c0 && c2) v += c0 * c2 * Sb[4];
                if (c1 && c2) v += c1 * c2 * Sb[5];
                fb[q] = v;
            }
            a.abar_final[x] = abar;
            a.phibar[x] = (float)a.w[5];
            if (a.record) {
                a.record[x] = M.rp;
                a.record[n + x] = u[0];
                a.record[2 * n + x] = u[1];
                a.record[3 * n + x] = u[2];
            }
            if (a.port_transpose && pm) port_transpose<Q>(*pm, fb);
            if (a.write_lambda) {
                TL* B = static_cast<TL*>(a.lam);
#pragma unroll
                for (int q = 0; q < Q; ++q) B[opp<Q>(q) * n + x] = Cvt<TL>::from(fb[q] * a.lam_scale);
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

template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_canon_pop(Geometry G, const T* A, const uint32_t* __restrict__ mask,
                                                     const PortMap* ports, int parity, int apply_ports, float* out) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
        float g[Q];
        if (m & MASK_SOLID) {
#pragma unroll
            for (int q = 0; q < Q; ++q) g[q] = pdec<Q, T>(A[(int64_t)q * G.n + x], q);
        } else {
            load_pop<Q, T>(A, G, x, m, parity, g);
            if (apply_ports && (m & MASK_PORT)) apply_port<Q>(ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], g);
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) out[(int64_t)q * G.n + x] = g[q];
    }
}

template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_upload_pop(Geometry G, T* A, const float* in) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
#pragma unroll
        for (int q = 0; q < Q; ++q) A[(int64_t)q * G.n + x] = penc<Q, T>(in[(int64_t)q * G.n + x], q);
    }
}

// Natural-order lambda after an adjoint step (after_odd) or after a seed /
// parity-0 adjoint step.
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_canon_lam(Geometry G, const T* B, const uint32_t* __restrict__ mask,
                                                     int after_odd, float inv_scale, float* out) {
    using L = Lat<Q>;
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            float v = 0.f;
            if (!(m & MASK_SOLID)) {
                int64_t idx;
                if (!after_odd || (m & (1u << q))) idx = opp<Q>(q) * G.n + x;
                else idx = (int64_t)q * G.n + neighbor(G, x, m, -L::cx(q), -L::cy(q), -L::cz(q));
                v = Cvt<T>::to(B[idx]) * inv_scale;
            }
            out[(int64_t)q * G.n + x] = v;
        }
    }
}

// Natural lambda (cotangent of the post-port state) -> stored seed layout.
template <int Q, typename T>
__global__ void __launch_bounds__(BLOCK) k_seed_lam(Geometry G, T* B, const uint32_t* __restrict__ mask,
                                                    const PortMap* ports, const float* in, float scale,
                                                    int port_transpose_on) {
    for (int64_t x = (int64_t)blockIdx.x * BLOCK + threadIdx.x; x < G.n; x += (int64_t)gridDim.x * BLOCK) {
        const uint32_t m = mask[x];
        if (m & MASK_SOLID) continue;
        float v[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] = in[(int64_t)q * G.n + x];
        if (port_transpose_on && (m & MASK_PORT)) port_transpose<Q>(ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], v);
#pragma unroll
        for (int q = 0; q < Q; ++q) B[opp<Q>(q) * G.n + x] = Cvt<T>::from(v[q] * scale);
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

// ------------------------------------------------------------------ launchers
#define LBM_STORAGE_DISPATCH(storage, T, ...)            \
    switch (storage) {                                   \
        case ST_F32: {                                   \
            using T = float;                             \
            __VA_ARGS__;                                 \
            break;                                       \
        }                                                \
        case ST_F16: {                                   \
            using T = __half;                            \
            __VA_ARGS__;                                 \
            break;                                       \
        }                                                \
        default: {                                       \
            using T = __nv_bfloat16;                     \
            __VA_ARGS__;                                 \
            break;                                       \
        }                                                \
    }

static int blocks_for(int64_t n, int cap) {
    int64_t b = (n + BLOCK - 1) / BLOCK;
    if (cap > 0 && b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

cudaError_t launch_init(int Q, int storage, const Geometry& G, const Physics& P, void* pop, const uint32_t* mask,
                        cudaStream_t s) {
    const int grid = blocks_for(G.n, 0);
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T, k_init<19, T><<<grid, BLOCK, 0, s>>>(G, P, static_cast<T*>(pop), mask))
    } else {
        LBM_STORAGE_DISPATCH(storage, T, k_init<27, T><<<grid, BLOCK, 0, s>>>(G, P, static_cast<T*>(pop), mask))
    }
    return cudaGetLastError();
}

cudaError_t launch_forward(int Q, int coll, int storage, const FwdArgs& a, int grid, cudaStream_t s) {
    if (Q == 19) {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(storage, T, k_forward<19, CK_MRT, T><<<grid, BLOCK, 0, s>>>(a))
        } else {
            LBM_STORAGE_DISPATCH(storage, T, k_forward<19, CK_PAIRS, T><<<grid, BLOCK, 0, s>>>(a))
        }
    } else {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(storage, T, k_forward<27, CK_MRT, T><<<grid, BLOCK, 0, s>>>(a))
        } else {
            LBM_STORAGE_DISPATCH(storage, T, k_forward<27, CK_PAIRS, T><<<grid, BLOCK, 0, s>>>(a))
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_adjoint(int Q, int coll, int lstorage, const AdjArgs& a, int grid, cudaStream_t s) {
    if (Q == 19) {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(lstorage, T, k_adjoint<19, CK_MRT, T><<<grid, BLOCK, 0, s>>>(a))
        } else {
            LBM_STORAGE_DISPATCH(lstorage, T, k_adjoint<19, CK_PAIRS, T><<<grid, BLOCK, 0, s>>>(a))
        }
    } else {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(lstorage, T, k_adjoint<27, CK_MRT, T><<<grid, BLOCK, 0, s>>>(a))
        } else {
            LBM_STORAGE_DISPATCH(lstorage, T, k_adjoint<27, CK_PAIRS, T><<<grid, BLOCK, 0, s>>>(a))
        }
    }
    return cudaGetLastError();
}

template <int Q, typename T>
static void objective_dispatch(int lstorage, int mode, const ObjArgs& a, int grid, cudaStream_t s) {
    if (mode == 0) {
        k_objective<Q, T, float, 0><<<grid, BLOCK, 0, s>>>(a);
    } else {
        LBM_STORAGE_DISPATCH(lstorage, TL, k_objective<Q, T, TL, 1><<<grid, BLOCK, 0, s>>>(a))
    }
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
                             const PortMap* ports, int parity, int apply_ports, float* out, int grid,
                             cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_canon_pop<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(pop), mask, ports,
                                                                        parity, apply_ports, out))
    } else {
        LBM_STORAGE_DISPATCH(storage, T,
                             k_canon_pop<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(pop), mask, ports,
                                                                        parity, apply_ports, out))
    }
    return cudaGetLastError();
}

cudaError_t launch_upload_pop(int Q, int storage, const Geometry& G, void* pop, const float* in, int grid,
                              cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(storage, T, k_upload_pop<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(pop), in))
    } else {
        LBM_STORAGE_DISPATCH(storage, T, k_upload_pop<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(pop), in))
    }
    return cudaGetLastError();
}

cudaError_t launch_canon_lam(int Q, int lstorage, const Geometry& G, const void* lam, const uint32_t* mask,
                             int after_odd, float inv_scale, float* out, int grid, cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_canon_lam<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(lam), mask,
                                                                        after_odd, inv_scale, out))
    } else {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_canon_lam<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<const T*>(lam), mask,
                                                                        after_odd, inv_scale, out))
    }
    return cudaGetLastError();
}

cudaError_t launch_seed_lam(int Q, int lstorage, const Geometry& G, void* lam, const uint32_t* mask,
                            const PortMap* ports, const float* in, float scale, int port_transpose_on, int grid,
                            cudaStream_t s) {
    if (Q == 19) {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_seed_lam<19, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(lam), mask, ports, in,
                                                                       scale, port_transpose_on))
    } else {
        LBM_STORAGE_DISPATCH(lstorage, T,
                             k_seed_lam<27, T><<<grid, BLOCK, 0, s>>>(G, static_cast<T*>(lam), mask, ports, in,
                                                                       scale, port_transpose_on))
    }
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
