// lbm_device.cuh -- device building blocks shared by the sm_100a kernels
// (lbm_forward.cu, lbm_adjoint.cu, lbm_misc.cu): storage conversions, pull
// addressing, port maps, the collision and its transpose, compensated
// reductions, and launch helpers.
//
// Memory layout (all on one GPU):
//   populations  two arrays (current, next), each Q planes of n cells, plane q
//                at pop + q*n; cells in the reference Grid order
//                (i*ny + j)*nz + k, so axis 2 is the contiguous one.  FP32
//                stores g = f - w; FP16/BF16 store g/w.
//   mask         one uint32 per cell (lbm_common.cuh)
//   alpha, phi   FP32 per cell
//   lambda       two arrays of Q planes, adjoint populations (FP32/FP16/BF16,
//                global scale)
//   record       4 FP32 planes (rho-1, u) of the forward state the adjoint
//                linearises at
//
// Streaming is a pull between the two arrays (see pull_index below): a step
// reads the post-collision populations streaming in from the neighbours of
// the current array and writes the cell's own slots of the other one.  A
// blocked link (halfway bounce-back, Streaming::new solver.rs:84-119) reads
// the cell's own opposite slot instead.  The adjoint transposes the pull:
// the same pattern with the velocities reversed (pull from x + c_q),
// linearised at a recorded (rho, u).
#pragma once
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <mutex>
#include <unordered_map>

#include "lbm_launch.h"
#include "lbm_tma.cuh"

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

// Stochastic rounding to the 16-bit formats: FP16 through the hardware's
// stochastic-rounding conversion; BF16 (FP32's exponent range, so no
// subnormal halves to care about) by adding uniform random bits below the
// kept mantissa and truncating.  A nearly steady state is re-rounded
// every step; with round-to-nearest the same rounding errors repeat and the
// mass drifts linearly in time, with stochastic rounding they average out.
template <typename T>
__device__ __forceinline__ T round_stochastic(float v, uint32_t r);
template <>
__device__ __forceinline__ __half round_stochastic<__half>(float v, uint32_t r) {
    // the hardware stochastic rounding (cvt.rs) drops the right number of
    // bits for subnormal halves too, where adding a fixed 13 random bits
    // below the normal mantissa would bias the result toward zero
    // (r ^ r >> 16: the LCG's high bits reach both halves of the word)
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(0.f), "f"(v), "r"(r ^ (r >> 16)));
    return __ushort_as_half((unsigned short)(d & 0xffffu));
}
template <>
__device__ __forceinline__ __nv_bfloat16 round_stochastic<__nv_bfloat16>(float v, uint32_t r) {
    return __float2bfloat16_rz(__uint_as_float(__float_as_uint(v) + (r >> 16)));  // 16 dropped bits
}

// Per-cell random stream: one integer hash of (cell, absolute step), then an
// LCG step per stored value (its high bits feed the rounding).  Deterministic,
// so recomputation from a checkpoint reproduces the stored states exactly.
__device__ __forceinline__ uint32_t cell_seed(uint32_t x, uint32_t step) {
    uint32_t h = x * 0x9E3779B1u ^ (step + 0x632BE5ABu) * 0x85EBCA77u;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}
__device__ __forceinline__ uint32_t lcg(uint32_t& s) {
    s = s * 1664525u + 1013904223u;
    return s;
}

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
template <int Q, typename T>
__device__ __forceinline__ T penc_sr(float g, int q, uint32_t& rs) {
    if constexpr (Cvt<T>::scaled) return round_stochastic<T>(g * (float)(1.0 / Lat<Q>::wd(q)), lcg(rs));
    else return Cvt<T>::from(g);
}

// Stored element <-> value in storage units: g = f - w for FP32, the
// weight-relative (f - w)/w for the 16-bit formats (the stepping kernels
// compute in these units, in which the 16-bit collision needs no weights).
template <typename T>
__device__ __forceinline__ float sdec(T v) {
    return Cvt<T>::to(v);
}
template <typename T>
__device__ __forceinline__ T senc_sr(float v, uint32_t& rs) {
    if constexpr (Cvt<T>::scaled) return round_stochastic<T>(v, lcg(rs));
    else return Cvt<T>::from(v);
}

// Two values to FP16 with stochastic rounding in one conversion (sm_100a
// cvt.rs): `hi` lands in the upper half, `lo` in the lower, each rounded
// with random bits taken from rbits.
__device__ __forceinline__ uint32_t sr_half2(float hi, float lo, uint32_t rbits) {
    uint32_t d;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(hi), "f"(lo), "r"(rbits));
    return d;
}

// All Q values of a cell in storage units -> stored elements, handed to
// put(q, element).  FP16 converts the directions in pairs (one random word
// per pair); the other formats one by one.
template <int Q, typename T, typename Put>
__device__ __forceinline__ void senc_sr_all(const float (&v)[Q], uint32_t& rs, Put&& put) {
    if constexpr (std::is_same<T, __half>::value) {
#pragma unroll
        for (int q = 0; q + 1 < Q; q += 2) {
            const uint32_t d = sr_half2(v[q + 1], v[q], lcg(rs));
            put(q, __ushort_as_half((unsigned short)(d & 0xffffu)));
            put(q + 1, __ushort_as_half((unsigned short)(d >> 16)));
        }
        if constexpr (Q % 2) put(Q - 1, round_stochastic<T>(v[Q - 1], lcg(rs)));
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) put(q, senc_sr<T>(v[q], rs));
    }
}

// ------------------------------------------------------------------ indexing
// All population indices q*n + x fit in 32 bits (the runtime checks
// Q*n < 2^32), which keeps the per-direction address arithmetic in 32-bit
// integer units.
__device__ __forceinline__ uint32_t neighbor(const Geometry& G, uint32_t x, uint32_t m, int dx, int dy, int dz) {
    if (!(m & MASK_WRAP)) return x + (uint32_t)(dx * (int)G.sx + dy * (int)G.sy + dz);
    int k = (int)(x % (uint32_t)G.nz);
    uint32_t ij = x / (uint32_t)G.nz;
    int j = (int)(ij % (uint32_t)G.ny);
    int i = (int)(ij / (uint32_t)G.ny);
    i += dx;
    j += dy;
    k += dz;
    if (i < 0) i += G.nx;
    else if (i >= G.nx) i -= G.nx;
    if (j < 0) j += G.ny;
    else if (j >= G.ny) j -= G.ny;
    if (k < 0) k += G.nz;
    else if (k >= G.nz) k -= G.nz;
    return ((uint32_t)i * (uint32_t)G.ny + (uint32_t)j) * (uint32_t)G.nz + (uint32_t)k;
}

__device__ __forceinline__ void coords(const Geometry& G, int64_t x, int64_t& i, int64_t& j, int64_t& k) {
    k = x % G.nz;
    int64_t ij = x / G.nz;
    j = ij % G.ny;
    i = ij / G.ny;
}

// Linear offset of the neighbour x + sign*c_q (no wrap): a constant per direction.
template <int Q>
__device__ __forceinline__ uint32_t lin(const Geometry& G, int q, int sign) {
    using L = Lat<Q>;
    return (uint32_t)(sign * (L::cx(q) * (int)G.sx + L::cy(q) * (int)G.sy + L::cz(q)));
}

// Two population arrays, each Q planes of n cells.  The current array holds
// the post-collision populations f*: slot (q, x) = f*_q(x).  One step pulls
// (Streaming::stream, solver.rs:131-157): f_q(x) = f*_q(x - c_q), or the
// halfway bounce-back f*_opp(q)(x) when x - c_q is a wall or solid (mask bit
// q); it collides and writes f*'_q(x) to slot (q, x) of the other array.
// Every slot of the current array is read by exactly one (cell, direction),
// so the inverse of the pull (loading a given streamed state) is a scatter
// through the same index.  Solid cells are never stepped: their own slots
// hold their populations in both arrays.
template <int Q>
__device__ __forceinline__ uint32_t pull_index(const Geometry& G, uint32_t x, uint32_t m, int q) {
    using L = Lat<Q>;
    const uint32_t n = (uint32_t)G.n;
    if (m & (1u << q)) return opp<Q>(q) * n + x;
    if (!(m & MASK_WRAP)) return q * n + x + lin<Q>(G, q, -1);
    return q * n + neighbor(G, x, m, -L::cx(q), -L::cy(q), -L::cz(q));
}

// Transposed pull of the adjoint step: the cotangent of f*_q(y) gathers from
// (q, y + c_q), or from the own slot opp(q) when y + c_q is a wall or solid
// (mask bit opp(q)).
template <int Q>
__device__ __forceinline__ uint32_t pull_adj_index(const Geometry& G, uint32_t x, uint32_t m, int q) {
    using L = Lat<Q>;
    const uint32_t n = (uint32_t)G.n;
    if (m & (1u << opp<Q>(q))) return opp<Q>(q) * n + x;
    if (!(m & MASK_WRAP)) return q * n + x + lin<Q>(G, q, +1);
    return q * n + neighbor(G, x, m, L::cx(q), L::cy(q), L::cz(q));
}

// Streamed populations of a fluid cell (g = f - w).
template <int Q, typename T>
__device__ __forceinline__ void load_pop(const T* __restrict__ A, const Geometry& G, uint32_t x, uint32_t m,
                                         float (&g)[Q]) {
#pragma unroll
    for (int q = 0; q < Q; ++q) g[q] = pdec<Q, T>(A[pull_index<Q>(G, x, m, q)], q);
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

// ------------------------------------------------------------------ extrapolating ports
// Non-equilibrium extrapolation from the inward neighbour x + nb_off
// (ports.rs reconstruct_neighbor :484-497; moving/boundary.rs
// port_populations :445-458): f = eq(rho_b, u_b) + f_n - eq(rho_n, u_n) with
// u_n = j_n / rho_n.  In shifted variables g = f - w the weights cancel:
// g = g_n + eq(rho_b, u_b) - eq(rho_n, u_n).  R is float or double.
template <typename R>
__device__ __forceinline__ void nee_targets(const PortMap& P, R rp_n, const R (&u_n)[3], R& rp_b, R (&u_b)[3]) {
    rp_b = P.rb_nb ? rp_n : (R)P.rb1;
#pragma unroll
    for (int d = 0; d < 3; ++d) u_b[d] = ((P.ub_nb >> d) & 1) ? u_n[d] : (R)P.u_port[d];
}

template <int Q, typename R>
__device__ __forceinline__ void nee_moments(const R (&gn)[Q], R& rp, R (&u)[3]) {
    using L = Lat<Q>;
    R j[3] = {0, 0, 0};
    rp = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        rp += gn[q];
        if (L::cx(q)) j[0] += L::cx(q) * gn[q];
        if (L::cy(q)) j[1] += L::cy(q) * gn[q];
        if (L::cz(q)) j[2] += L::cz(q) * gn[q];
    }
    const R inv = (R)1 / ((R)1 + rp);
#pragma unroll
    for (int d = 0; d < 3; ++d) u[d] = j[d] * inv;
}

// out <- the port cell's populations from the neighbour's streamed gn.
template <int Q, typename R>
__device__ __forceinline__ void nee_apply(const PortMap& P, const R (&gn)[Q], R (&out)[Q]) {
    using L = Lat<Q>;
    R rp, u[3], rb, ub[3];
    nee_moments<Q, R>(gn, rp, u);
    nee_targets<R>(P, rp, u, rb, ub);
    const R rho = (R)1 + rp, rho_b = (R)1 + rb;
    const R u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2], ub2 = ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const R cb = L::cx(q) * ub[0] + L::cy(q) * ub[1] + L::cz(q) * ub[2];
        const R cn = L::cx(q) * u[0] + L::cy(q) * u[1] + L::cz(q) * u[2];
        // eq_b - eq_n = w [(rho_b - rho_n) + rho_b (3 cb + 4.5 cb^2 - 1.5 ub^2) - rho_n (...)]
        const R d = (rb - rp) + rho_b * (3 * cb + (R)4.5 * cb * cb - (R)1.5 * ub2) -
                    rho * (3 * cn + (R)4.5 * cn * cn - (R)1.5 * u2);
        out[q] = gn[q] + (R)L::wd(q) * d;
    }
}

// v <- the cotangent of the neighbour's streamed populations given v, the
// cotangent of the port cell's populations, at the neighbour's (rho - 1, u)
// (port_populations_vjp, moving/boundary.rs:462-506, with
// equilibrium_vjp; the neighbor_non_equilibrium port's axial velocity
// follows the neighbour's the same way).
template <int Q>
__device__ __forceinline__ void nee_transpose(const PortMap& P, float rp_n, const float (&u_n)[3], float (&v)[Q]) {
    using L = Lat<Q>;
    float rb, ub[3];
    nee_targets<float>(P, rp_n, u_n, rb, ub);
    const float rho_n = 1.f + rp_n, rho_b = 1.f + rb;
    const float un2 = u_n[0] * u_n[0] + u_n[1] * u_n[1] + u_n[2] * u_n[2];
    const float ub2 = ub[0] * ub[0] + ub[1] * ub[1] + ub[2] * ub[2];
    float rbb = 0.f, rnb = 0.f, ubb[3] = {0.f, 0.f, 0.f}, unb[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float g = v[q] * L::w(q);
        const float cb = L::cx(q) * ub[0] + L::cy(q) * ub[1] + L::cz(q) * ub[2];
        const float cn = L::cx(q) * u_n[0] + L::cy(q) * u_n[1] + L::cz(q) * u_n[2];
        rbb += g * (1.f + 3.f * cb + 4.5f * cb * cb - 1.5f * ub2);
        rnb -= g * (1.f + 3.f * cn + 4.5f * cn * cn - 1.5f * un2);
        const float c[3] = {(float)L::cx(q), (float)L::cy(q), (float)L::cz(q)};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ubb[d] += g * (3.f * c[d] + 9.f * cb * c[d] - 3.f * ub[d]);
            unb[d] -= g * (3.f * c[d] + 9.f * cn * c[d] - 3.f * u_n[d]);
        }
    }
    if (P.rb_nb) rnb += rbb;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ubb[d] *= rho_b;
        unb[d] *= rho_n;
        if ((P.ub_nb >> d) & 1) unb[d] += ubb[d];
    }
    // u_n = j / rho_n: j_bar = u_bar / rho_n, rho_bar -= u_bar . u_n / rho_n
    const float inv = 1.f / rho_n;
    float jb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        jb[d] = unb[d] * inv;
        rnb -= unb[d] * u_n[d] * inv;
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) v[q] += rnb + L::cx(q) * jb[0] + L::cy(q) * jb[1] + L::cz(q) * jb[2];
}

// ------------------------------------------------------------------ regularized port
// Regularized known-stress port (ports.rs reconstruct_regularized :455-482):
// the legacy target fixes (rho, u); every population is replaced by
// eq(rho, u) + sum_r stress_r B_qr, with the deviatoric basis B_qr = 4.5 w_q
// (c_a c_b - delta_ab / 3) over (xx, yy, zz, 2xy, 2xz, 2yz) and the stress
// fitted to the known populations' non-equilibrium parts.
template <int Q>
__device__ __forceinline__ constexpr float stress_basis(int q, int r) {
    using L = Lat<Q>;
    const int c[3] = {L::cx(q), L::cy(q), L::cz(q)};
    const int ia = r < 3 ? r : (r == 5 ? 1 : 0);
    const int ib = r < 3 ? r : (r == 3 ? 1 : 2);
    const float qq = (float)(c[ia] * c[ib]) - (ia == ib ? 1.f / 3.f : 0.f);
    return 4.5f * L::w(q) * (r < 3 ? qq : 2.f * qq);
}

template <int Q>
__device__ __forceinline__ void regularized_apply(const PortMap& P, float (&g)[Q]) {
    using L = Lat<Q>;
    float t[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) t[q] = g[q];
    apply_port<Q>(P, t);
    float rp, u[3];
    nee_moments<Q, float>(t, rp, u);
    const float rho = 1.f + rp, u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    // e = eq - w in shifted variables
    float st[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const float cu = L::cx(q) * u[0] + L::cy(q) * u[1] + L::cz(q) * u[2];
        t[q] = L::w(q) * (rp + rho * (3.f * cu + 4.5f * cu * cu - 1.5f * u2));
        const float ne = g[q] - t[q];
#pragma unroll
        for (int r = 0; r < 6; ++r) st[r] = fmaf(P.sop[r][q], ne, st[r]);
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        float acc = t[q];
#pragma unroll
        for (int r = 0; r < 6; ++r) acc = fmaf(st[r], stress_basis<Q>(q, r), acc);
        g[q] = acc;
    }
}

// v <- the cotangent of the streamed populations given v, the cotangent of
// the rebuilt ones, at the rebuilt cell's (rho - 1, u): the map is nonlinear
// only through the legacy target's density and velocity, which the rebuilt
// cell carries unchanged (the stress basis has no mass or momentum).
template <int Q>
__device__ __forceinline__ void regularized_transpose(const PortMap& P, float rp, const float (&u)[3], float (&v)[Q]) {
    using L = Lat<Q>;
    float sb[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < 6; ++r) sb[r] = fmaf(v[q], stress_basis<Q>(q, r), sb[r]);
    const float rho = 1.f + rp, u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    float rb = 0.f, ub[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        float d = 0.f;
#pragma unroll
        for (int r = 0; r < 6; ++r) d = fmaf(sb[r], P.sop[r][q], d);
        // the stress reads the known populations directly (d) and the
        // equilibrium through -d
        const float eb = (v[q] - d) * L::w(q);
        v[q] = d;
        const float cu = L::cx(q) * u[0] + L::cy(q) * u[1] + L::cz(q) * u[2];
        rb += eb * (1.f + 3.f * cu + 4.5f * cu * cu - 1.5f * u2);
        const float c[3] = {(float)L::cx(q), (float)L::cy(q), (float)L::cz(q)};
#pragma unroll
        for (int k = 0; k < 3; ++k) ub[k] += eb * rho * (3.f * c[k] + 9.f * cu * c[k] - 3.f * u[k]);
    }
    const float inv = 1.f / rho;
    float jb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        jb[k] = ub[k] * inv;
        rb -= ub[k] * u[k] * inv;
    }
    // through the legacy target (affine; its transpose is port_transpose)
    float tb[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) tb[q] = rb + L::cx(q) * jb[0] + L::cy(q) * jb[1] + L::cz(q) * jb[2];
    port_transpose<Q>(P, tb);
#pragma unroll
    for (int q = 0; q < Q; ++q) v[q] += tb[q];
}

// Transposed port map of one port cell, in place on v.  rp / u: the density
// - 1 and velocity j / rho of the cell the map is linearised at (the inward
// neighbour for the extrapolations, the rebuilt cell itself for the
// regularized port; unused by the affine legacy map).
template <int Q>
__device__ __forceinline__ void port_vjp(const PortMap& P, float rp, const float (&u)[3], float (&v)[Q]) {
    if (P.recon == 3) regularized_transpose<Q>(P, rp, u, v);
    else if (P.recon) nee_transpose<Q>(P, rp, u, v);
    else port_transpose<Q>(P, v);
}

// The cell whose (rho, u) a port cell's transpose is linearised at.
__device__ __forceinline__ int64_t port_lin_cell(const PortMap& P, int64_t x) {
    return (P.recon == 1 || P.recon == 2) ? x + P.nb_off : x;
}

// The post-port populations g of port cell x (shifted) from the population
// array A: the legacy affine map on its own streamed g, the regularized
// port, or the extrapolation from the inward neighbour's streamed
// populations (read through the same pull).  Returns the exchanged mass;
// rp_n / u_n receive the (rho - 1, j / rho) the transpose is linearised at
// (port_lin_cell's) for the nonlinear ports.
template <int Q, typename T>
__device__ __forceinline__ float port_state(const PortMap& P, const T* __restrict__ A, const Geometry& G,
                                            const uint32_t* __restrict__ mask, uint32_t x, float (&g)[Q],
                                            float* rp_n = nullptr, float* u_n = nullptr) {
    if (!P.recon) return apply_port<Q>(P, g);
    if (P.recon == 3) {
        float s0 = 0.f, s1 = 0.f;
#pragma unroll
        for (int q = 0; q < Q; ++q) s0 += g[q];
        regularized_apply<Q>(P, g);
#pragma unroll
        for (int q = 0; q < Q; ++q) s1 += g[q];
        if (rp_n) {
            float u[3];
            nee_moments<Q, float>(g, *rp_n, u);
            u_n[0] = u[0];
            u_n[1] = u[1];
            u_n[2] = u[2];
        }
        return s1 - s0;
    }
    const uint32_t xn = (uint32_t)((int64_t)x + P.nb_off);
    float gn[Q], out[Q];
    load_pop<Q, T>(A, G, xn, mask[xn], gn);
    nee_apply<Q, float>(P, gn, out);
    if (rp_n) {
        float u[3];
        nee_moments<Q, float>(gn, *rp_n, u);
        u_n[0] = u[0];
        u_n[1] = u[1];
        u_n[2] = u[2];
    }
    float exch = 0.f;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        exch += out[q] - g[q];
        g[q] = out[q];
    }
    return exch;
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
    // approximate reciprocals (a few ulp; the FP32 state carries ~1e-7 anyway)
    const float inv_s = __fdividef(1.f, 1.f + 0.5f * alpha);
    const float inv_rho = __fdividef(1.f, M.rho);
    M.u[0] = (jx * inv_rho + 0.5f * P.a[0]) * inv_s;
    M.u[1] = (jy * inv_rho + 0.5f * P.a[1]) * inv_s;
    M.u[2] = (jz * inv_rho + 0.5f * P.a[2]) * inv_s;
#pragma unroll
    for (int d = 0; d < 3; ++d) M.F[d] = M.rho * (P.a[d] - alpha * M.u[d]);
    return M;
}

template <int Q>
__device__ __forceinline__ double dotc_d(int q, const double (&v)[3]) {
    using L = Lat<Q>;
    double s = 0.0;
    if (L::cx(q)) s += L::cx(q) * v[0];
    if (L::cy(q)) s += L::cy(q) * v[1];
    if (L::cz(q)) s += L::cz(q) * v[2];
    return s;
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

// Pair sums s = v_i + v_opp(i), d = v_i - v_opp(i) feed the moments, the
// TRT relaxation (moving/collision.rs:457-488, in pair form) and the mass
// remainder in one pass.  SC = 0: v = g = f - w; SC = 1: v = (f - w)/w, the
// 16-bit storage form, in which the weights drop out of the pair formulas.
// Returns the macroscopic state of the loaded populations (implicit
// half-step Brinkman velocity and Guo force, solver.rs:190-196); with
// `post` the populations are replaced by their post-collision values.
//
// BGK is the case om == omega.  MRT adds one rank-one correction per even
// moment whose rate differs from the shear rate: the odd moments of the
// Gram-Schmidt basis span exactly the antisymmetric subspace, so MRT with
// all even rates equal to omega is TRT.  The rest population takes the mass
// remainder: the FP32 weights do not sum to one, which would otherwise leak
// (rho - 1)(sum w - 1) per cell and step -- systematic where the pressure
// has one sign.
template <int Q, int COLL, int SC>
__device__ __forceinline__ Macro collide_fused(float (&v)[Q], float alpha, const Physics& P, bool post, float om,
                                              float omm) {
    using L = Lat<Q>;
    constexpr int NP = L::NPAIR;
    float S[NP], D[NP];
    float rp = SC ? L::w(0) * v[0] : v[0];
    float jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const int i = k + 1, o = opp<Q>(i);
        S[k] = v[i] + v[o];
        D[k] = v[i] - v[o];
        constexpr float one = 1.f;
        const float w = SC ? L::w(i) : one;
        rp = fmaf(w, S[k], rp);
        if (L::cx(i)) jx = fmaf(w * L::cx(i), D[k], jx);
        if (L::cy(i)) jy = fmaf(w * L::cy(i), D[k], jy);
        if (L::cz(i)) jz = fmaf(w * L::cz(i), D[k], jz);
    }
    Macro M;
    M.rp = rp;
    M.rho = 1.f + rp;
    // approximate reciprocals (a few ulp; the FP32 state carries ~1e-7 anyway)
    const float inv_s = __fdividef(1.f, 1.f + 0.5f * alpha);
    const float inv_rho = __fdividef(1.f, M.rho);
    M.u[0] = (jx * inv_rho + 0.5f * P.a[0]) * inv_s;
    M.u[1] = (jy * inv_rho + 0.5f * P.a[1]) * inv_s;
    M.u[2] = (jz * inv_rho + 0.5f * P.a[2]) * inv_s;
#pragma unroll
    for (int d = 0; d < 3; ++d) M.F[d] = M.rho * (P.a[d] - alpha * M.u[d]);
    if (!post) return M;

    const float kp = 1.f - 0.5f * om, km = 1.f - 0.5f * omm;
    const float hp = 0.5f * (1.f - om), hm = 0.5f * (1.f - omm);
    const float rho = M.rho;
    const float usq15 = 1.5f * (M.u[0] * M.u[0] + M.u[1] * M.u[1] + M.u[2] * M.u[2]);
    const float uf3 = 3.f * (M.u[0] * M.F[0] + M.u[1] * M.F[1] + M.u[2] * M.F[2]);
    float dproj[MAX_PROJ];
    if constexpr (COLL == CK_MRT) {
        // y = f - eq + src/2 of the rest population (g or g/w form)
        const float w0 = SC ? 1.f : L::w(0);
        const float y0 = v[0] - w0 * (rp - rho * usq15) - 0.5f * w0 * uf3;
#pragma unroll
        for (int p = 0; p < MAX_PROJ; ++p)
            if (p < P.n_proj) dproj[p] = (SC ? L::w(0) : 1.f) * P.proj_right[p][0] * y0;
    }
    float rem = rp;  // mass left for the rest population
    if constexpr (COLL != CK_MRT) {
        // Pair relaxation with the cell's constants folded:
        //   P' = hp S + w [E0 + A cu^2 + 9 kp cu cf],  E0 = om (rp - rho 1.5 u^2) - kp 3 u.F,  A = 4.5 om rho
        //   D' = hm D + w [G cu + 3 km cf],              G = 3 om_odd rho
        // (the equilibrium and source terms of the MRT branch, regrouped).
        const float E0 = fmaf(om, fmaf(-rho, usq15, rp), -kp * uf3);
        const float A = 4.5f * om * rho, G = 3.f * omm * rho;
        const float K9 = 9.f * kp, K3 = 3.f * km;
        // MRT_BULK: the bulk moment Eb = sum_i w_i b_i y_i of y = f - eq + src/2,
        // b_i = |c_i|^2 - 1 (zero on the axis directions); per pair
        // y_p = S/2 - w [e0 + 4.5 cu (rho cu - cf)], e0 = rp - 1.5 rho u^2 + 1.5 u.F
        float Eb = 0.f, e0 = 0.f;
        if constexpr (COLL == CK_MRT_BULK) {
            const float w0 = SC ? 1.f : L::w(0);
            const float y0 = v[0] - w0 * (rp - rho * usq15) - 0.5f * w0 * uf3;
            Eb = -(SC ? L::w(0) : 1.f) * y0;
            e0 = fmaf(-rho, usq15, rp) + 0.5f * uf3;
        }
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int i = k + 1, o = opp<Q>(i);
            const float cu = dotc<Q>(i, M.u);
            const float cf = dotc<Q>(i, M.F);
            if constexpr (COLL == CK_MRT_BULK) {
                const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
                if (c2 != 1) {  // folded after unrolling
                    const float wy = SC ? 1.f : L::w(i);
                    const float yp = fmaf(-wy, fmaf(4.5f * cu, fmaf(rho, cu, -cf), e0), 0.5f * S[k]);
                    Eb = fmaf((SC ? 2.f * L::w(i) : 2.f) * (float)(c2 - 1), yp, Eb);
                }
            }
            const float tp = fmaf(cu * cf, K9, fmaf(cu * cu, A, E0));
            const float tm = fmaf(cu, G, cf * K3);
            float Pp, Dm;
            if constexpr (SC) {
                Pp = fmaf(hp, S[k], tp);
                Dm = fmaf(hm, D[k], tm);
            } else {
                Pp = fmaf(tp, L::w(i), hp * S[k]);
                Dm = fmaf(tm, L::w(i), hm * D[k]);
            }
            v[i] = Pp + Dm;
            v[o] = Pp - Dm;
            rem = fmaf(SC ? -2.f * L::w(i) : -2.f, Pp, rem);
        }
        if constexpr (COLL == CK_MRT_BULK) {
            // rank-one bulk correction: v_i -= (s_bulk - omega) Eb w_i b_i / |b|^2_W,
            // |b|^2_W = 2/3 on both lattices; the rest population keeps the mass
            const float cb = P.proj_rate[0] * Eb * 1.5f;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const int i = k + 1, o = opp<Q>(i);
                const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
                if (c2 != 1) {  // folded after unrolling
                    const float dv = cb * (float)(c2 - 1) * (SC ? 1.f : L::w(i));
                    v[i] -= dv;
                    v[o] -= dv;
                    rem = fmaf(SC ? 2.f * L::w(i) : 2.f, dv, rem);
                }
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int i = k + 1, o = opp<Q>(i);
            const float w = SC ? 1.f : L::w(i);  // weight of the g form (1 in the g/w form)
            const float cu = dotc<Q>(i, M.u);
            const float cf = dotc<Q>(i, M.F);
            const float geqp = w * fmaf(rho, fmaf(4.5f * cu, cu, -usq15), rp);  // symmetric part of eq
            const float eqm = (3.f * w) * rho * cu;                             // antisymmetric part of eq
            const float spv = w * fmaf(9.f * cu, cf, -uf3);                     // symmetric part of the source
            const float smv = (3.f * w) * cf;                                   // antisymmetric part
            float Pp = fmaf(hp, S[k], fmaf(kp, spv, om * geqp));
            const float Dm = fmaf(hm, D[k], fmaf(km, smv, omm * eqm));
            if constexpr (COLL == CK_MRT) {
                const float yp = 0.5f * S[k] - geqp + 0.5f * spv;
#pragma unroll
                for (int p = 0; p < MAX_PROJ; ++p)
                    if (p < P.n_proj) dproj[p] = fmaf((SC ? 2.f * L::w(i) : 2.f) * P.proj_right[p][i], yp, dproj[p]);
            }
            v[i] = Pp + Dm;
            v[o] = Pp - Dm;
            rem = fmaf(SC ? -2.f * L::w(i) : -2.f, Pp, rem);
        }
        if constexpr (COLL == CK_MRT) {
#pragma unroll
            for (int p = 0; p < MAX_PROJ; ++p) {
                if (p < P.n_proj) {
                    const float c = P.proj_rate[p] * dproj[p];
#pragma unroll
                    for (int k = 0; k < NP; ++k) {
                        const int i = k + 1, o = opp<Q>(i);
                        const float dv = c * (SC ? P.proj_lw[p][i] : P.proj_left[p][i]);
                        v[i] -= dv;
                        v[o] -= dv;
                        rem = fmaf(SC ? 2.f * L::w(i) : 2.f, dv, rem);
                    }
                }
            }
        }
    }
    v[0] = SC ? rem * (float)(1.0 / L::wd(0)) : rem;
    return M;
}

// The same collision in FP64 arithmetic for FP32 storage (g = f - w form):
// the populations are widened once, collided with the exact weights, and
// rounded once on the way out.  FP32 arithmetic rounds the equilibrium
// momentum (rho u, the weights) to ~1e-7 relative, and in a nearly uniform
// flow those roundings repeat coherently from cell to cell and step to step:
// the steady state then carries a bias of ~1e-7 in density (the pressure drop
// ~1e-6 relative on the 64^3 channel), where the stored state's own rounding
// alone leaves ~1e-9.  Selected per problem (collision_fp64); the rates and
// MRT basis vectors are the FP32 ones of Physics.
template <int Q, int COLL>
__device__ __forceinline__ Macro collide_fused_dp(float (&vf)[Q], float alpha_f, const Physics& P, bool post,
                                                 float om_f, float omm_f) {
    using L = Lat<Q>;
    constexpr int NP = L::NPAIR;
    double v[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) v[q] = vf[q];
    double S[NP], D[NP];
    double rp = v[0], j[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const int i = k + 1, o = opp<Q>(i);
        S[k] = v[i] + v[o];
        D[k] = v[i] - v[o];
        rp += S[k];
        if (L::cx(i)) j[0] += L::cx(i) * D[k];
        if (L::cy(i)) j[1] += L::cy(i) * D[k];
        if (L::cz(i)) j[2] += L::cz(i) * D[k];
    }
    const double alpha = alpha_f, rho = 1.0 + rp, s = 1.0 + 0.5 * alpha;
    double u[3], F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        u[d] = (j[d] / rho + 0.5 * (double)P.a[d]) / s;
        F[d] = rho * ((double)P.a[d] - alpha * u[d]);
    }
    Macro M;
    M.rp = (float)rp;
    M.rho = (float)rho;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        M.u[d] = (float)u[d];
        M.F[d] = (float)F[d];
    }
    if (!post) return M;
    const double om = om_f, omm = omm_f;
    const double kp = 1.0 - 0.5 * om, km = 1.0 - 0.5 * omm;
    const double hp = 0.5 * (1.0 - om), hm = 0.5 * (1.0 - omm);
    const double usq15 = 1.5 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double uf3 = 3.0 * (u[0] * F[0] + u[1] * F[1] + u[2] * F[2]);
    // y = f - eq + src/2 of the rest population (MRT projections)
    const double y0 = v[0] - L::wd(0) * (rp - rho * usq15) - 0.5 * L::wd(0) * uf3;
    double dproj[MAX_PROJ];
#pragma unroll
    for (int p = 0; p < MAX_PROJ; ++p) dproj[p] = (COLL == CK_MRT && p < P.n_proj) ? (double)P.proj_right[p][0] * y0 : 0.0;
    double Eb = -y0;  // MRT_BULK: sum_i w_i b_i y_i with b = |c|^2 - 1
    double rem = rp;
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const int i = k + 1, o = opp<Q>(i);
        const double w = L::wd(i);
        const double cu = dotc_d<Q>(i, u), cf = dotc_d<Q>(i, F);
        const double geqp = w * (rho * (4.5 * cu * cu - usq15) + rp);  // symmetric part of eq (g form)
        const double eqm = 3.0 * w * rho * cu;                          // antisymmetric part
        const double spv = w * (9.0 * cu * cf - uf3);                    // symmetric part of the source
        const double smv = 3.0 * w * cf;                                 // antisymmetric part
        if constexpr (COLL == CK_MRT_BULK) {
            const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
            if (c2 != 1) Eb += 2.0 * (c2 - 1) * (0.5 * S[k] - geqp + 0.5 * spv);
        }
        if constexpr (COLL == CK_MRT) {
            const double yp = 0.5 * S[k] - geqp + 0.5 * spv;
#pragma unroll
            for (int p = 0; p < MAX_PROJ; ++p)
                if (p < P.n_proj) dproj[p] += 2.0 * (double)P.proj_right[p][i] * yp;
        }
        const double Pp = hp * S[k] + kp * spv + om * geqp;
        const double Dm = hm * D[k] + km * smv + omm * eqm;
        v[i] = Pp + Dm;
        v[o] = Pp - Dm;
        rem -= 2.0 * Pp;
    }
    if constexpr (COLL == CK_MRT_BULK) {
        // rank-one bulk correction, |b|^2_W = 2/3; the rest population keeps the mass
        const double cb = (double)P.proj_rate[0] * Eb * 1.5;
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int i = k + 1, o = opp<Q>(i);
            const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
            if (c2 != 1) {
                const double dv = cb * (c2 - 1) * L::wd(i);
                v[i] -= dv;
                v[o] -= dv;
                rem += 2.0 * dv;
            }
        }
    }
    if constexpr (COLL == CK_MRT) {
#pragma unroll
        for (int p = 0; p < MAX_PROJ; ++p) {
            if (p < P.n_proj) {
                const double c = (double)P.proj_rate[p] * dproj[p];
#pragma unroll
                for (int k = 0; k < NP; ++k) {
                    const int i = k + 1, o = opp<Q>(i);
                    const double dv = c * (double)P.proj_left[p][i];
                    v[i] -= dv;
                    v[o] -= dv;
                    rem += 2.0 * dv;
                }
            }
        }
    }
    v[0] = rem;
#pragma unroll
    for (int q = 0; q < Q; ++q) vf[q] = (float)v[q];
    return M;
}

// Collision transpose at the recorded (rho, u): given gb = d(loss)/d(post),
// returns d(loss)/d(f) in gb and d(loss)/d(alpha).  post = f - R y + src with
// y = f - eq(rho, u) + src(u, F)/2; the cotangents of eq and src need only
// the weighted zeroth, first and second moments of z = R^T gb and of
// h = gb - z/2.  For TRT they are the moments of gb scaled by omega / om
// (even / odd), taken pair by pair; the MRT rank-one terms add analytic
// multiples of the precomputed moments of their basis vectors.  Then the
// Brinkman chain F = rho (a - alpha u), u = (m/rho + a/2)/(1 + alpha/2).
template <int Q, int COLL>
__device__ __forceinline__ float collide_vjp(float (&gb)[Q], float rp, const float (&u)[3], float alpha,
                                             const Physics& P, float om, float omm, float k = 1.f) {
    using L = Lat<Q>;
    constexpr int NP = L::NPAIR;
    const float rho = 1.f + rp;
    const float s = 1.f + 0.5f * alpha;
    float F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d] = rho * (P.a[d] - alpha * u[d]);
    // weighted moments of gb, pair by pair; the pair sums and differences are
    // kept for the output pass, which applies the TRT part of the transpose
    // (gb - R^T gb per pair: (1 - om)/2 sm +- (1 - omm)/2 df)
    float M0 = L::w(0) * gb[0];
    float M1[3] = {0.f, 0.f, 0.f}, M2[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float SM[NP], DF[NP];
    float g0 = (1.f - om) * gb[0];  // the rest population's output, less rho_bar
#pragma unroll
    for (int k = 0; k < NP; ++k) {
        const int i = k + 1, o = opp<Q>(i);
        const float sm = gb[i] + gb[o], df = gb[i] - gb[o];
        SM[k] = sm;
        DF[k] = df;
        const float w = L::w(i);
        const int c0 = L::cx(i), c1 = L::cy(i), c2 = L::cz(i);
        M0 = fmaf(w, sm, M0);
        if (c0) {
            M1[0] = fmaf(w * c0, df, M1[0]);
            M2[0] = fmaf(w, sm, M2[0]);
        }
        if (c1) {
            M1[1] = fmaf(w * c1, df, M1[1]);
            M2[1] = fmaf(w, sm, M2[1]);
        }
        if (c2) {
            M1[2] = fmaf(w * c2, df, M1[2]);
            M2[2] = fmaf(w, sm, M2[2]);
        }
        if (c0 && c1) M2[3] = fmaf(w * c0 * c1, sm, M2[3]);
        if (c0 && c2) M2[4] = fmaf(w * c0 * c2, sm, M2[4]);
        if (c1 && c2) M2[5] = fmaf(w * c1 * c2, sm, M2[5]);
    }
    float Z0 = om * M0, H0 = (1.f - 0.5f * om) * M0;
    float Z1[3], H1[3], Z2[6], H2[6];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        Z1[d] = omm * M1[d];
        H1[d] = (1.f - 0.5f * omm) * M1[d];
    }
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        Z2[e] = om * M2[e];
        H2[e] = (1.f - 0.5f * om) * M2[e];
    }
    float bulk_c = 0.f;  // MRT_BULK: the bulk correction's coefficient
    if constexpr (COLL == CK_MRT_BULK) {
        // the bulk correction folded: b_i = |c_i|^2 - 1, |b|^2_W = 2/3,
        // sum_i w_i b_i = 0 and sum_i w_i b_i c_ia c_ib = 2/9 delta_ab on both lattices
        float e = -L::w(0) * gb[0];
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const int i = k + 1;
            const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
            if (c2 != 1) e = fmaf(L::w(i) * (float)(c2 - 1), SM[k], e);  // folded after unrolling
        }
        bulk_c = P.proj_rate[0] * e * 1.5f;
        const float c = bulk_c;
        g0 += c;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            Z2[d] = fmaf(c, 2.f / 9.f, Z2[d]);
            H2[d] = fmaf(-0.5f * c, 2.f / 9.f, H2[d]);
        }
    }
    float cproj[MAX_PROJ];  // MRT: the rank-one corrections' coefficients
    if constexpr (COLL == CK_MRT) {
#pragma unroll
        for (int p = 0; p < MAX_PROJ; ++p) {
            cproj[p] = 0.f;
            if (p < P.n_proj) {
                float e = 0.f;
#pragma unroll
                for (int i = 0; i < Q; ++i) e = fmaf(P.proj_left[p][i], gb[i], e);
                const float c = P.proj_rate[p] * e;
                cproj[p] = c;
                g0 = fmaf(-c, P.proj_right[p][0], g0);
                Z0 = fmaf(c, P.proj_m0[p], Z0);
                H0 = fmaf(-0.5f * c, P.proj_m0[p], H0);
#pragma unroll
                for (int e2 = 0; e2 < 6; ++e2) {
                    Z2[e2] = fmaf(c, P.proj_m2[p][e2], Z2[e2]);
                    H2[e2] = fmaf(-0.5f * c, P.proj_m2[p][e2], H2[e2]);
                }
            }
        }
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
    const float inv_s = __fdividef(1.f, s);
    const float inv = __fdividef(inv_s, rho);
    float mb[3];
    float sbar = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mb[d] = ub[d] * inv;
        rho_bar -= ub[d] * (s * u[d] - 0.5f * P.a[d]) * inv;
        sbar -= ub[d] * u[d] * inv_s;
    }
    abar += 0.5f * sbar;
    // output, times k: gb - R^T gb + rho_bar + c . mb, pair by pair (with
    // the MRT corrections, which are even: the same for i and opp(i)); the
    // scale k of the stored cotangent enters the few per-cell coefficients
    // instead of every population
    const float hp = 0.5f * (1.f - om) * k, hm = 0.5f * (1.f - omm) * k;
    const float kr = k * rho_bar, kbulk = k * bulk_c;
    float kmb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) kmb[d] = k * mb[d];
    gb[0] = fmaf(k, g0, kr);
#pragma unroll
    for (int kk = 0; kk < NP; ++kk) {
        const int i = kk + 1, o = opp<Q>(i);
        float base = kr;
        if constexpr (COLL == CK_MRT_BULK) {
            const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
            if (c2 != 1) base = fmaf(-kbulk, (float)(c2 - 1), base);  // folded after unrolling
        }
        float pi = fmaf(hp, SM[kk], base), po = pi;
        if constexpr (COLL == CK_MRT) {
#pragma unroll
            for (int p = 0; p < MAX_PROJ; ++p)
                if (p < P.n_proj) {
                    pi = fmaf(-k * cproj[p], P.proj_right[p][i], pi);
                    po = fmaf(-k * cproj[p], P.proj_right[p][o], po);
                }
        }
        // c . kmb accumulated from the first nonzero component of the
        // direction whose first component is positive (no negations)
        const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
        const int first = c[0] ? 0 : (c[1] ? 1 : 2);
        const int sg = c[first] > 0 ? 1 : -1;
        float cm = kmb[first];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d != first && c[d]) cm = sg * c[d] > 0 ? cm + kmb[d] : cm - kmb[d];
        if (sg > 0) {
            const float d = fmaf(hm, DF[kk], cm);  // hm DF + c . mb
            gb[i] = pi + d;
            gb[o] = po - d;
        } else {
            const float d = fmaf(-hm, DF[kk], cm);  // -(hm DF + c . mb)
            gb[i] = pi - d;
            gb[o] = po + d;
        }
    }
    return abar;
}

// Second moments S_ab = sum_q c_a c_b g_q (xx yy zz xy xz yz) of g = f - w.
template <int Q>
__device__ __forceinline__ void second_moments(const float (&g)[Q], float (&S)[6]) {
    using L = Lat<Q>;
#pragma unroll
    for (int e = 0; e < 6; ++e) S[e] = 0.f;
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
}

// VJP of the weighted responses of one fluid cell (vector_vjp,
// solver.rs:896-947, plus the pressure drop and the viscous dissipation
// sigma:sigma / (2 rho nu), sigma = -(1 - omega/2) (Pi_neq + (uF + Fu)/2))
// with respect to the cell's streamed populations g = f - w, given rho - 1,
// the Brinkman velocity u and the second moments S of g.  fb = d/dg; returns
// the cotangent of alpha.  The responses depend on g only through these
// moments, so the adjoint step can seed a state from its record alone.
template <int Q>
__device__ __forceinline__ float response_vjp(float rp, const float (&u)[3], const float (&S)[6], float alpha,
                                              float dpw, bool port, const SeedParams& sp, const Physics& P,
                                              float (&fb)[Q]) {
    using L = Lat<Q>;
    const float k = 1.f - 0.5f / sp.tau;
    const float nu = (sp.tau - 0.5f) / 3.f;
    const float rho = 1.f + rp;
    float F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d] = rho * (P.a[d] - alpha * u[d]);
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    float sig[6];
    float ss = 0.f;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const float pi = S[e] - (e < 3 ? rp / 3.f : 0.f) - rho * u[ia[e]] * u[ib[e]];
        const float t = 0.5f * (u[ia[e]] * F[ib[e]] + u[ib[e]] * F[ia[e]]);
        sig[e] = -k * (pi + t);
        ss += (e < 3 ? 1.f : 2.f) * sig[e] * sig[e];
    }
    // cotangents of rho, u, F, M2 (all lattice units)
    const float V = sp.vel;
    const float U[3] = {u[0] * V, u[1] * V, u[2] * V};
    const float usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
    const float R = rho * sp.dens;
    const float W3 = sp.w[3], W4 = sp.w[4], W7 = sp.w[7];
    float rb = 0.f, abar = 0.f, ub[3], Fb[3] = {0.f, 0.f, 0.f}, Sb[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float kin = W3 + W4 * alpha / sp.dt_s;
#pragma unroll
    for (int d = 0; d < 3; ++d) ub[d] = sp.w[d] * V + kin * R * 2.f * U[d] * V;
    rb += kin * sp.dens * usq;
    abar += W4 * R / sp.dt_s * usq;
    if (port) rb += sp.w[6] * dpw * sp.dens * V * V / 3.f;
    if (W7 != 0.f) {
        rb += -W7 * ss / (2.f * rho * rho * nu);
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const float mult = (e < 3 ? 1.f : 2.f);  // off-diagonals appear twice
            const float pb = -k * W7 * sig[e] / (rho * nu) * mult;
            const int i0 = ia[e], i1 = ib[e];
            Sb[e] += pb;
            rb -= pb * ((e < 3 ? 1.f / 3.f : 0.f) + u[i0] * u[i1]);
            if (e < 3) {
                ub[i0] -= 2.f * rho * pb * u[i0];
                ub[i0] += pb * F[i0];
                Fb[i0] += pb * u[i0];
            } else {
                ub[i0] -= rho * pb * u[i1];
                ub[i1] -= rho * pb * u[i0];
                ub[i0] += 0.5f * pb * F[i1];
                ub[i1] += 0.5f * pb * F[i0];
                Fb[i1] += 0.5f * pb * u[i0];
                Fb[i0] += 0.5f * pb * u[i1];
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        rb += Fb[d] * (P.a[d] - alpha * u[d]);
        abar -= Fb[d] * rho * u[d];
        ub[d] -= Fb[d] * rho * alpha;
    }
    const float s = 1.f + 0.5f * alpha;
    const float inv = 1.f / (s * rho);
    float mb[3], sbar = 0.f;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mb[d] = ub[d] * inv;
        rb -= ub[d] * (s * u[d] - 0.5f * P.a[d]) * inv;
        sbar -= ub[d] * u[d] / s;
    }
    abar += 0.5f * sbar;
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
    return abar;
}

// Integrands of the responses of one fluid cell (vector_cell, solver.rs:
// 835-895, plus the viscous dissipation of response_vjp), in FP32 from the
// cell's moments: out = {U_x, U_y, U_z, R |U|^2, R alpha |U|^2 / dt,
// sigma:sigma / (2 rho nu)} in the units that sums_to_responses scales.  The
// design density and the pressure drop are added by the caller.
template <int Q>
__device__ __forceinline__ void response_cell(float rp, const float (&u)[3], const float (&S)[6], float alpha,
                                              const SeedParams& sp, const Physics& P, float (&out)[6]) {
    const float k = 1.f - 0.5f / sp.tau;
    const float nu = (sp.tau - 0.5f) / 3.f;
    const float rho = 1.f + rp;
    float F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d] = rho * (P.a[d] - alpha * u[d]);
    const int ia[6] = {0, 1, 2, 0, 0, 1}, ib[6] = {0, 1, 2, 1, 2, 2};
    float ss = 0.f;
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        const float pi = S[e] - (e < 3 ? rp / 3.f : 0.f) - rho * u[ia[e]] * u[ib[e]];
        const float t = 0.5f * (u[ia[e]] * F[ib[e]] + u[ib[e]] * F[ia[e]]);
        const float sg = -k * (pi + t);
        ss += (e < 3 ? 1.f : 2.f) * sg * sg;
    }
    const float V = sp.vel;
    const float U[3] = {u[0] * V, u[1] * V, u[2] * V};
    const float usq = U[0] * U[0] + U[1] * U[1] + U[2] * U[2];
    const float R = rho * sp.dens;
    out[0] = U[0];
    out[1] = U[1];
    out[2] = U[2];
    out[3] = R * usq;
    out[4] = R * alpha / sp.dt_s * usq;
    out[5] = ss / (2.f * rho * nu);
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

// Per-thread admission accumulators (a thread sees a few tens of cells, so
// single precision partial sums are exact to ~1e-7 of their own size; the
// block and grid reductions are compensated double).
struct DiagLocal {
    float mass, exch, minf, maxu2;
    int nf;
    __device__ void init() {
        mass = exch = 0.f;
        minf = INFINITY;
        maxu2 = 0.f;
        nf = 0;
    }
};

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
    __shared__ DiagAcc sh[32];
    for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        if (lane < (int)(blockDim.x >> 5)) v = sh[lane];
        else v.init();
        for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    }
    return v;
}

// Writes one block's partial, and lets the last block to finish combine all
// partials in a fixed order (deterministic) into *out.  No block waits.
__device__ void finish_diag(const DiagLocal& loc, StepDiag* out, const Reduce& red) {
    __shared__ bool last;
    DiagAcc v;
    v.mh = loc.mass;
    v.ml = 0.0;
    v.eh = loc.exch;
    v.el = 0.0;
    v.minf = loc.minf;
    v.maxu2 = loc.maxu2;
    v.nf = loc.nf;
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
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
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
    __shared__ Sums<NS> sh[32];
    for (int off = 16; off > 0; off >>= 1) v.shfl_merge(off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        if (lane < (int)(blockDim.x >> 5)) v = sh[lane];
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
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
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


// ------------------------------------------------------------------ launch helpers
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

[[maybe_unused]] static int blocks_for(int64_t n, int cap, int tile = BLOCK) {
    int64_t b = (n + tile - 1) / tile;
    if (cap > 0 && b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

// One wave of resident blocks (occupancy of this exact kernel x SM count);
// the grid-stride loops then give every thread the same number of cells.
[[maybe_unused]] static int persistent_grid(const void* kernel, int64_t n, size_t smem = 0, int threads = BLOCK, int tile = BLOCK) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> per_sm;
    [[maybe_unused]] static int sms = 0;
    int b;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (sms == 0) {
            int dev = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (sms <= 0) sms = 148;
        }
        auto it = per_sm.find(kernel);
        if (it == per_sm.end()) {
            int nb = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess || nb <= 0) nb = 1;
            it = per_sm.emplace(kernel, nb).first;
        }
        b = it->second * sms;
    }
    return blocks_for(n, b, tile);
}


}  // namespace
}  // namespace lbm

namespace lbm {
namespace {

// ------------------------------------------------------------------ staged pipelines
// A tile is TILE consecutive cells.  For every direction the AA access of a
// whole tile is one contiguous run of a population plane: the cells' own
// slots (parity 0) or the run shifted by the direction's constant linear
// offset (parity 1).  A producer warp issues one bulk copy per run into a
// ring of STAGES shared-memory buffers (cp.async.bulk completing on a "full"
// mbarrier); eight consumer warps compute one cell each and release the
// buffer on an "empty" mbarrier.  Runs are fetched 16-byte aligned and one
// vector longer than the tile; each consumer indexes its element with the
// run's misalignment.  Blocked links (walls, solids) and cells on periodic
// faces read their few populations from global memory directly.
constexpr int CONSUMER_WARPS = 8;
constexpr int TILE = CONSUMER_WARPS * 32;
constexpr int TPB = CONSUMER_WARPS * 32 + 32;
// Ring depth per storage width: a 16-bit tile carries half the bytes of a
// 32-bit one, so more of them are kept in flight for the same bytes.
#ifndef LBM_STAGES_32
#define LBM_STAGES_32 3
#endif
#ifndef LBM_STAGES_16
#define LBM_STAGES_16 3
#endif
template <typename T>
struct Ring {
    static constexpr int STAGES = sizeof(T) == 4 ? LBM_STAGES_32 : LBM_STAGES_16;
    static_assert(STAGES >= 2 && STAGES <= 10, "ring depth");
};
constexpr int PIPE_HEAD = 256;  // full/empty/rdone mbarriers of up to 10 stages

template <typename T>
struct Vec16 {
    static constexpr int V = 16 / (int)sizeof(T);  // elements per 16 bytes
    static constexpr int RUN = TILE + V;            // elements per staged run
    static constexpr int BYTES = RUN * (int)sizeof(T);
};
constexpr int FRUN = TILE + 4;  // float / uint32 runs (mask, alpha, record)
constexpr int FRUN_BYTES = FRUN * 4;

template <typename S>
__host__ __device__ constexpr size_t stage_stride() {
    return (sizeof(S) + 127) / 128 * 128;
}
template <typename S, int NS>
__host__ __device__ constexpr size_t pipe_bytes() {
    return PIPE_HEAD + NS * stage_stride<S>();
}
// Ring depth of a stage type: the storage width's depth, reduced to two
// stages where the deeper ring would leave room for only one block per SM
// (half of the 227 KB a block may use, less the static reduction scratch).
template <typename S, typename T>
__host__ __device__ constexpr int ring_depth() {
    return (Ring<T>::STAGES > 2 && pipe_bytes<S, Ring<T>::STAGES>() > 105 * 1024) ? 2 : Ring<T>::STAGES;
}
template <typename S>
__device__ __forceinline__ S* stage_at(unsigned char* smem, int s) {
    return reinterpret_cast<S*>(smem + PIPE_HEAD + s * stage_stride<S>());
}

// Misalignment of direction q's staged run when the plane stride n and the
// strides sx, sy are multiples of the 16-byte vector V: the run starts at
// q*n + x0 + dir*lin(q) and x0 is a multiple of the tile, so only c_z is left.
template <int Q, typename T, int DIR>
__device__ __forceinline__ constexpr int rund_aligned(int q) {
    constexpr int V = Vec16<T>::V;
    const int d = DIR * Lat<Q>::cz(q);
    return d < 0 ? d + V : d;
}

// Minimum population f = w + g (or w (1 + g/w) in 16-bit storage units) of
// one cell: the minimum is taken per weight class (|c|^2) first.
template <int Q, int SC>
__device__ __forceinline__ float min_population(const float (&v)[Q]) {
    using L = Lat<Q>;
    float m[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int k = (L::cx(q) != 0) + (L::cy(q) != 0) + (L::cz(q) != 0);
        m[k] = fminf(m[k], v[q]);
    }
    float mn = INFINITY;
#pragma unroll
    for (int k = 0; k < (Q == 19 ? 3 : 4); ++k) {
        float w = 0.f;  // the class weight (a compile-time constant after unrolling)
#pragma unroll
        for (int r = 0; r < Q; ++r)
            if ((L::cx(r) != 0) + (L::cy(r) != 0) + (L::cz(r) != 0) == k) w = L::w(r);
        mn = fminf(mn, SC ? w * (1.f + m[k]) : w + m[k]);
    }
    return mn;
}

// Aligned store of one cell's values into its own slots of the output array
// (populations in storage units with stochastic rounding for 16-bit storage,
// or adjoint values scaled by `scale`).
template <int Q, typename T>
__device__ __forceinline__ void store_own_pop(T* A, uint32_t n, uint32_t x, const float (&v)[Q], uint32_t step) {
    uint32_t rs = 0;
    if constexpr (Cvt<T>::scaled) rs = cell_seed(x, step);
    senc_sr_all<Q, T>(v, rs, [&](int q, T e) { A[q * n + x] = e; });
}

template <int Q, typename T>
__device__ __forceinline__ void store_own_lam(T* B, uint32_t n, uint32_t x, const float (&v)[Q], float scale) {
#pragma unroll
    for (int q = 0; q < Q; ++q) B[q * n + x] = Cvt<T>::from(v[q] * scale);
}

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
    return cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace
}  // namespace lbm
