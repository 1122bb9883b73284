// lbm_vec2.cuh -- two-lane FP32 arithmetic for the 16-bit stepping kernels.
//
// sm_100a executes packed FP32 pairs (add / sub / mul / fma .f32x2) as one
// instruction.  A 16-bit step is bound by instruction issue, not bytes, so
// its consumer threads take two cells each and run the collision transpose
// once for both, lane by lane.  `R` is float (one cell) or F2 (two cells);
// the arithmetic below is written once for both.
#pragma once
#include <cuda_runtime.h>

#include "lbm_common.cuh"
#include "lbm_launch.h"

namespace lbm {
namespace {

struct F2 {
    float2 v;
};

__device__ __forceinline__ unsigned long long f2_bits(F2 a) {
    return (unsigned long long)__float_as_uint(a.v.x) | ((unsigned long long)__float_as_uint(a.v.y) << 32);
}
__device__ __forceinline__ F2 f2_from_bits(unsigned long long b) {
    return {make_float2(__uint_as_float((unsigned)(b & 0xffffffffull)), __uint_as_float((unsigned)(b >> 32)))};
}

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return f2_from_bits(d);
}
__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }

__device__ __forceinline__ F2 mad(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ float mad(float a, float b, float c) { return fmaf(a, b, c); }

// a constant in both lanes
template <typename R>
__device__ __forceinline__ R K(float c);
template <>
__device__ __forceinline__ float K<float>(float c) {
    return c;
}
template <>
__device__ __forceinline__ F2 K<F2>(float c) {
    return {make_float2(c, c)};
}

// approximate quotient a / b lane by lane (a few ulp)
__device__ __forceinline__ float qdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ F2 qdiv(F2 a, F2 b) { return {make_float2(__fdividef(a.v.x, b.v.x), __fdividef(a.v.y, b.v.y))}; }

// Collision transpose (the VJP of collide_fused, CK_PAIRS and CK_MRT_BULK)
// for R = float or F2: the same algebra as collide_vjp in lbm_device.cuh,
// with the linear output scaled by `k` (the stored cotangent's scale step)
// inside the final pass instead of by a multiply per population.  gb: the
// cotangent of the post-collision populations, replaced by that of the
// pre-collision ones times k; rp, u: the recorded (rho - 1, u); returns the
// alpha cotangent (unscaled).
template <int Q, int COLL, typename R>
__device__ __forceinline__ R collide_vjp_lanes(R (&gb)[Q], R rp, const R (&u)[3], R alpha, const Physics& P,
                                               float om, float omm, float k) {
    using L = Lat<Q>;
    constexpr int NP = L::NPAIR;
    static_assert(COLL != CK_MRT, "the general MRT transpose runs on the one-lane path");
    const R one = K<R>(1.f);
    const R rho = one + rp;
    const R s = mad(K<R>(0.5f), alpha, one);
    R F[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) F[d] = rho * (K<R>(P.a[d]) - alpha * u[d]);
    // weighted moments, pair by pair; sums and differences kept for the output
    R M0 = K<R>(L::w(0)) * gb[0];
    R M1[3] = {K<R>(0.f), K<R>(0.f), K<R>(0.f)};
    R M2[6] = {K<R>(0.f), K<R>(0.f), K<R>(0.f), K<R>(0.f), K<R>(0.f), K<R>(0.f)};
    R SM[NP], DF[NP];
#pragma unroll
    for (int kk = 0; kk < NP; ++kk) {
        const int i = kk + 1, o = opp<Q>(i);
        const R sm = gb[i] + gb[o], df = gb[i] - gb[o];
        SM[kk] = sm;
        DF[kk] = df;
        const float w = L::w(i);
        const int c0 = L::cx(i), c1 = L::cy(i), c2 = L::cz(i);
        M0 = mad(K<R>(w), sm, M0);
        if (c0) {
            M1[0] = mad(K<R>(w * c0), df, M1[0]);
            M2[0] = mad(K<R>(w), sm, M2[0]);
        }
        if (c1) {
            M1[1] = mad(K<R>(w * c1), df, M1[1]);
            M2[1] = mad(K<R>(w), sm, M2[1]);
        }
        if (c2) {
            M1[2] = mad(K<R>(w * c2), df, M1[2]);
            M2[2] = mad(K<R>(w), sm, M2[2]);
        }
        if (c0 && c1) M2[3] = mad(K<R>(w * c0 * c1), sm, M2[3]);
        if (c0 && c2) M2[4] = mad(K<R>(w * c0 * c2), sm, M2[4]);
        if (c1 && c2) M2[5] = mad(K<R>(w * c1 * c2), sm, M2[5]);
    }
    const float hz = 1.f - 0.5f * om, hzm = 1.f - 0.5f * omm;
    // M2 u and M2 F (symmetric 3x3 stored xx yy zz xy xz yz)
    auto mul = [](const R (&S)[6], const R* v, R* out) {
        out[0] = mad(S[0], v[0], mad(S[3], v[1], S[4] * v[2]));
        out[1] = mad(S[3], v[0], mad(S[1], v[1], S[5] * v[2]));
        out[2] = mad(S[4], v[0], mad(S[5], v[1], S[2] * v[2]));
    };
    R M2u[3], M2F[3];
    mul(M2, u, M2u);
    mul(M2, F, M2F);
    // Z2 u = om M2u (+ bulk), H2 u = hz M2u (- bulk / 2), H2 F likewise
    R Z2u[3], H2u[3], H2F[3];
    R g0 = K<R>(1.f - om) * gb[0];  // the rest population's output, less rho_bar
    R bulk_c = K<R>(0.f);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        Z2u[d] = K<R>(om) * M2u[d];
        H2u[d] = K<R>(hz) * M2u[d];
        H2F[d] = K<R>(hz) * M2F[d];
    }
    if constexpr (COLL == CK_MRT_BULK) {
        // b_i = |c_i|^2 - 1, |b|^2_W = 2/3, sum_i w_i b_i c_ia c_ib = 2/9 delta_ab
        R e = K<R>(-L::w(0)) * gb[0];
#pragma unroll
        for (int kk = 0; kk < NP; ++kk) {
            const int i = kk + 1;
            const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
            if (c2 != 1) e = mad(K<R>(L::w(i) * (float)(c2 - 1)), SM[kk], e);
        }
        bulk_c = K<R>(P.proj_rate[0] * 1.5f) * e;
        g0 = g0 + bulk_c;
        const R c29 = K<R>(2.f / 9.f) * bulk_c, c19 = K<R>(-1.f / 9.f) * bulk_c;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            Z2u[d] = mad(c29, u[d], Z2u[d]);
            H2u[d] = mad(c19, u[d], H2u[d]);
            H2F[d] = mad(c19, F[d], H2F[d]);
        }
    }
    const R Z0 = K<R>(om) * M0, H0 = K<R>(hz) * M0;
    R Z1[3], H1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        Z1[d] = K<R>(omm) * M1[d];
        H1[d] = K<R>(hzm) * M1[d];
    }
    const R usq = mad(u[0], u[0], mad(u[1], u[1], u[2] * u[2]));
    R rho_bar = mad(Z0, mad(K<R>(-1.5f), usq, one),
                    mad(K<R>(3.f), mad(u[0], Z1[0], mad(u[1], Z1[1], u[2] * Z1[2])),
                        K<R>(4.5f) * mad(u[0], Z2u[0], mad(u[1], Z2u[1], u[2] * Z2u[2]))));
    R ub[3], Fb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const R t = mad(K<R>(3.f), Z1[d], mad(K<R>(9.f), Z2u[d], K<R>(-3.f) * u[d] * Z0));
        ub[d] = mad(rho, t, mad(K<R>(9.f), H2F[d], K<R>(-3.f) * F[d] * H0));
        Fb[d] = mad(K<R>(3.f), H1[d], mad(K<R>(9.f), H2u[d], K<R>(-3.f) * u[d] * H0));
    }
    R abar = K<R>(0.f);
    const R ra = rho * alpha;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        rho_bar = mad(Fb[d], K<R>(P.a[d]) - alpha * u[d], rho_bar);
        abar = abar - rho * Fb[d] * u[d];
        ub[d] = ub[d] - ra * Fb[d];
    }
    const R inv_s = qdiv(one, s);
    const R inv = qdiv(inv_s, rho);
    R mb[3];
    R sbar = K<R>(0.f);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        mb[d] = ub[d] * inv;
        rho_bar = rho_bar - ub[d] * mad(s, u[d], K<R>(-0.5f * P.a[d])) * inv;
        sbar = sbar - ub[d] * u[d] * inv_s;
    }
    abar = mad(K<R>(0.5f), sbar, abar);
    // output, scaled by k: gb - R^T gb + rho_bar + c . mb pair by pair
    const R kr = K<R>(k) * rho_bar;
    R kmb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) kmb[d] = K<R>(k) * mb[d];
    const R khp = K<R>(0.5f * (1.f - om) * k), khm = K<R>(0.5f * (1.f - omm) * k);
    const R nkhm = K<R>(-0.5f * (1.f - omm) * k);
    gb[0] = mad(K<R>(k), g0, kr);
    R kbulk = K<R>(k) * bulk_c;
#pragma unroll
    for (int kk = 0; kk < NP; ++kk) {
        const int i = kk + 1, o = opp<Q>(i);
        R base = kr;
        if constexpr (COLL == CK_MRT_BULK) {
            const int c2 = L::cx(i) * L::cx(i) + L::cy(i) * L::cy(i) + L::cz(i) * L::cz(i);
            if (c2 != 1) base = mad(K<R>(-(float)(c2 - 1)), kbulk, base);
        }
        const R pi = mad(khp, SM[kk], base);
        // c . mb with the sign that makes the first nonzero component of c
        // positive (no negation): sg c . kmb accumulated from that component
        const int c[3] = {L::cx(i), L::cy(i), L::cz(i)};
        const int first = c[0] ? 0 : (c[1] ? 1 : 2);
        const int sg = c[first] > 0 ? 1 : -1;
        R cm = kmb[first];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (d != first && c[d]) cm = sg * c[d] > 0 ? cm + kmb[d] : cm - kmb[d];
        if (sg > 0) {
            const R d = mad(khm, DF[kk], cm);  // hm DF + c . mb
            gb[i] = pi + d;
            gb[o] = pi - d;
        } else {
            const R d = mad(nkhm, DF[kk], cm);  // -(hm DF + c . mb)
            gb[i] = pi - d;
            gb[o] = pi + d;
        }
    }
    return abar;
}

}  // namespace
}  // namespace lbm
