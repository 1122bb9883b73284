// lbm_krylov.cu -- vector updates of the BiCGStab steady adjoint.
//
// The steady adjoint solves (I - L) x = s for the fixed point of the
// transposed step L linearised at the final state (implexity-ad/src/
// implicit.rs:49-67 semantics; the Neumann series sum_k L^k s is the other
// solver).  BiCGStab (van der Vorst, 1992) needs two applications of I - L per
// iteration -- the fused adjoint kernel (k_adjoint with KRY = 1) stores them
// and sums the dot products it can see -- and the three vector updates here.
// Everything stays on the device: the solver's scalars (rho, alpha, omega,
// beta) are formed by every thread from the compensated FP64 dot products in
// a small device block (SC_* in lbm_launch.h), so the host only reads the
// residual now and then.
//
// The solution x itself is never formed: the design gradient needs only
// B^T x (B = d step / d alpha), and B^T is linear, so the alpha cotangent
// accumulates alpha_i B^T p_i + omega_i B^T s_i from the per-cell alpha
// cotangents the two operator launches of iteration i write.
//
// Vectors are FP32 arrays in the adjoint layout (Q planes of n cells); solid
// cells' slots are zero in every vector and stay zero (no kernel writes them).
#include "lbm_device.cuh"

namespace lbm {
namespace {

__device__ __forceinline__ double pair(const double* sc, int k) { return __ldcg(sc + k) + __ldcg(sc + k + 1); }
__device__ __forceinline__ double finite_or_zero(double v) { return isfinite(v) ? v : 0.0; }

// rhat = p = r (the seed), rho_0 = <rhat, r> = <r, r>.
template <int Q>
__global__ void __launch_bounds__(BLOCK) k_kry_init(KryVectors a) {
    const uint32_t n = (uint32_t)a.n;
    double rr = 0.0;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < n; x += gridDim.x * BLOCK) {
        if (a.mask[x] & MASK_SOLID) continue;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float v = a.r[q * n + x];
            a.rhat[q * n + x] = v;
            a.p[q * n + x] = v;
            rr += (double)v * (double)v;
        }
    }
    Sums<2> sm;
    sm.init();
    sm.h[0] = rr;
    sm.h[1] = rr;
    finish_sums<2>(sm, a.sc + SC_KR, a.red);
}

// alpha = rho / <rhat, v>;  s = r - alpha v.
template <int Q>
__global__ void __launch_bounds__(BLOCK) k_kry_s(KryVectors a) {
    const uint32_t n = (uint32_t)a.n;
    const double rho = pair(a.sc, SC_KR);
    const double alpha = finite_or_zero(rho / pair(a.sc, SC_K1));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.sc[SC_RHO_PREV] = rho;
        a.sc[SC_ALPHA] = alpha;
    }
    const float al = (float)alpha;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < n; x += gridDim.x * BLOCK) {
        if (a.mask[x] & MASK_SOLID) continue;
#pragma unroll
        for (int q = 0; q < Q; ++q) a.s[q * n + x] = fmaf(-al, a.v[q * n + x], a.r[q * n + x]);
    }
}

// omega = <s, t> / <t, t>;  r = s - omega t;  abar += alpha B^T p + omega B^T s;
// the new <rhat, r> and <r, r>.
template <int Q>
__global__ void __launch_bounds__(BLOCK) k_kry_r(KryVectors a) {
    const uint32_t n = (uint32_t)a.n;
    const double omega = finite_or_zero(pair(a.sc, SC_K3 + 2) / pair(a.sc, SC_K3 + 4));
    const double alpha = __ldcg(a.sc + SC_ALPHA);
    if (blockIdx.x == 0 && threadIdx.x == 0) a.sc[SC_OMEGA] = omega;
    const float om = (float)omega, al = (float)alpha;
    double rr = 0.0, hr = 0.0;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < n; x += gridDim.x * BLOCK) {
        if (a.mask[x] & MASK_SOLID) continue;
        a.abar[x] = fmaf(om, a.abar_s[x], fmaf(al, a.abar_p[x], a.abar[x]));
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float v = fmaf(-om, a.t[q * n + x], a.s[q * n + x]);
            a.r[q * n + x] = v;
            rr += (double)v * (double)v;
            hr += (double)a.rhat[q * n + x] * (double)v;
        }
    }
    Sums<2> sm;
    sm.init();
    sm.h[0] = hr;
    sm.h[1] = rr;
    finish_sums<2>(sm, a.sc + SC_KR, a.red);
}

// beta = (rho_new / rho) (alpha / omega);  p = r + beta (p - omega v).
template <int Q>
__global__ void __launch_bounds__(BLOCK) k_kry_p(KryVectors a) {
    const uint32_t n = (uint32_t)a.n;
    const double omega = __ldcg(a.sc + SC_OMEGA);
    const double beta =
        omega != 0.0 ? finite_or_zero(pair(a.sc, SC_KR) / __ldcg(a.sc + SC_RHO_PREV) * (__ldcg(a.sc + SC_ALPHA) / omega))
                     : 0.0;
    const float be = (float)beta, om = (float)omega;
    for (uint32_t x = blockIdx.x * BLOCK + threadIdx.x; x < n; x += gridDim.x * BLOCK) {
        if (a.mask[x] & MASK_SOLID) continue;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const uint32_t i = q * n + x;
            a.p[i] = fmaf(be, fmaf(-om, a.v[i], a.p[i]), a.r[i]);
        }
    }
}

template <int Q>
cudaError_t launch_q(int op, const KryVectors& a, int grid, cudaStream_t s) {
    switch (op) {
        case KRY_INIT: k_kry_init<Q><<<grid, BLOCK, 0, s>>>(a); break;
        case KRY_S: k_kry_s<Q><<<grid, BLOCK, 0, s>>>(a); break;
        case KRY_R: k_kry_r<Q><<<grid, BLOCK, 0, s>>>(a); break;
        case KRY_P: k_kry_p<Q><<<grid, BLOCK, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_krylov(int Q, int op, const KryVectors& kv, int grid, cudaStream_t s) {
    if (Q == 19) return launch_q<19>(op, kv, grid, s);
    if (Q == 27) return launch_q<27>(op, kv, grid, s);
    return cudaErrorInvalidValue;
}

}  // namespace lbm
