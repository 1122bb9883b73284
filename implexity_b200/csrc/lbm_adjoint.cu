// lbm_adjoint.cu -- one transposed step of the discrete adjoint.
//
// interval_vjp (solver.rs:642-674) restated for the two-array layout: the
// stored adjoint array holds Ports^T C^T of the cotangent of the streamed
// state; one transposed step pulls it with the velocities reversed (the
// transpose of the pull of Streaming::stream, solver.rs:131-157), takes the
// collision transpose at the recorded forward (rho, u) (collide_pairs_vjp,
// moving/collision.rs:492-570, with the Brinkman chain of moving/psm.rs:
// 402-486), accumulates the alpha cotangent per cell, applies the transposed
// port map at port cells (apply_ports_vjp, ports.rs:582-621) and stores into
// the cell's own slots of the other array.  Loads are staged like the
// forward step (lbm_device.cuh).
#include "lbm_device.cuh"

namespace lbm {
namespace {

template <int Q, typename T, int NREC>
struct AdjStage {
    T run[Q][Vec16<T>::RUN];
    float rec[NREC][FRUN];
    uint32_t mask[FRUN];
    float alpha[FRUN];
};

// One cell c of a staged tile of the transposed step (mask m, the running
// alpha cotangent ab_prev): the general path.
template <int Q, int COLL, typename T, int AL, int STG, typename S>
__device__ __forceinline__ void adj_one_cell(const AdjArgs& a, const S* st, int c, uint32_t x, uint32_t m, float ab_prev,
                                             const T* B, T* D, uint32_t n, float s_in, float k_out, double& nsum) {
    const bool fluid = !(m & MASK_SOLID);
    if (!fluid) return;
    float v[Q];
    if (!(m & MASK_WRAP)) {
#pragma unroll
        for (int q = 0; q < Q; ++q)
            v[q] = Cvt<T>::to(st->run[q][(AL ? rund_aligned<Q, T, 1>(q) : a.rund[q]) + c]);
        if (m & LINK_BITS) {
            // transposed bounce-back: the cell's own opposite slot
#pragma unroll
            for (int q = 1; q < Q; ++q)
                if ((m >> opp<Q>(q)) & 1u) v[q] = Cvt<T>::to(B[opp<Q>(q) * n + x]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] = Cvt<T>::to(B[pull_adj_index<Q>(a.G, x, m, q)]);
    }
    const float u[3] = {st->rec[1][a.recd[1] + c], st->rec[2][a.recd[2] + c], st->rec[3][a.recd[3] + c]};
    const float rp = st->rec[0][a.recd[0] + c];
    // v stays in the stored scale (the transposed step is linear): the
    // alpha cotangent is rescaled once, the output by out_scale / in_scale --
    // inside the collision transpose, unless a stage seed or a port transpose
    // still acts on v before it is stored
    float om = a.P.omega, omm = a.P.om;
    if (a.omega_cell) om = omm = a.omega_cell[x];  // Tau::PerCell (BGK only)
    const bool post = (STG && a.stage) || (a.port_transpose && (m & MASK_PORT));
    float ab = collide_vjp<Q, COLL>(v, rp, u, st->alpha[c], a.P, om, omm, post ? 1.f : k_out) * a.in_scale_inv;
    if constexpr (STG) {
        if (a.stage) {
            // the stage seed of this state: d(w . responses)/dg from its record
            float Sm[6], fb[Q];
#pragma unroll
            for (int e = 0; e < 6; ++e) Sm[e] = st->rec[4 + e][a.recd[4 + e] + c];
            const PortMap* pm = (m & MASK_PORT) ? &a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1] : nullptr;
            ab += response_vjp<Q>(rp, u, Sm, st->alpha[c], pm ? pm->dp_weight : 0.f, pm != nullptr, a.seed,
                                  a.P, fb);
#pragma unroll
            for (int q = 0; q < Q; ++q) v[q] = fmaf(fb[q], s_in, v[q]);
        }
    }
    a.abar[x] = fmaf(ab, a.abar_factor, ab_prev);
    if (a.port_transpose && (m & MASK_PORT)) {
        const PortMap& pm = a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1];
        if (!pm.recon) {
            port_transpose<Q>(pm, v);
        } else {
            // nonlinear ports, linearised at the recorded (rho, j / rho)
            // of port_lin_cell (zero acceleration: u = j / (rho (1 +
            // alpha / 2))); an extrapolating port's share for its
            // neighbour stays in this cell's slots until the move that
            // follows the step (launch_nee_move)
            const size_t xm = (size_t)port_lin_cell(pm, x);
            const float sc = 1.f + 0.5f * a.alpha[xm];
            const float um[3] = {a.record[(size_t)n + xm] * sc, a.record[2 * (size_t)n + xm] * sc,
                                 a.record[3 * (size_t)n + xm] * sc};
            port_vjp<Q>(pm, a.record[xm], um, v);
        }
    }
    if (post) {
#pragma unroll
        for (int q = 0; q < Q; ++q) v[q] *= k_out;
    }
    store_own_lam<Q, T>(D, n, x, v, 1.f);
    if (a.norm2) {
#pragma unroll
        for (int q = 0; q < Q; ++q) nsum += (double)v[q] * (double)v[q];
    }
}

// STG = 1: the stage-objective variant, which reads the second moments of
// the recorded state as well and adds the state's response VJP.
// Residency: D3Q19 with 16-bit storage runs three blocks per SM (72
// registers): its step is bound by latency and instruction issue, not bytes,
// and a third block's warps hide more of it; the others keep two blocks.
template <int Q, int COLL, typename T, int AL, int STG>
__global__ void __launch_bounds__(TPB, (sizeof(T) == 2 && Q == 19 ? 3 : 2)) k_adjoint(AdjArgs a) {
    constexpr int NREC = STG ? 10 : 4;
    using S = AdjStage<Q, T, NREC>;
    constexpr int NCOPY = Q + NREC + 2;  // runs of lambda, the record, mask and alpha
    constexpr int STAGES = ring_depth<S, T>();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);  // stage loaded
    uint64_t* empty = full + STAGES;                      // stage consumed
    const T* B = static_cast<const T*>(a.src);
    T* D = static_cast<T*>(a.dst);
    const uint32_t n = (uint32_t)a.G.n;
    const uint32_t ntiles = (n + TILE - 1) / TILE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double nsum = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CONSUMER_WARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (warp == 0) {
        // producer warp, as in the forward step: each lane issues its runs' copies.
        // (The outputs leave through direct stores: this step is bound by its
        // arithmetic, and staging the outputs would add a block-wide wait.)
        const uint32_t mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
#pragma unroll 1
        for (uint32_t i = 0; i < mine + STAGES; ++i) {
            const int s = (int)(i % STAGES);
            const uint32_t round = i / STAGES;
            S* st = stage_at<S>(smem, s);
            if (round > 0) {
                bool done = true;
                if (lane == 0) done = mbar_wait(&empty[s], (round - 1) & 1u, a.err);
                if (!__shfl_sync(0xffffffffu, done, 0)) break;
            }
            if (i < mine) {
                const uint32_t x0 = (blockIdx.x + i * gridDim.x) * TILE;
                if (lane == 0) mbar_expect_tx(&full[s], Q * Vec16<T>::BYTES + (NREC + 2) * FRUN_BYTES);
                __syncwarp();
#pragma unroll 1
                for (int k = lane; k < NCOPY; k += 32) {
                    if (k < Q) bulk_g2s(&st->run[k][0], B + (a.run0[k] + x0), Vec16<T>::BYTES, &full[s]);
                    else if (k < Q + NREC)
                        bulk_g2s(&st->rec[k - Q][0], a.record + (a.rec0[k - Q] + x0), FRUN_BYTES, &full[s]);
                    else if (k == Q + NREC) bulk_g2s(&st->mask[0], a.mask + x0, FRUN_BYTES, &full[s]);
                    else bulk_g2s(&st->alpha[0], a.alpha + x0, FRUN_BYTES, &full[s]);
                }
            }
        }
    } else {
        const int c0 = threadIdx.x - 32;
        int s = 0;
        uint32_t round = 0;
        const float s_in = 1.f / a.in_scale_inv;        // stored scale of the input
        const float k_out = a.out_scale * a.in_scale_inv;  // stored input -> stored output
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const uint32_t x = tile * TILE + c0;
            // the running alpha cotangent, read before the wait so that its
            // latency hides behind the staged copies and the collision
            const float ab_prev = (!a.overwrite_abar && x < n) ? a.abar[x] : 0.f;
            const bool ok = mbar_wait(&full[s], round & 1u, a.err);
            const S* st = stage_at<S>(smem, s);
            adj_one_cell<Q, COLL, T, AL, STG>(a, st, c0, x, ok && x < n ? st->mask[c0] : MASK_SOLID, ab_prev, B, D, n,
                                              s_in, k_out, nsum);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            if (++s == STAGES) {
                s = 0;
                ++round;
            }
        }
    }
    if (a.norm2) {
        Sums<1> sm;
        sm.init();
        sm.h[0] = nsum;
        finish_sums<1>(sm, a.norm2, a.red);
    }
}

template <int Q, int COLL, typename T, int AL, int STG>
cudaError_t run_adjoint_al(const AdjArgs& a, cudaStream_t s) {
    constexpr size_t smem = pipe_bytes<AdjStage<Q, T, STG ? 10 : 4>, ring_depth<AdjStage<Q, T, STG ? 10 : 4>, T>()>();
    static bool attr = false;
    if (!attr) {
        cudaError_t e = set_smem(k_adjoint<Q, COLL, T, AL, STG>, smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int grid = persistent_grid((const void*)k_adjoint<Q, COLL, T, AL, STG>, a.G.n, smem, TPB, TILE);
    k_adjoint<Q, COLL, T, AL, STG><<<grid, TPB, smem, s>>>(a);
    return cudaGetLastError();
}

template <int Q, typename T>
bool adj_table_is_aligned(const int32_t* rund) {
    for (int q = 0; q < Q; ++q) {
        const int d = Q == 19 ? Lat<19>::cz(q) : Lat<27>::cz(q);
        if (rund[q] != (d < 0 ? d + Vec16<T>::V : d)) return false;
    }
    return true;
}

template <int Q, int COLL, typename T>
cudaError_t run_adjoint(const AdjArgs& a, cudaStream_t s) {
    const bool al = adj_table_is_aligned<Q, T>(a.rund);
    if (a.rec_planes == 10)
        return al ? run_adjoint_al<Q, COLL, T, 1, 1>(a, s) : run_adjoint_al<Q, COLL, T, 0, 1>(a, s);
    return al ? run_adjoint_al<Q, COLL, T, 1, 0>(a, s) : run_adjoint_al<Q, COLL, T, 0, 0>(a, s);
}

}  // namespace

cudaError_t launch_adjoint(int Q, int coll, int lstorage, const AdjArgs& a0, int grid, cudaStream_t s) {
    (void)grid;
    AdjArgs a = a0;
    run_table(Q, a.G, +1, lstorage == ST_F32 ? 4 : 8, a.run0, a.rund);
    if (a.rec_planes != 4 && a.rec_planes != 10) return cudaErrorInvalidValue;
    for (int k = 0; k < a.rec_planes; ++k) {
        const int64_t first = (int64_t)k * a.G.n;
        a.recd[k] = (int32_t)(first % 4);
        a.rec0[k] = first - a.recd[k];
    }
    // every bulk copy needs 16-byte aligned addresses: refuse to launch otherwise
    if (!staged_aligned(a.src, a.run0, Q, lstorage == ST_F32 ? 4 : 2) ||
        !staged_aligned(a.record, a.rec0, a.rec_planes, 4) ||
        !staged_aligned(a.mask, nullptr, 0, 4) || !staged_aligned(a.alpha, nullptr, 0, 4))
        return cudaErrorMisalignedAddress;
    if (Q == 19) {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(lstorage, T, return run_adjoint<19, CK_MRT, T>(a, s))
        } else if (coll == CK_MRT_BULK) {
            LBM_STORAGE_DISPATCH(lstorage, T, return run_adjoint<19, CK_MRT_BULK, T>(a, s))
        } else {
            LBM_STORAGE_DISPATCH(lstorage, T, return run_adjoint<19, CK_PAIRS, T>(a, s))
        }
    } else {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(lstorage, T, return run_adjoint<27, CK_MRT, T>(a, s))
        } else if (coll == CK_MRT_BULK) {
            LBM_STORAGE_DISPATCH(lstorage, T, return run_adjoint<27, CK_MRT_BULK, T>(a, s))
        } else {
            LBM_STORAGE_DISPATCH(lstorage, T, return run_adjoint<27, CK_PAIRS, T>(a, s))
        }
    }
    return cudaGetLastError();
}

}  // namespace lbm
