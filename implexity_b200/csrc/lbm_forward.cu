// lbm_forward.cu -- the fused collide-stream step (AA pattern, in place).
//
// One launch = one time step of the whole grid: load (AA parity) -> port
// reconstruction (ports.rs:560-579) -> admission reductions of the loaded
// state (solver.rs:714-755) -> optional (rho, u) record for the adjoint ->
// collision (BGK/TRT/MRT with Guo-Brinkman forcing) -> AA store.  The loads
// are staged through shared memory by a producer warp (bulk asynchronous
// copies into a STAGES-deep ring); see lbm_device.cuh.
#include "lbm_device.cuh"

namespace lbm {
namespace {

template <int Q, typename T>
struct FwdStage {
    T run[Q][Vec16<T>::RUN];
    uint32_t mask[FRUN];
    float alpha[FRUN];
};

template <int Q, int COLL, typename T, int PAR>
__global__ void __launch_bounds__(TPB, (Q == 19 ? 3 : 2)) k_forward(FwdArgs a) {
    using L = Lat<Q>;
    using S = FwdStage<Q, T>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + STAGES;
    T* A = static_cast<T*>(a.pop);
    const uint32_t n = (uint32_t)a.G.n;
    const uint32_t ntiles = (n + TILE - 1) / TILE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    DiagLocal acc;
    acc.init();
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
        // producer: one lane issues the runs of every tile of this block
        if (lane == 0) {
            int s = 0;
            uint32_t round = 0;  // completed passes over the ring
            for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
                if (round > 0 && !mbar_wait(&empty[s], (round - 1) & 1u, a.err)) break;
                S* st = stage_at<S>(smem, s);
                const uint32_t x0 = tile * TILE;
                mbar_expect_tx(&full[s], Q * Vec16<T>::BYTES + 2 * FRUN_BYTES);
#pragma unroll 1
                for (int q = 0; q < Q; ++q) bulk_g2s(&st->run[q][0], A + (a.run0[q] + x0), Vec16<T>::BYTES, &full[s]);
                bulk_g2s(&st->mask[0], a.mask + x0, FRUN_BYTES, &full[s]);
                bulk_g2s(&st->alpha[0], a.alpha + x0, FRUN_BYTES, &full[s]);
                if (++s == STAGES) {
                    s = 0;
                    ++round;
                }
            }
        }
    } else {
        const int c = threadIdx.x - 32;
        int s = 0;
        uint32_t round = 0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const bool ok = mbar_wait(&full[s], round & 1u, a.err);
            const S* st = stage_at<S>(smem, s);
            const uint32_t x = tile * TILE + c;
            if (ok && x < n) {
                const uint32_t m = st->mask[c];
                if (!(m & MASK_SOLID)) {
                    float g[Q];
                    if (PAR == 0 || !(m & MASK_WRAP)) {
#pragma unroll
                        for (int q = 0; q < Q; ++q) {
                            if (PAR == 1 && ((m >> q) & 1u)) g[q] = pdec<Q, T>(A[q * n + x], q);
                            else g[q] = pdec<Q, T>(st->run[q][a.rund[q] + c], q);
                        }
                    } else {
                        load_pop<Q, T>(A, a.G, x, m, PAR, g);
                    }
                    float exch = 0.f;
                    if (a.apply_ports && (m & MASK_PORT))
                        exch = apply_port<Q>(a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], g);
                    const float alpha = st->alpha[c];
                    Macro M = macroscopic<Q>(g, alpha, a.P);
                    if (a.diag) {
                        acc.mass += M.rp;
                        acc.exch += exch;
                        float mn = INFINITY;
#pragma unroll
                        for (int q = 0; q < Q; ++q) mn = fminf(mn, L::w(q) + g[q]);
                        acc.minf = fminf(acc.minf, mn);
                        acc.maxu2 = fmaxf(acc.maxu2, M.u[0] * M.u[0] + M.u[1] * M.u[1] + M.u[2] * M.u[2]);
                        // any non-finite population makes the density sum non-finite
                        if (!isfinite(M.rp)) acc.nf = 1;
                    }
                    if (a.record) {
                        a.record[x] = M.rp;
                        a.record[n + x] = M.u[0];
                        a.record[2 * n + x] = M.u[1];
                        a.record[3 * n + x] = M.u[2];
                    }
                    if (a.collide) {
                        collide<Q, COLL>(g, M, a.P);
                        store_pop_p<Q, T, PAR>(A, a.G, x, m, g, a.step);
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            if (++s == STAGES) {
                s = 0;
                ++round;
            }
        }
    }
    if (a.diag) finish_diag(acc, a.diag, a.red);
}

template <int Q, int COLL, typename T, int PAR>
cudaError_t run_forward(const FwdArgs& a, cudaStream_t s) {
    constexpr size_t smem = pipe_bytes<FwdStage<Q, T>>();
    static bool attr = false;
    if (!attr) {
        cudaError_t e = set_smem(k_forward<Q, COLL, T, PAR>, smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int grid = persistent_grid((const void*)k_forward<Q, COLL, T, PAR>, a.G.n, smem, TPB, TILE);
    k_forward<Q, COLL, T, PAR><<<grid, TPB, smem, s>>>(a);
    return cudaGetLastError();
}

template <int Q, int COLL, typename T>
cudaError_t run_forward_p(const FwdArgs& a, cudaStream_t s) {
    return a.parity == 0 ? run_forward<Q, COLL, T, 0>(a, s) : run_forward<Q, COLL, T, 1>(a, s);
}

}  // namespace

void run_table(int Q, const Geometry& G, int parity, int dir, int vec, int64_t* run0, int32_t* rund) {
    for (int q = 0; q < Q; ++q) {
        int64_t first;
        if (parity == 0) {
            first = (int64_t)q * G.n;
        } else {
            const int cx = Q == 19 ? Lat<19>::cx(q) : Lat<27>::cx(q);
            const int cy = Q == 19 ? Lat<19>::cy(q) : Lat<27>::cy(q);
            const int cz = Q == 19 ? Lat<19>::cz(q) : Lat<27>::cz(q);
            const int o = q == 0 ? 0 : Q - q;
            first = (int64_t)o * G.n + dir * (cx * G.sx + cy * G.sy + cz);
        }
        int64_t d = first % vec;
        if (d < 0) d += vec;
        run0[q] = first - d;
        rund[q] = (int32_t)d;
    }
}

cudaError_t launch_forward(int Q, int coll, int storage, const FwdArgs& a0, int grid, cudaStream_t s) {
    (void)grid;
    FwdArgs a = a0;
    run_table(Q, a.G, a.parity, -1, storage == ST_F32 ? 4 : 8, a.run0, a.rund);
    if (Q == 19) {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward_p<19, CK_MRT, T>(a, s))
        } else {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward_p<19, CK_PAIRS, T>(a, s))
        }
    } else {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward_p<27, CK_MRT, T>(a, s))
        } else {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward_p<27, CK_PAIRS, T>(a, s))
        }
    }
    return cudaGetLastError();
}

}  // namespace lbm
