// lbm_forward.cu -- the fused stream-collide step (pull, two arrays).
//
// One launch = one time step of the whole grid: pull from the current array
// (Streaming::stream with halfway bounce-back, solver.rs:131-157) -> port
// reconstruction (ports.rs:560-579; an extrapolating port cell pulls its
// inward neighbour's populations as well) -> admission reductions of the streamed
// state (solver.rs:714-755) -> optional (rho, u) record for the adjoint ->
// collision (BGK/TRT/MRT with Guo-Brinkman forcing) -> aligned store into the
// cell's own slots of the other array.  The pulled runs are staged through
// shared memory by a producer warp (bulk asynchronous copies into a
// STAGES-deep ring); see lbm_device.cuh.  Reading one array and writing
// another keeps every DRAM stream one-directional, which on this memory
// system sustains about a third more bandwidth than the in-place AA pattern.
#include "lbm_device.cuh"

namespace lbm {
namespace {

template <int Q, typename T>
struct FwdStage {
    T run[Q][Vec16<T>::RUN];
    uint32_t mask[FRUN];
    float alpha[FRUN];
};

// RSP = 1: the step also sums the responses of the state it reads (the
// stage objective's per-state values; vector_cell, solver.rs:835-895).
// DP = 1: FP64 collision arithmetic (FP32 storage only; collide_fused_dp).
template <int Q, int COLL, typename T, int AL, int RSP, int DP>
__global__ void __launch_bounds__(TPB, (Q == 19 ? 3 : 2)) k_forward(FwdArgs a) {
    using L = Lat<Q>;
    using S = FwdStage<Q, T>;
    constexpr int STAGES = ring_depth<S, T>();
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);  // stage loaded
    uint64_t* empty = full + STAGES;                      // stage consumed (outputs written into it)
    uint64_t* rdone = empty + STAGES;                     // stage inputs read by every consumer warp
    const T* A = static_cast<const T*>(a.src);
    T* D = static_cast<T*>(a.dst);
    const uint32_t n = (uint32_t)a.G.n;
    const uint32_t ntiles = (n + TILE - 1) / TILE;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // Outputs of a full tile leave through the stage: every consumer writes
    // its cell's values into the aligned head of each run once all warps have
    // read the stage, and the producer copies the Q runs to the cells' own
    // slots with bulk stores.  The last, partial tile stores directly.
    const bool bulk_ok = a.collide && a.bulk_store;
    DiagLocal acc;
    acc.init();
    double rsum[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // per-thread response sums (RSP)
    if (threadIdx.x == 0) {
#pragma unroll
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CONSUMER_WARPS);
            mbar_init(&rdone[s], CONSUMER_WARPS);
        }
        mbar_fence_init();
    }
    __syncthreads();
    if (warp == 0) {
        // producer warp: lane q issues the copy of direction q's run (lanes Q, Q+1
        // the mask and alpha runs), so a tile's copies leave in one instruction
        const uint32_t mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
        const int q = lane < Q ? lane : 0;
        const int64_t run0 = a.run0[q];
#pragma unroll 1
        for (uint32_t i = 0; i < mine + STAGES; ++i) {
            const int s = (int)(i % STAGES);
            const uint32_t round = i / STAGES;
            S* st = stage_at<S>(smem, s);
            if (round > 0) {
                // the tile loaded STAGES iterations ago is consumed; store it
                // (lane 0 waits; the whole warp leaves together on a timeout)
                bool done = true;
                if (lane == 0) done = mbar_wait(&empty[s], (round - 1) & 1u, a.err);
                if (!__shfl_sync(0xffffffffu, done, 0)) break;
                const uint32_t x0 = (blockIdx.x + (i - STAGES) * gridDim.x) * TILE;
                if (bulk_ok && x0 + TILE <= n) {
                    if (lane < Q) {
                        bulk_s2g(D + ((size_t)lane * n + x0), &st->run[lane][0], TILE * (int)sizeof(T));
                        bulk_commit();
                        bulk_wait_read0();  // the stage may be refilled once the stores have read it
                    }
                    __syncwarp();
                }
            }
            if (i < mine) {
                const uint32_t x0 = (blockIdx.x + i * gridDim.x) * TILE;
                if (lane == 0) mbar_expect_tx(&full[s], Q * Vec16<T>::BYTES + 2 * FRUN_BYTES);
                __syncwarp();
                if (lane < Q) bulk_g2s(&st->run[lane][0], A + (run0 + x0), Vec16<T>::BYTES, &full[s]);
                else if (lane == Q) bulk_g2s(&st->mask[0], a.mask + x0, FRUN_BYTES, &full[s]);
                else if (lane == Q + 1) bulk_g2s(&st->alpha[0], a.alpha + x0, FRUN_BYTES, &full[s]);
            }
        }
        bulk_wait_all();
    } else {
        const int c = threadIdx.x - 32;
        int s = 0;
        uint32_t round = 0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            const bool ok = mbar_wait(&full[s], round & 1u, a.err);
            S* st = stage_at<S>(smem, s);
            const uint32_t x = tile * TILE + c;
            const bool bulk = bulk_ok && tile * TILE + TILE <= n;
            // populations in storage units (g = f - w, or (f - w)/w for 16-bit storage)
            constexpr int SC = Cvt<T>::scaled ? 1 : 0;
            float v[Q];
            const uint32_t m = ok && x < n ? st->mask[c] : MASK_SOLID;
            const bool fluid = !(m & MASK_SOLID);
            if constexpr (RSP) {
                if (!fluid && ok && x < n) rsum[5] += (double)a.phi[x];
            }
            if (fluid) {
                if (!(m & MASK_WRAP)) {
#pragma unroll
                    for (int q = 0; q < Q; ++q)
                        v[q] = sdec<T>(st->run[q][(AL ? rund_aligned<Q, T, -1>(q) : a.rund[q]) + c]);
                    if (m & LINK_BITS) {
                        // halfway bounce-back: the cell's own opposite slot
#pragma unroll
                        for (int q = 1; q < Q; ++q)
                            if ((m >> q) & 1u) v[q] = sdec<T>(A[opp<Q>(q) * n + x]);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < Q; ++q) v[q] = sdec<T>(A[pull_index<Q>(a.G, x, m, q)]);
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&rdone[s]);
            if (fluid) {
                const float alpha = st->alpha[c];
                float exch = 0.f;
                if (a.apply_ports && (m & MASK_PORT)) {
                    // the port maps act on g = f - w
                    if constexpr (SC) {
#pragma unroll
                        for (int q = 0; q < Q; ++q) v[q] *= L::w(q);
                    }
                    exch = port_state<Q, T>(a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1], A, a.G, a.mask, x, v);
                    if constexpr (SC) {
#pragma unroll
                        for (int q = 0; q < Q; ++q) v[q] *= (float)(1.0 / L::wd(q));
                    }
                }
                const float mn = a.diag ? min_population<Q, SC>(v) : 0.f;
                float S[6];
                if (RSP || (a.record && a.record_s)) {
                    // second moments of g: the stage seeds of the adjoint, the dissipation
                    float g[Q];
#pragma unroll
                    for (int q = 0; q < Q; ++q) g[q] = SC ? L::w(q) * v[q] : v[q];
                    second_moments<Q>(g, S);
                    if (a.record && a.record_s) {
#pragma unroll
                        for (int e = 0; e < 6; ++e) a.record[(size_t)(4 + e) * n + x] = S[e];
                    }
                }
                // relaxation rates: the problem's, or the cell's own (Tau::PerCell, BGK only)
                float om = a.P.omega, omm = a.P.om;
                if (a.omega_cell) om = omm = a.omega_cell[x];
                Macro M;
                if constexpr (DP) M = collide_fused_dp<Q, COLL>(v, alpha, a.P, a.collide, om, omm);
                else M = collide_fused<Q, COLL, SC>(v, alpha, a.P, a.collide, om, omm);
                if constexpr (RSP) {
                    float r6[6];
                    response_cell<Q>(M.rp, M.u, S, alpha, a.sp, a.P, r6);
#pragma unroll
                    for (int k = 0; k < 5; ++k) rsum[k] += (double)r6[k];
                    rsum[5] += (double)a.phi[x];
                    if (m & MASK_PORT) {
                        const float dpw = a.ports[((m >> MASK_PORT_SHIFT) & 7u) - 1].dp_weight;
                        rsum[6] += (double)(dpw * a.sp.dens * M.rp * a.sp.vel * a.sp.vel / 3.f);
                    }
                    rsum[7] += (double)r6[5];
                }
                if (a.diag) {
                    acc.mass += M.rp;
                    acc.exch += exch;
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
                if (a.collide && !bulk) store_own_pop<Q, T>(D, n, x, v, a.step);
            }
            if (bulk) {
                // every warp has read its inputs: overwrite the run heads with this cell's outputs
                // (a solid cell carries its held populations over)
                if (!mbar_wait(&rdone[s], round & 1u, a.err)) {
                    // nothing is stored for this tile; the error flag fails the step
                } else if (fluid) {
                    uint32_t rs = 0;
                    if constexpr (Cvt<T>::scaled) rs = cell_seed(x, a.step);
                    senc_sr_all<Q, T>(v, rs, [&](int q, T e) { st->run[q][c] = e; });
                } else {
#pragma unroll
                    for (int q = 0; q < Q; ++q) st->run[q][c] = A[q * n + x];
                }
                fence_proxy_async_smem();
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
    if constexpr (RSP) {
        Sums<8> t;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            t.h[k] = rsum[k];
            t.l[k] = 0.0;
        }
        finish_sums<8>(t, a.stage, a.red2);
    }
}

template <int Q, int COLL, typename T, int AL, int RSP, int DP>
cudaError_t run_forward_rs(const FwdArgs& a, cudaStream_t s) {
    constexpr size_t smem = pipe_bytes<FwdStage<Q, T>, ring_depth<FwdStage<Q, T>, T>()>();
    static bool attr = false;
    if (!attr) {
        cudaError_t e = set_smem(k_forward<Q, COLL, T, AL, RSP, DP>, smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int grid = persistent_grid((const void*)k_forward<Q, COLL, T, AL, RSP, DP>, a.G.n, smem, TPB, TILE);
    k_forward<Q, COLL, T, AL, RSP, DP><<<grid, TPB, smem, s>>>(a);
    return cudaGetLastError();
}

template <int Q, int COLL, typename T, int AL>
cudaError_t run_forward_al(const FwdArgs& a, cudaStream_t s) {
    if (a.dp_collision) {
        // FP64 collision arithmetic exists for FP32 storage only
        if constexpr (std::is_same<T, float>::value)
            return a.stage ? run_forward_rs<Q, COLL, T, AL, 1, 1>(a, s) : run_forward_rs<Q, COLL, T, AL, 0, 1>(a, s);
        else
            return cudaErrorInvalidValue;
    }
    return a.stage ? run_forward_rs<Q, COLL, T, AL, 1, 0>(a, s) : run_forward_rs<Q, COLL, T, AL, 0, 0>(a, s);
}

// The run offsets are compile-time constants when every run table entry
// matches rund_aligned (plane stride and strides multiples of the vector).
template <int Q, typename T, int DIR>
bool table_is_aligned(const int32_t* rund) {
    for (int q = 0; q < Q; ++q) {
        const int d = DIR * (Q == 19 ? Lat<19>::cz(q) : Lat<27>::cz(q));
        if (rund[q] != (d < 0 ? d + Vec16<T>::V : d)) return false;
    }
    return true;
}

template <int Q, int COLL, typename T>
cudaError_t run_forward(const FwdArgs& a, cudaStream_t s) {
    return table_is_aligned<Q, T, -1>(a.rund) ? run_forward_al<Q, COLL, T, 1>(a, s) : run_forward_al<Q, COLL, T, 0>(a, s);
}

}  // namespace

bool staged_aligned(const void* base, const int64_t* run0, int nrun, size_t elem) {
    const uintptr_t b = reinterpret_cast<uintptr_t>(base);
    if (b % 16) return false;
    for (int q = 0; q < nrun; ++q)
        if ((b + (uintptr_t)(run0[q] * (int64_t)elem)) % 16) return false;
    return true;
}

void run_table(int Q, const Geometry& G, int dir, int vec, int64_t* run0, int32_t* rund) {
    for (int q = 0; q < Q; ++q) {
        const int cx = Q == 19 ? Lat<19>::cx(q) : Lat<27>::cx(q);
        const int cy = Q == 19 ? Lat<19>::cy(q) : Lat<27>::cy(q);
        const int cz = Q == 19 ? Lat<19>::cz(q) : Lat<27>::cz(q);
        const int64_t first = (int64_t)q * G.n + dir * (cx * G.sx + cy * G.sy + cz);
        int64_t d = first % vec;
        if (d < 0) d += vec;
        run0[q] = first - d;
        rund[q] = (int32_t)d;
    }
}

cudaError_t launch_forward(int Q, int coll, int storage, const FwdArgs& a0, int grid, cudaStream_t s) {
    (void)grid;
    FwdArgs a = a0;
    run_table(Q, a.G, -1, storage == ST_F32 ? 4 : 8, a.run0, a.rund);
    // every bulk copy needs 16-byte aligned addresses: refuse to launch otherwise
    const size_t es = storage == ST_F32 ? 4 : 2;
    if (!staged_aligned(a.src, a.run0, Q, es) || !staged_aligned(a.mask, nullptr, 0, 4) ||
        !staged_aligned(a.alpha, nullptr, 0, 4) || (a.bulk_store && !staged_aligned(a.dst, nullptr, 0, es)))
        return cudaErrorMisalignedAddress;
    if (Q == 19) {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward<19, CK_MRT, T>(a, s))
        } else if (coll == CK_MRT_BULK) {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward<19, CK_MRT_BULK, T>(a, s))
        } else {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward<19, CK_PAIRS, T>(a, s))
        }
    } else {
        if (coll == CK_MRT) {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward<27, CK_MRT, T>(a, s))
        } else if (coll == CK_MRT_BULK) {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward<27, CK_MRT_BULK, T>(a, s))
        } else {
            LBM_STORAGE_DISPATCH(storage, T, return run_forward<27, CK_PAIRS, T>(a, s))
        }
    }
    return cudaGetLastError();
}

}  // namespace lbm
