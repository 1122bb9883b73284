// lbm_noalloc.cu -- admission statistics of a caller-held device state without
// any device allocation (lbm_state_stats_noalloc, include/lbm_b200.h).
//
// Some callers cannot call cudaMalloc: code running inside another
// framework's memory pool or arena (the pool owns every device allocation and
// forbids out-of-band ones), or embedded hosts that budget device memory up
// front.  They already hold
// their populations on the device and only want the numbers the admission
// check of LbmProblem::admit (solver.rs:708-793) computes for one state.
// The reduction here is the same one the stepping kernels run every step
// (per-block compensated partials, then the last block combines them), but
// its scratch is a file-scope static __device__ array instead of memory from
// an lbm_handle: every GPU that loads the library holds it until the process
// exits.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "../../include/lbm_b200.h"
#include "lbm_device.cuh"

namespace lbm {

// Scratch layout: the last-block ticket counter in the first 256 bytes, then
// NOALLOC_PARTIALS doubles per block for at most NOALLOC_MAX_BLOCKS blocks
// (65 792 bytes in all).  The launch never uses more blocks than that; the
// grid-stride loop covers any larger state.
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_BLOCKS = 1024;
constexpr int NOALLOC_PARTIALS = 8;
constexpr size_t NOALLOC_SCRATCH_BYTES = 256 + (size_t)NOALLOC_MAX_BLOCKS * NOALLOC_PARTIALS * sizeof(double);

static __device__ __align__(256) unsigned char g_stats_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

// One pass over the state: fluid mass sum(rho), minimum population over fluid
// cells, maximum |u| with the implicit half-step Brinkman velocity
// (solver.rs:190-196), and a flag for non-finite populations.
template <int Q>
__global__ void __launch_bounds__(NOALLOC_THREADS) k_state_stats(const float* __restrict__ f, uint32_t n,
                                                                 const uint8_t* __restrict__ solid,
                                                                 const float* __restrict__ alpha, float ax, float ay,
                                                                 float az, unsigned char* scratch, double* out) {
    using L = Lat<Q>;
    double mass = 0.0;
    float minf = INFINITY, maxu2 = 0.f;
    int nf = 0;
    for (uint32_t x = blockIdx.x * NOALLOC_THREADS + threadIdx.x; x < n; x += gridDim.x * NOALLOC_THREADS) {
        float rho = 0.f, jx = 0.f, jy = 0.f, jz = 0.f, mn = INFINITY;
        bool finite = true;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float v = f[q * n + x];
            rho += v;
            if (L::cx(q)) jx += L::cx(q) * v;
            if (L::cy(q)) jy += L::cy(q) * v;
            if (L::cz(q)) jz += L::cz(q) * v;
            mn = fminf(mn, v);
            finite = finite && isfinite(v);
        }
        // finiteness over every cell, solid ones included; the other
        // statistics over fluid cells (solver.rs:714-726)
        if (!finite) nf = 1;
        if (solid && solid[x]) continue;
        const float s = 1.f + 0.5f * (alpha ? alpha[x] : 0.f);
        const float ux = (jx / rho + 0.5f * ax) / s, uy = (jy / rho + 0.5f * ay) / s, uz = (jz / rho + 0.5f * az) / s;
        mass += (double)rho;
        minf = fminf(minf, mn);
        maxu2 = fmaxf(maxu2, ux * ux + uy * uy + uz * uz);
    }
    DiagAcc v;
    v.mh = mass;
    v.ml = 0.0;
    v.eh = v.el = 0.0;
    v.minf = minf;
    v.maxu2 = maxu2;
    v.nf = nf;
    v = block_reduce(v);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    double* partial = reinterpret_cast<double*>(scratch + 256);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double* p = partial + (size_t)blockIdx.x * NOALLOC_PARTIALS;
        p[0] = v.mh;
        p[1] = v.ml;
        p[2] = v.minf;
        p[3] = v.maxu2;
        p[4] = v.nf;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    DiagAcc acc;
    acc.init();
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double* p = partial + (size_t)b * NOALLOC_PARTIALS;
        DiagAcc o;
        o.init();
        o.mh = __ldcg(p + 0);
        o.ml = __ldcg(p + 1);
        o.minf = (float)__ldcg(p + 2);
        o.maxu2 = (float)__ldcg(p + 3);
        o.nf = (int)__ldcg(p + 4);
        acc.merge(o);
    }
    acc = block_reduce(acc);
    if (threadIdx.x == 0) {
        out[0] = acc.mh + acc.ml;
        out[1] = acc.minf;
        out[2] = sqrt((double)acc.maxu2);
        out[3] = acc.nf ? 1.0 : 0.0;
        *counter = 0;
        __threadfence();
    }
}

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
void* g_scratch_ptr[MAX_DEVICES] = {};

// Device address of g_stats_scratch on the current device, looked up once per
// device (the host-side name of the array is not a device address).  The
// cached address belongs to the device's primary context: after
// cudaDeviceReset the module is loaded again and the array may move, so the
// entry point must not be used on that device for the rest of the process.
cudaError_t scratch_on_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_stats_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

}  // namespace
}  // namespace lbm

using namespace lbm;

extern "C" lbm_status lbm_state_stats_noalloc(int32_t q, int64_t cells, const float* populations,
                                             const uint8_t* solid, const float* alpha,
                                             const double* acceleration_lattice, double* out4, void* stream) {
    if (q != 19 && q != 27) {
        set_thread_error("lbm_state_stats_noalloc: q must be 19 or 27");
        return LBM_E_CONTRACT;
    }
    if (cells < 1 || (int64_t)q * cells >= (int64_t(1) << 31)) {
        set_thread_error(
            "lbm_state_stats_noalloc: q * cells must lie in [1, 2^31); larger states exceed its 32-bit indexing");
        return LBM_E_CONTRACT;
    }
    if (!populations || !out4) {
        set_thread_error("lbm_state_stats_noalloc: populations and out4 must be device pointers");
        return LBM_E_CONTRACT;
    }
    float a[3] = {0.f, 0.f, 0.f};
    if (acceleration_lattice)
        for (int d = 0; d < 3; ++d) {
            if (!std::isfinite(acceleration_lattice[d])) {
                set_thread_error("lbm_state_stats_noalloc: acceleration_lattice requires three finite components");
                return LBM_E_CONTRACT;
            }
            a[d] = (float)acceleration_lattice[d];
        }
    void* scratch = nullptr;
    cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) {
        set_thread_error((std::string("lbm_state_stats_noalloc: scratch set-up failed: ") + cudaGetErrorString(e)).c_str());
        return LBM_E_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the ticket counter must start at zero (a call that stopped early could
    // have left it set)
    e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess) {
        int64_t blocks = (cells + NOALLOC_THREADS - 1) / NOALLOC_THREADS;
        const int grid = (int)std::min<int64_t>(blocks, NOALLOC_MAX_BLOCKS);
        unsigned char* sp = static_cast<unsigned char*>(scratch);
        if (q == 19)
            k_state_stats<19><<<grid, NOALLOC_THREADS, 0, s>>>(populations, (uint32_t)cells, solid, alpha, a[0], a[1],
                                                              a[2], sp, out4);
        else
            k_state_stats<27><<<grid, NOALLOC_THREADS, 0, s>>>(populations, (uint32_t)cells, solid, alpha, a[0], a[1],
                                                              a[2], sp, out4);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_thread_error((std::string("lbm_state_stats_noalloc: ") + cudaGetErrorString(e)).c_str());
        return LBM_E_CUDA;
    }
    return LBM_OK;
}
