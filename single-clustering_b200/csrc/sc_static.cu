// sc_static.cu — modularity for callers that cannot allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: a host framework that
// already owns all device memory through its own pool, a code path with a hard
// device-memory budget, or a section where an allocation's implicit
// synchronisation is not allowed. sc_modularity_static computes the same value
// as sc_modularity using only memory the caller passes in (the graph handle
// and a device array of labels) plus the fixed scratch array below, which every
// GPU that loads this library holds until the process exits.
//
// The scratch is shared by every call on a device and keeps the previous call's
// contents; each call clears what it accumulates into before use. Calls whose
// work overlaps on the GPU (two streams, two host threads) race on it: the
// caller must serialise them.
#include <mutex>

#include "sc_prims.cuh"

namespace sc {

namespace {

constexpr uint32_t STATIC_MAX_COMMUNITIES = 1u << 16;  // 65,536 communities
constexpr uint32_t STATIC_TAIL = 8;                     // result and flags
// [0, MAX): Σ strength per community, [MAX, 2 MAX): internal weight per
// community, then STATIC_TAIL control words. 1 MiB + 64 B per device.
__device__ __align__(256) double g_static_scratch[2 * STATIC_MAX_COMMUNITIES + STATIC_TAIL];

constexpr int MAX_DEVICES = 64;
// Per device: the address of g_static_scratch and the CUDA context it was looked
// up in. A context that is destroyed and re-created (cudaDeviceReset, or the
// primary context released and retained again) maps the array afresh, so the
// address is looked up again whenever the current context is not the cached one.
struct ScratchAddr {
    void* ctx = nullptr;
    double* addr = nullptr;
};
ScratchAddr g_scratch_addr[MAX_DEVICES];
std::mutex g_scratch_mu;

using CtxGetCurrentFn = int (*)(void**);  // cuCtxGetCurrent(CUcontext*)

void* current_context() {
    static CtxGetCurrentFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return (CtxGetCurrentFn)p;
    }();
    void* ctx = nullptr;
    if (!fn || fn(&ctx) != 0) fail(SC_E_CUDA, "cuCtxGetCurrent is unavailable");
    return ctx;
}

// Host code must not use g_static_scratch's name as a device address: look the
// address up with the device current, once per device and context.
double* scratch_for(int device) {
    if (device < 0 || device >= MAX_DEVICES) fail(SC_E_INVALID_ARGUMENT, "device %d out of range", device);
    void* ctx = current_context();
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    ScratchAddr& a = g_scratch_addr[device];
    if (!a.addr || a.ctx != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) throw_cuda(e, "cudaGetSymbolAddress(g_static_scratch)", __FILE__, __LINE__);
        a.addr = (double*)p;
        a.ctx = ctx;
    }
    return a.addr;
}

__global__ void k_static_clear(double* scratch) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * STATIC_MAX_COMMUNITIES + STATIC_TAIL;
         i += gridDim.x * blockDim.x)
        scratch[i] = 0.0;
}

// Per node: Σ strength of its community and the largest label; labels past the
// limit raise a flag instead of being accumulated.
__global__ void k_static_nodes(const uint32_t* __restrict__ labels, uint64_t n, const double* __restrict__ strength,
                               double* scratch) {
    unsigned long long* ctrl = (unsigned long long*)(scratch + 2 * STATIC_MAX_COMMUNITIES);
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = labels[v];
        if (c >= STATIC_MAX_COMMUNITIES) {
            atomicOr(ctrl + 1, 1ull);
            continue;
        }
        atomicMax(ctrl + 0, (unsigned long long)c + 1);
        atomicAdd(scratch + c, strength[v]);
    }
}

// Per stored entry with row <= neighbour inside one community: its weight.
__global__ void k_static_internal(const uint32_t* __restrict__ erow, const uint32_t* __restrict__ nbr,
                                  const float* __restrict__ w, uint64_t E, const uint32_t* __restrict__ labels,
                                  double* scratch) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = erow[e], u = nbr[e];
        if (v > u) continue;
        const uint32_t c = labels[v];
        if (c < STATIC_MAX_COMMUNITIES && labels[u] == c)
            atomicAdd(scratch + STATIC_MAX_COMMUNITIES + c, (double)w[e]);
    }
}

// Σ_c [2 internal_c / 2m - gamma (K_c / 2m)^2] over c < max label + 1, in
// community order from -0.0 (objective.rs:240-243), by one warp.
__global__ void k_static_sum(double* scratch, double gamma, double two_m) {
    const unsigned long long* ctrl = (const unsigned long long*)(scratch + 2 * STATIC_MAX_COMMUNITIES);
    const uint64_t C = ctrl[0];
    const double q = warp_ordered_sum(0, C, -0.0, [&](uint64_t c) {
        const double s = __ddiv_rn(scratch[c], two_m);
        return __dsub_rn(__ddiv_rn(__dmul_rn(2.0, scratch[STATIC_MAX_COMMUNITIES + c]), two_m),
                         __dmul_rn(gamma, __dmul_rn(s, s)));
    });
    if (threadIdx.x == 0) scratch[2 * STATIC_MAX_COMMUNITIES + 2] = q;
}

}  // namespace

// modularity with compact device labels and no device allocation. In the exact
// regime (every sum of edge weights exact in f64, see sc_graph.cu) the result
// is the reference's value bit for bit; outside it the per-community sums are
// taken in atomic order and may differ from sc_modularity in the last bits.
double modularity_static(Ctx& c, const DevGraph& g, const uint32_t* d_labels, uint64_t n, double gamma) {
    const double m = g.total_weight;
    if (m == 0.0) return 0.0;  // objective.rs:222-225
    double* scratch = scratch_for(c.device);
    k_static_clear<<<64, 256, 0, c.stream>>>(scratch);
    if (n) k_static_nodes<<<grid_for(n, 256), 256, 0, c.stream>>>(d_labels, n, g.strength, scratch);
    if (g.E) k_static_internal<<<grid_for(g.E, 256), 256, 0, c.stream>>>(g.erow, g.nbr, g.w, g.E, d_labels, scratch);
    k_static_sum<<<1, 32, 0, c.stream>>>(scratch, gamma, 2.0 * m);
    SC_LAUNCH_CHECK();
    c.launches += 4;
    double tail[3];
    SC_CUDA(cudaMemcpyAsync(tail, scratch + 2 * STATIC_MAX_COMMUNITIES, sizeof tail, cudaMemcpyDeviceToHost,
                            c.stream));
    SC_CUDA(cudaStreamSynchronize(c.stream));
    unsigned long long over;
    std::memcpy(&over, &tail[1], sizeof over);
    if (over)
        fail(SC_E_UNSUPPORTED,
             "sc_modularity_static supports labels below %u (at most %u communities); use sc_modularity",
             STATIC_MAX_COMMUNITIES, STATIC_MAX_COMMUNITIES);
    return tail[2];
}

}  // namespace sc
