// sc_common.cu — errors, formatting, the ordered f64 chain and graph storage.
#include <cstdarg>
#include <mutex>

#include "sc_prims.cuh"

namespace sc {

void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
    Failure f{};
    f.info.code = (e == cudaErrorMemoryAllocation) ? SC_E_OUT_OF_MEMORY : SC_E_CUDA;
    std::snprintf(f.info.message, sizeof f.info.message, "CUDA error %s (%s) in %s at %s:%d",
                  cudaGetErrorName(e), cudaGetErrorString(e), what, file, line);
    throw f;
}

void fail(sc_status code, const char* fmt, ...) {
    Failure f{};
    f.info.code = code;
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(f.info.message, sizeof f.info.message, fmt, ap);
    va_end(ap);
    throw f;
}

// Display of f64 as Rust prints it: shortest text that round-trips, integers
// without a fractional part.
std::string fmt_f64(double x) {
    if (std::isnan(x)) return "NaN";
    if (std::isinf(x)) return x > 0 ? "inf" : "-inf";
    char buf[64];
    for (int prec = 1; prec <= 17; ++prec) {
        std::snprintf(buf, sizeof buf, "%.*g", prec, x);
        if (std::strtod(buf, nullptr) == x) break;
    }
    // expand exponent notation the way Rust's Display does (no exponent)
    if (std::strchr(buf, 'e')) {
        std::snprintf(buf, sizeof buf, "%.17f", x);
        std::string s(buf);
        while (!s.empty() && s.back() == '0') s.pop_back();
        if (!s.empty() && s.back() == '.') s.pop_back();
        return s;
    }
    return std::string(buf);
}

// Display text of ClusteringError (src/error.rs:70-112).
void fail_info(sc_error_info i) {
    Failure f{};
    f.info = i;
    char* m = f.info.message;
    size_t cap = sizeof f.info.message;
    switch (i.code) {
        case SC_E_NODE_INDEX_OUT_OF_RANGE:
            std::snprintf(m, cap, "node index %llu is out of range for a graph with %llu nodes",
                          (unsigned long long)i.node, (unsigned long long)i.n_nodes);
            break;
        case SC_E_NON_FINITE_WEIGHT:
            std::snprintf(m, cap, "edge (%llu, %llu) has a non-finite weight",
                          (unsigned long long)i.edge_from, (unsigned long long)i.edge_to);
            break;
        case SC_E_NEGATIVE_WEIGHT:
            std::snprintf(m, cap,
                          "edge (%llu, %llu) has negative weight %s; weights must be non-negative",
                          (unsigned long long)i.edge_from, (unsigned long long)i.edge_to,
                          fmt_f64(i.weight).c_str());
            break;
        case SC_E_INVALID_NODE_WEIGHT:
            std::snprintf(m, cap, "node %llu has invalid weight %s; must be finite and non-negative",
                          (unsigned long long)i.node, fmt_f64(i.weight).c_str());
            break;
        case SC_E_NODE_WEIGHT_LENGTH_MISMATCH:
            std::snprintf(m, cap, "node weight vector has length %llu, expected %llu",
                          (unsigned long long)i.got, (unsigned long long)i.expected_len);
            break;
        case SC_E_MEMBERSHIP_LENGTH_MISMATCH:
            std::snprintf(m, cap, "membership vector has length %llu, expected %llu",
                          (unsigned long long)i.got, (unsigned long long)i.expected_len);
            break;
        case SC_E_TOO_MANY_NODES:
            std::snprintf(m, cap,
                          "graph has %llu nodes, exceeding the %llu addressable by u32 adjacency",
                          (unsigned long long)i.n_nodes, (unsigned long long)MAX_NODES);
            break;
        case SC_E_ASYMMETRIC_GRAPH:
            std::snprintf(m, cap,
                          "adjacency is not symmetric: \xCE\xA3 strength = %s, expected 2 \xC2\xB7 "
                          "total_weight = %s. A k-NN graph must be symmetrised before use.",
                          fmt_f64(i.degree_sum).c_str(), fmt_f64(i.expected).c_str());
            break;
        default:
            break;  // InvalidConfig / InvalidCsr carry their own text
    }
    throw f;
}

cudaMemPool_t user_graph_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) fail(SC_E_INVALID_ARGUMENT, "device %d out of range", device);
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        SC_CUDA(cudaMemPoolCreate(&pool, &props));
        uint64_t keep = UINT64_MAX;  // freed graph memory stays for the next graph
        SC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        pools[device] = pool;
    }
    return pools[device];
}

void check_device_status(Ctx& c) {
    Mailbox mb(c);
    const uint32_t* h = mb.get(c.d_status, 1);
    mb.wait();
    raise_device_status(c, *h);
}

void raise_device_status(Ctx& c, uint32_t st) {
    if (st == DEV_OK) return;
    SC_CUDA(cudaMemsetAsync(c.d_status, 0, sizeof(uint32_t), c.stream));
    if (st & DEV_TIMEOUT) fail(SC_E_TIMEOUT, "a bounded device wait gave up (status 0x%x)", st);
    fail(SC_E_INTERNAL, "a device-side check failed (status 0x%x)", st);
}

__global__ void k_ordered_sum(const double* __restrict__ terms, uint64_t n, double init,
                              double* out) {
    const unsigned lane = threadIdx.x & 31u;
    double s = init;
    for (uint64_t base = 0; base < n; base += 32) {
        uint64_t i = base + lane;
        double t = i < n ? terms[i] : 0.0;
        unsigned cnt = (unsigned)((n - base) < 32 ? (n - base) : 32);
        for (unsigned j = 0; j < cnt; ++j) {
            double x = __shfl_sync(0xFFFFFFFFu, t, (int)j);
            s = __dadd_rn(s, x);
        }
    }
    if (lane == 0) *out = s;
}

double ordered_sum(Ctx& c, const double* d_terms, uint64_t n) { return ordered_sum_from(c, d_terms, n, -0.0); }

double ordered_sum_from(Ctx& c, const double* d_terms, uint64_t n, double init) {
    DBuf<double> out(c, 1);
    k_ordered_sum<<<1, 32, 0, c.stream>>>(d_terms, n, init, out.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    return to_host(c, out.get());
}

void DevGraph::free_all() {
    void* ps[] = {ptr, nbr, w, erow, node_w, strength, self_loop, emb, edge_sf, edge_i, edge_j, edge_e};
    if (ptr || nbr || w || erow || node_w || strength || self_loop || emb || edge_sf || edge_i || edge_j || edge_e) {
        int prev = 0;
        cudaGetDevice(&prev);
        if (prev != device) cudaSetDevice(device);
        // Pool memory goes back to its pool only through cudaFreeAsync (a plain
        // cudaFree leaves it counted as in use). A graph handed to the user may
        // still be read by work queued on any context's stream: wait for the
        // device, free on the legacy stream and wait for that, so the call stays
        // synchronous for the caller.
        if (!stream) cudaDeviceSynchronize();
        for (void* p : ps)
            if (p) cudaFreeAsync(p, stream ? stream : (cudaStream_t)0);
        if (!stream) cudaStreamSynchronize((cudaStream_t)0);
        if (prev != device) cudaSetDevice(prev);
    }
    ptr = nullptr;
    nbr = nullptr;
    w = nullptr;
    erow = nullptr;
    node_w = nullptr;
    strength = nullptr;
    self_loop = nullptr;
    emb = nullptr;
    edge_sf = nullptr;
    edge_i = nullptr;
    edge_j = nullptr;
    edge_e = nullptr;
    edge_m = 0;
    edge_ready = false;
}

}  // namespace sc
