// sc_internal.cuh — shared definitions of the sm_100a Leiden / kNN library.
//
// The whole library is compiled with -fmad=false: Rust never contracts a*b+c
// into an FMA, and the parity functions (finish, aggregate, partition
// aggregates, quality, modularity) must reproduce its f64 results bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <memory>
#include <mutex>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/sc_gpu.h"

namespace sc {

constexpr uint32_t UNASSIGNED = 0xFFFFFFFFu;
constexpr uint32_t NONE32 = 0xFFFFFFFFu;
constexpr uint64_t MAX_NODES = 0xFFFFFFFFull;  // csr_network.rs:36

// Device status word bits (written by guarded kernels, read by the host).
enum DevStatus : uint32_t {
    DEV_OK = 0,
    DEV_BOUNDS = 1u << 0,    // an index check failed; the access was skipped
    DEV_TIMEOUT = 1u << 1,   // a bounded wait gave up
    DEV_OVERFLOW = 1u << 2,  // a capacity was exceeded
};

// ------------------------------------------------------------------ errors
struct Error {
    sc_status code = SC_OK;
    sc_error_info info{};
};

// Thrown inside the library, caught at the C ABI boundary. `info.code` is the
// status and `info.message` the Display text of the matching ClusteringError.
struct Failure {
    sc_error_info info;
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);
[[noreturn]] void fail(sc_status code, const char* fmt, ...);
[[noreturn]] void fail_info(sc_error_info info);  // formats info.message from the payload

#define SC_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) ::sc::throw_cuda(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define SC_LAUNCH_CHECK() SC_CUDA(cudaGetLastError())

// ------------------------------------------------------------------ context
constexpr uint32_t HUB_DEGREE = 1024;  // degree above which a node's hash lives in global memory
constexpr uint32_t DEFAULT_WAIT_LIMIT = 1u << 26;  // try_wait iterations of a bounded mbarrier wait

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;      // the device's default pool (stream-ordered temporaries)
    uint32_t* d_status = nullptr;      // device status word
    unsigned long long* d_refine_ctr = nullptr;  // refinement counters summed over a run (3 words)
    Error last;
    sc_run_stats stats{};
    uint64_t launches = 0;             // kernels launched by the current call
    int sm_count = 148;
    size_t smem_optin = 0;
    sc_tuning tuning{8, 16, 32, 4096};  // decide-kernel routing (sc_set_tuning / sc_autotune)
    // iterations a pipeline wait of the kNN kernel tries before it gives up
    // (sc_set_wait_limit); the waits that drain copies already issued keep the
    // library's default, so nothing can land in shared memory after a CTA exits
    uint32_t wait_limit = DEFAULT_WAIT_LIMIT;
    // test hook (sc_test_knn_hold_tiles): the kNN producer issues no point
    // tiles, so the contraction's first wait runs out and the call times out
    uint32_t knn_hold_tiles = 0;
    // kNN point clusters of the pruned search (sc_set_knn_clusters): 0 picks
    // a count from n, 1 scans every tile
    uint32_t knn_clusters = 0;
    sc_knn_stats knn_stats{};  // the last kNN search on this context
    // side streams for kernels of one step that may run concurrently (fork / join by events)
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[3] = {nullptr, nullptr, nullptr};
    // auxiliary stream for work that overlaps the next step (local moving's re-queue)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_aux_start = nullptr, ev_aux_done = nullptr;
    // pinned host buffer for the small device->host reads that steer the host loop
    // (bucket counts, counters, sizes): copies into it are truly asynchronous, so
    // several can be queued and completed by one stream synchronisation
    uint8_t* mailbox = nullptr;
    // pinned staging lanes of large host -> device uploads (created on first use)
    struct Staging* staging = nullptr;
};
constexpr int SIDE_STREAMS = 3;
constexpr size_t MAILBOX_BYTES = 4096;
constexpr int STAGE_LANES = 4;                     // host threads of a staged upload
constexpr size_t STAGE_CHUNK = size_t(4) << 20;     // bytes per pinned buffer (two per lane)
constexpr size_t STAGE_MIN_BYTES = size_t(16) << 20;  // smaller uploads use one plain copy

// Host -> device copy of `bytes` from pageable `src`, ordered on the context's
// stream (large copies go through the pinned staging lanes); src may be reused
// when it returns.
void upload(Ctx& c, void* dst, const void* src, size_t bytes);
void release_staging(Ctx& c);
// The device's pool of user-graph arrays (created on first use, kept until exit).
cudaMemPool_t user_graph_pool(int device);
// u32 device labels -> u64 host labels (widened on the device, one copy)
void download_labels(Ctx& c, const uint32_t* d_labels, uint64_t n, uint64_t* host_out);

// Stream-ordered device buffer of T, from the context's pool on its stream.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(Ctx& c, size_t count) { alloc(c, count); }
    void alloc(Ctx& c, size_t count) {
        release();
        s = c.stream;
        n = count;
        if (count) {
            cudaError_t e = cudaMallocFromPoolAsync((void**)&p, count * sizeof(T), c.pool, s);
            if (e == cudaErrorMemoryAllocation) {
                cudaGetLastError();
                fail(SC_E_OUT_OF_MEMORY, "device allocation of %zu bytes failed", count * sizeof(T));
            }
            if (e != cudaSuccess) throw_cuda(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
        }
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        n = 0;
    }
    ~DBuf() { release(); }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    DBuf(DBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            n = o.n;
            s = o.s;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    T* get() const { return p; }
    size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------------ graph
// Device-resident CSRNetworkData (csr_network.rs:38-60) plus cached per-node
// self-loop weights and the row id of every stored entry.
struct DevGraph {
    int device = 0;
    uint64_t n = 0;           // node_count
    uint64_t E = 0;           // stored entries
    uint64_t* ptr = nullptr;  // n+1
    uint32_t* nbr = nullptr;  // E, strictly increasing per row
    float* w = nullptr;       // E
    uint32_t* erow = nullptr; // E, row of each entry
    double* node_w = nullptr; // n
    double* strength = nullptr;   // n
    double* self_loop = nullptr;  // n (0.0 where there is none)
    double total_weight = 0.0;
    uint64_t edge_count = 0;
    bool any_self_loops = false;
    uint32_t max_degree = 0;
    // exact-summation regime (every subset sum of edge weights is exact in f64)
    int e0_w = 0;             // exponent of the lowest set bit over stored weights
    bool exact_w = true;
    int e0_nw = 0;            // same over node weights
    bool exact_nw = true;
    double total_node_weight = 0.0;  // Σ node_w, Rust `sum()` order
    // A disjoint union of instances (batched runs) sums nothing across
    // instances, so its summation regime is that of its heaviest instance:
    // the largest instance total of Σ strength and of Σ node weight (0: not a
    // union, the graph's own totals decide).
    double part_max_2m = 0.0;
    double part_max_nw = 0.0;
    // The kNN embedding projected to EMB_R components per node (n x EMB_R,
    // from the graph pool), read by the learned warm start's features; null
    // when none was attached.
    float* emb = nullptr;
    // The learned warm start's structural edge features (those that depend on
    // neither the resolution nor a context partition), computed on first use
    // and kept until the graph is freed or its embedding replaced, all from
    // the graph pool: per undirected edge i < j in ascending order, its
    // EDGE_SF features, endpoints and stored entries (i, j), (j, i).
    mutable std::mutex edge_mu;
    mutable float* edge_sf = nullptr;
    mutable uint32_t* edge_i = nullptr;
    mutable uint32_t* edge_j = nullptr;
    mutable uint64_t* edge_e = nullptr;  // 2 per edge
    mutable uint64_t edge_m = 0;
    mutable bool edge_ready = false;
    uint64_t n_hubs = 0;      // nodes whose degree exceeds the shared-memory hash
    // stored weights bitwise symmetric: 0 not yet known, 1 yes, 2 no (computed
    // once, on first need; a benign race between contexts computes it twice)
    mutable std::atomic<int> sym_state{0};
    // Arrays of graphs built from user input come from a pool of their own,
    // one per device (pooled == false): in the default pool a graph held across
    // runs would take blocks that a run's large temporaries reuse from one run
    // to the next, and a pool that has to grow in the middle of a run stalls
    // it; cudaMalloc / cudaFree instead cost up to 0.1 s per graph. The graphs a
    // run builds (coarse levels, aggregates) come from the default pool. A graph
    // owned by a running call returns its arrays on that call's stream, one
    // handed to the user (stream == nullptr) once the device is idle.
    bool pooled = true;
    cudaStream_t stream = nullptr;
    void free_all();
    ~DevGraph() { free_all(); }
};

constexpr int EMB_R = 16;  // components of a graph's projected embedding

// Attaches the projection of the n x d row-major host embedding X to g
// (replacing any earlier one).
void graph_set_embedding(Ctx& c, DevGraph& g, const float* X, uint64_t d);

// ------------------------------------------------------------------ helpers
inline unsigned grid_for(uint64_t work, unsigned block, unsigned cap = 148u * 16u) {
    uint64_t g = (work + block - 1) / block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

__host__ __device__ inline uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__host__ __device__ inline uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
    return splitmix(splitmix(splitmix(seed) ^ a) ^ b);
}

// Exponent of the lowest set bit of a finite non-zero value (INT32_MAX for 0).
__host__ __device__ inline int lowbit_exp_f32(float x) {
    uint32_t b;
    memcpy(&b, &x, 4);
    b &= 0x7FFFFFFFu;
    if (b == 0) return 0x7FFFFFFF;
    int e = (int)(b >> 23);
    uint32_t m = b & 0x7FFFFFu;
#ifdef __CUDA_ARCH__
    if (e == 0) return -149 + (__ffs((int)m) - 1);
    m |= 0x800000u;
    return (e - 150) + (__ffs((int)m) - 1);
#else
    if (e == 0) return -149 + __builtin_ctz(m);
    m |= 0x800000u;
    return (e - 150) + __builtin_ctz(m);
#endif
}
__host__ __device__ inline int lowbit_exp_f64(double x) {
    uint64_t b;
    memcpy(&b, &x, 8);
    b &= 0x7FFFFFFFFFFFFFFFull;
    if (b == 0) return 0x7FFFFFFF;
    int e = (int)(b >> 52);
    uint64_t m = b & 0xFFFFFFFFFFFFFull;
#ifdef __CUDA_ARCH__
    if (e == 0) return -1074 + (__ffsll((long long)m) - 1);
    m |= 0x10000000000000ull;
    return (e - 1075) + (__ffsll((long long)m) - 1);
#else
    if (e == 0) return -1074 + __builtin_ctzll(m);
    m |= 0x10000000000000ull;
    return (e - 1075) + __builtin_ctzll(m);
#endif
}

// ------------------------------------------------------------------ API of the .cu files
// graph.cu
DevGraph* graph_from_csr(Ctx& c, const uint64_t* ptr, uint64_t n_ptr, const uint32_t* nbr,
                         uint64_t n_nbr, const float* w, uint64_t n_w, const double* node_w,
                         uint64_t n_node_w, bool device_inputs);
DevGraph* graph_from_edges(Ctx& c, uint64_t n, const uint64_t* from, const uint64_t* to,
                           const double* w, uint64_t m, const double* node_w);
DevGraph* graph_aggregate(Ctx& c, const DevGraph& g, const uint32_t* d_grp, uint32_t n_groups);
// disjoint union of `count` graphs, instance i's node ids shifted past instance i-1's
DevGraph* graph_union(Ctx& c, const DevGraph* const* gs, uint64_t count);
void graph_validate_symmetry(Ctx& c, const DevGraph& g);
bool graph_bitwise_symmetric(Ctx& c, const DevGraph& g);
void graph_copy_csr(Ctx& c, const DevGraph& g, uint64_t* ptr, uint32_t* nbr, float* w);
void graph_copy_node_data(Ctx& c, const DevGraph& g, double* node_w, double* strength);

// partition.cu
// Normalises arbitrary u64 labels (host) to ascending-rank ids on the device.
uint32_t renumber_u64_labels(Ctx& c, const uint64_t* d_labels, uint64_t n, uint32_t* d_out,
                             uint64_t* max_label_out);
// ascending-rank renumber of u32 ids < id_space; returns the number of distinct ids.
uint32_t renumber_ids(Ctx& c, const uint32_t* d_ids, uint64_t n, uint64_t id_space, uint32_t* d_out);
struct PartStats {
    uint64_t slots = 0;
    DBuf<uint32_t> size;
    DBuf<double> weight, strength, internal;
};
void partition_stats(Ctx& c, const DevGraph& g, const uint32_t* d_memb, uint64_t slots,
                     PartStats& out, bool need_internal);
// Σ terms in index order, as Rust's `Iterator::sum` (fold from -0.0).
double ordered_sum(Ctx& c, const double* d_terms, uint64_t n);
// ((init + t0) + t1) + ... in index order.
double ordered_sum_from(Ctx& c, const double* d_terms, uint64_t n, double init);
double quality(Ctx& c, const DevGraph& g, const uint32_t* d_memb, uint64_t slots, int objective,
               double gamma);
double modularity(Ctx& c, const DevGraph& g, const uint32_t* d_labels, uint64_t n_comms,
                  double gamma);

// static.cu: modularity from compact device labels, no device allocation
double modularity_static(Ctx& c, const DevGraph& g, const uint32_t* d_labels, uint64_t n, double gamma);

// leiden.cu
struct LeidenOut {
    std::vector<uint32_t> labels;
    uint64_t n_clusters = 0;
};
void leiden(Ctx& c, const DevGraph& g, const sc_leiden_config& cfg, const uint64_t* initial_host,
            uint32_t* d_labels_out, uint64_t* n_clusters);
// Every instance's leiden() over the disjoint union g of their graphs (instance
// I owns n[I] nodes, in order), instance I from initial[I] (host labels, nullable).
void leiden_union(Ctx& c, const DevGraph& g, uint32_t count, const uint64_t* n, const sc_leiden_config* cfgs,
                  const uint64_t* const* initial, uint32_t* d_labels_out, uint64_t* n_clusters);
bool tuning_valid(const sc_tuning& t);
// Times the first level under candidate routings, keeps the fastest on c.
uint32_t autotune(Ctx& c, const DevGraph& g, const sc_leiden_config& cfg, sc_tuning* chosen, double* ms_chosen,
                  double* ms_default);

// knn.cu
void knn_gaussian(Ctx& c, const float* X, uint64_t n, uint64_t d, uint64_t k,
                  const sc_knn_opts& opts, uint32_t* knn_index, float* knn_dist,
                  uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w, uint64_t conn_cap,
                  uint64_t* conn_nnz, DevGraph** graph_out);
void knn_search(Ctx& c, const float* X, uint64_t n, uint64_t d, uint64_t k, uint64_t q0, uint64_t q1,
                const sc_knn_opts& opts, uint32_t* knn_index, float* knn_d2);
uint32_t knn_autotune(Ctx& c, const float* X, uint64_t n, uint64_t d, uint64_t k, const sc_knn_opts& opts,
                      uint32_t* chosen, double* ms_chosen, double* ms_full);
void knn_connectivities(Ctx& c, const uint32_t* knn_index, const float* knn_d2, uint64_t n, uint64_t k,
                        const sc_knn_opts& opts, uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                        uint64_t conn_cap, uint64_t* conn_nnz, DevGraph** graph_out);

// mlp.cu: learned warm start (edge MLP; proposal = components of confident edges)
struct Mlp;
Mlp* mlp_create(Ctx& c, uint64_t seed);
void mlp_destroy(Mlp* m);
uint32_t mlp_param_count();
uint32_t mlp_feature_count();
bool mlp_get(Ctx& c, const Mlp& m, float* params, float* scaler);  // returns whether a scaler is set
void mlp_set(Ctx& c, Mlp& m, const float* params, const float* scaler);
// coarse / fine: compact device labels of the partitions at the neighbouring
// lower / higher resolutions (nullable)
void mlp_features(Ctx& c, Mlp& m, const DevGraph& g, double gamma, const uint32_t* coarse, const uint32_t* fine,
                  float* feat_host, uint32_t* ei_host, uint32_t* ej_host, uint64_t cap, uint64_t* M_out);
double mlp_train(Ctx& c, Mlp& m, const DevGraph& g, const uint32_t* d_memb, double gamma, const uint32_t* coarse,
                 const uint32_t* fine, uint32_t epochs, double lr, float* grad_out_host);
uint64_t mlp_propose(Ctx& c, Mlp& m, const DevGraph& g, double gamma, const uint32_t* coarse, const uint32_t* fine,
                     double thr, double core_fraction, uint32_t* d_labels, float* prob_host, uint64_t prob_cap);

// common.cu
void check_device_status(Ctx& c);
// the failure for a status word already read back (none for DEV_OK); clears it
void raise_device_status(Ctx& c, uint32_t st);
// Rust-style shortest round-trip text of an f64 (Display of f64).
std::string fmt_f64(double x);

}  // namespace sc
