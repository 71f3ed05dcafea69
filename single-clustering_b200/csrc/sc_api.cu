// sc_api.cu — the extern "C" boundary (include/sc_gpu.h). Every entry point
// catches library failures and turns them into an sc_status plus the context's
// last-error record; nothing escapes as a C++ exception or an abort.
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <random>
#include <thread>
#include <chrono>

#include "sc_prims.cuh"

struct sc_ctx {
    sc::Ctx c;
};
struct sc_graph {
    sc::DevGraph* g = nullptr;
};
struct sc_mlp {
    sc::Mlp* m = nullptr;
    int device = 0;
};

namespace {

sc_status fill_error(sc_ctx* ctx, const sc_error_info& info) {
    if (ctx) {
        ctx->c.last.code = (sc_status)info.code;
        ctx->c.last.info = info;
    }
    return (sc_status)info.code;
}

template <class F>
sc_status guarded(sc_ctx* ctx, F&& f) {
    if (!ctx) return SC_E_INVALID_ARGUMENT;
    ctx->c.last = sc::Error{};
    ctx->c.launches = 0;
    try {
        SC_CUDA(cudaSetDevice(ctx->c.device));
        f(ctx->c);
        return SC_OK;
    } catch (sc::Failure& fl) {
        return fill_error(ctx, fl.info);
    } catch (std::bad_alloc&) {
        sc_error_info i{};
        i.code = SC_E_OUT_OF_MEMORY;
        std::snprintf(i.message, sizeof i.message, "host allocation failed");
        return fill_error(ctx, i);
    } catch (...) {
        sc_error_info i{};
        i.code = SC_E_INTERNAL;
        std::snprintf(i.message, sizeof i.message, "unexpected internal exception");
        return fill_error(ctx, i);
    }
}

[[noreturn]] void bad_arg(const char* what) { sc::fail(SC_E_INVALID_ARGUMENT, "invalid argument: %s", what); }

void require(bool ok, const char* what) {
    if (!ok) bad_arg(what);
}

void check_membership_len(uint64_t got, uint64_t expected) {
    if (got != expected) {
        sc_error_info i{};
        i.code = SC_E_MEMBERSHIP_LENGTH_MISMATCH;
        i.got = got;
        i.expected_len = expected;
        sc::fail_info(i);
    }
}

void require_same_device(sc::Ctx& c, const sc::DevGraph& g) {
    if (c.device != g.device) bad_arg("graph lives on another device than the context");
}

// Stream, pool and status word of a context on `device` (SC_OK or the failure).
// side_streams: the decide kernels of one batch may fork onto 3 extra streams;
// a batch with more than 8 workers gives its workers none (the instances
// already fill the GPU; measured on a 128-instance sweep).
sc_status init_ctx(sc::Ctx& c, int device, bool side_streams = true) {
    c.device = device;
    if (cudaSetDevice(device) != cudaSuccess) return SC_E_CUDA;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) return SC_E_CUDA;
    if (cudaDeviceGetDefaultMemPool(&c.pool, device) != cudaSuccess) return SC_E_CUDA;
    uint64_t thresh = UINT64_MAX;  // keep freed blocks cached in the pool
    cudaMemPoolSetAttribute(c.pool, cudaMemPoolAttrReleaseThreshold, &thresh);
    for (int t = 0; side_streams && t < sc::SIDE_STREAMS; ++t) {
        if (cudaStreamCreateWithFlags(&c.side[t], cudaStreamNonBlocking) != cudaSuccess) return SC_E_CUDA;
        if (cudaEventCreateWithFlags(&c.ev_join[t], cudaEventDisableTiming) != cudaSuccess) return SC_E_CUDA;
    }
    if (side_streams && cudaEventCreateWithFlags(&c.ev_fork, cudaEventDisableTiming) != cudaSuccess)
        return SC_E_CUDA;
    if (side_streams) {
        if (cudaStreamCreateWithFlags(&c.aux, cudaStreamNonBlocking) != cudaSuccess) return SC_E_CUDA;
        if (cudaEventCreateWithFlags(&c.ev_aux_start, cudaEventDisableTiming) != cudaSuccess) return SC_E_CUDA;
        if (cudaEventCreateWithFlags(&c.ev_aux_done, cudaEventDisableTiming) != cudaSuccess) return SC_E_CUDA;
    }
    if (cudaHostAlloc((void**)&c.mailbox, sc::MAILBOX_BYTES, cudaHostAllocDefault) != cudaSuccess) {
        c.mailbox = nullptr;
        return SC_E_CUDA;
    }
    if (cudaMalloc(&c.d_status, sizeof(uint32_t)) != cudaSuccess) return SC_E_OUT_OF_MEMORY;
    cudaMemset(c.d_status, 0, sizeof(uint32_t));
    if (cudaMalloc(&c.d_refine_ctr, 4 * sizeof(unsigned long long)) != cudaSuccess) return SC_E_OUT_OF_MEMORY;
    cudaMemset(c.d_refine_ctr, 0, 4 * sizeof(unsigned long long));
    cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device);
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    c.smem_optin = (size_t)optin;
    return SC_OK;
}

void release_ctx(sc::Ctx& c) {
    cudaSetDevice(c.device);
    if (c.stream) {
        cudaStreamSynchronize(c.stream);
        cudaStreamDestroy(c.stream);
        c.stream = nullptr;
    }
    for (int t = 0; t < sc::SIDE_STREAMS; ++t) {
        if (c.side[t]) {
            cudaStreamSynchronize(c.side[t]);
            cudaStreamDestroy(c.side[t]);
        }
        if (c.ev_join[t]) cudaEventDestroy(c.ev_join[t]);
        c.side[t] = nullptr;
        c.ev_join[t] = nullptr;
    }
    if (c.ev_fork) cudaEventDestroy(c.ev_fork);
    c.ev_fork = nullptr;
    if (c.aux) {
        cudaStreamSynchronize(c.aux);
        cudaStreamDestroy(c.aux);
    }
    if (c.ev_aux_start) cudaEventDestroy(c.ev_aux_start);
    if (c.ev_aux_done) cudaEventDestroy(c.ev_aux_done);
    c.aux = nullptr;
    c.ev_aux_start = c.ev_aux_done = nullptr;
    sc::release_staging(c);
    if (c.mailbox) cudaFreeHost(c.mailbox);
    c.mailbox = nullptr;
    if (c.d_status) cudaFree(c.d_status);
    c.d_status = nullptr;
    if (c.d_refine_ctr) cudaFree(c.d_refine_ctr);
    c.d_refine_ctr = nullptr;
    c.pool = nullptr;  // the device's default pool: not ours to destroy
}

// Runs instance i of a batch on worker context w (labels copied to the host).
void run_instance(sc::Ctx& w, const sc::DevGraph& G, const sc_leiden_config& cfg, const uint64_t* initial,
                  uint64_t* labels_out, uint64_t* n_clusters) {
    sc::DBuf<uint32_t> lab(w, G.n);
    uint64_t ncl = 0;
    sc::leiden(w, G, cfg, initial, lab.get(), &ncl);
    sc::download_labels(w, lab.get(), G.n, labels_out);
    *n_clusters = ncl;
}

}  // namespace

extern "C" {

uint32_t sc_abi_version(void) { return SC_GPU_ABI_VERSION; }

sc_status sc_ctx_create(int32_t device, sc_ctx** out) {
    if (!out) return SC_E_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return SC_E_CUDA;
    }
    if (device < 0 || device >= count) return SC_E_INVALID_ARGUMENT;
    std::unique_ptr<sc_ctx> ctx(new sc_ctx());
    sc_status st = init_ctx(ctx->c, device);
    if (st != SC_OK) {
        release_ctx(ctx->c);
        return st;
    }
    *out = ctx.release();
    return SC_OK;
}

void sc_ctx_destroy(sc_ctx* ctx) {
    if (!ctx) return;
    release_ctx(ctx->c);
    delete ctx;
}

const char* sc_last_error_message(const sc_ctx* ctx) {
    if (!ctx) return "null context";
    return ctx->c.last.info.message;
}

sc_status sc_last_error_info(const sc_ctx* ctx, sc_error_info* out) {
    if (!ctx || !out) return SC_E_INVALID_ARGUMENT;
    *out = ctx->c.last.info;
    return SC_OK;
}

sc_status sc_last_run_stats(const sc_ctx* ctx, sc_run_stats* out) {
    if (!ctx || !out) return SC_E_INVALID_ARGUMENT;
    *out = ctx->c.stats;
    return SC_OK;
}

void sc_tuning_default(sc_tuning* t) {
    if (t) *t = sc_tuning{8, 16, 32, 4096};
}

sc_status sc_get_tuning(const sc_ctx* ctx, sc_tuning* out) {
    if (!ctx || !out) return SC_E_INVALID_ARGUMENT;
    *out = ctx->c.tuning;
    return SC_OK;
}

sc_status sc_set_tuning(sc_ctx* ctx, const sc_tuning* t) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(t != nullptr, "tuning is NULL");
        if (!sc::tuning_valid(*t))
            sc::fail(SC_E_INVALID_ARGUMENT, "tuning limits must satisfy lanes8 <= 8, lanes8 <= lanes16 <= 16, "
                                            "lanes16 <= lanes32 <= 32");
        c.tuning = *t;
    });
}

sc_status sc_set_wait_limit(sc_ctx* ctx, uint32_t limit) {
    return guarded(ctx, [&](sc::Ctx& c) {
        if (limit == 0) sc::fail(SC_E_INVALID_ARGUMENT, "the wait limit must be at least 1");
        c.wait_limit = limit;
    });
}

sc_status sc_get_wait_limit(const sc_ctx* ctx, uint32_t* out) {
    if (!ctx || !out) return SC_E_INVALID_ARGUMENT;
    *out = ctx->c.wait_limit;
    return SC_OK;
}

sc_status sc_set_knn_clusters(sc_ctx* ctx, uint32_t clusters) {
    return guarded(ctx, [&](sc::Ctx& c) {
        if (clusters > 256) sc::fail(SC_E_INVALID_ARGUMENT, "at most 256 kNN clusters, got %u", clusters);
        c.knn_clusters = clusters;
    });
}

sc_status sc_knn_autotune(sc_ctx* ctx, const float* X, uint64_t n, uint64_t d, uint64_t k, const sc_knn_opts* opts,
                          uint32_t* chosen_clusters, double* ms_chosen, double* ms_full, uint32_t* n_candidates) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(X != nullptr && opts != nullptr, "X or opts is NULL");
        const uint32_t nc = sc::knn_autotune(c, X, n, d, k, *opts, chosen_clusters, ms_chosen, ms_full);
        if (n_candidates) *n_candidates = nc;
    });
}

sc_status sc_knn_last_stats(const sc_ctx* ctx, sc_knn_stats* out) {
    if (!ctx || !out) return SC_E_INVALID_ARGUMENT;
    *out = ctx->c.knn_stats;
    return SC_OK;
}

sc_status sc_test_knn_hold_tiles(sc_ctx* ctx, int32_t on) {
    return guarded(ctx, [&](sc::Ctx& c) { c.knn_hold_tiles = on ? 1u : 0u; });
}

sc_status sc_autotune(sc_ctx* ctx, const sc_graph* g, const sc_leiden_config* cfg, sc_tuning* chosen,
                      double* ms_chosen, double* ms_default, uint32_t* n_candidates) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && cfg, "graph or config is NULL");
        require_same_device(c, *g->g);
        const uint32_t k = sc::autotune(c, *g->g, *cfg, chosen, ms_chosen, ms_default);
        if (n_candidates) *n_candidates = k;
    });
}

sc_status sc_ctx_synchronize(sc_ctx* ctx) {
    return guarded(ctx, [&](sc::Ctx& c) { SC_CUDA(cudaStreamSynchronize(c.stream)); });
}

void sc_leiden_config_default(sc_leiden_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->objective = SC_OBJECTIVE_RB;
    cfg->resolution = 1.0;
    cfg->has_seed = 1;
    cfg->seed = 42;
    cfg->n_iterations = 2;
    cfg->max_levels = 64;
    cfg->tolerance = 1e-9;
    cfg->refine = 1;
    cfg->refine_randomness = 0.01;
    cfg->patience = 2;
    cfg->has_max_community_weight = 0;
    cfg->max_community_weight = 0.0;
}

sc_status sc_graph_from_csr(sc_ctx* ctx, const uint64_t* node_ptrs, uint64_t n_node_ptrs,
                            const uint32_t* neighbors, uint64_t n_neighbors, const float* weights,
                            uint64_t n_weights, const double* node_weights, uint64_t n_node_weights,
                            sc_graph** out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(out != nullptr, "out is NULL");
        require(n_node_ptrs == 0 || node_ptrs, "node_ptrs is NULL");
        require(n_neighbors == 0 || neighbors, "neighbors is NULL");
        require(n_weights == 0 || weights, "weights is NULL");
        *out = nullptr;
        sc::DevGraph* g = sc::graph_from_csr(c, node_ptrs, n_node_ptrs, neighbors, n_neighbors, weights,
                                             n_weights, node_weights, n_node_weights, false);
        *out = new sc_graph{g};
    });
}

sc_status sc_graph_from_csr_device(sc_ctx* ctx, const uint64_t* node_ptrs, uint64_t n_node_ptrs,
                                   const uint32_t* neighbors, uint64_t n_neighbors,
                                   const float* weights, uint64_t n_weights,
                                   const double* node_weights, uint64_t n_node_weights,
                                   sc_graph** out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(out != nullptr, "out is NULL");
        require(n_node_ptrs == 0 || node_ptrs, "node_ptrs is NULL");
        *out = nullptr;
        sc::DevGraph* g = sc::graph_from_csr(c, node_ptrs, n_node_ptrs, neighbors, n_neighbors, weights,
                                             n_weights, node_weights, n_node_weights, true);
        *out = new sc_graph{g};
    });
}

sc_status sc_graph_from_edges(sc_ctx* ctx, uint64_t n_nodes, const uint64_t* from, const uint64_t* to,
                              const double* weights, uint64_t n_edges, const double* node_weights,
                              sc_graph** out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(out != nullptr, "out is NULL");
        require(n_edges == 0 || (from && to && weights), "edge arrays are NULL");
        *out = nullptr;
        sc::DevGraph* g = sc::graph_from_edges(c, n_nodes, from, to, weights, n_edges, node_weights);
        *out = new sc_graph{g};
    });
}

sc_status sc_graph_from_csr_matrix(sc_ctx* ctx, const uint64_t* row_ptrs, uint64_t n_rows,
                                   const uint64_t* col_indices, const double* values, uint64_t nnz,
                                   const double* node_weights, sc_graph** out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(out != nullptr, "out is NULL");
        require(row_ptrs != nullptr, "row_ptrs is NULL");
        *out = nullptr;
        // upper triangle, non-zero values (csr_network.rs:382-388), in triplet order
        std::vector<uint64_t> f, t;
        std::vector<double> w;
        f.reserve(nnz / 2 + 1);
        t.reserve(nnz / 2 + 1);
        w.reserve(nnz / 2 + 1);
        for (uint64_t r = 0; r < n_rows; ++r)
            for (uint64_t e = row_ptrs[r]; e < row_ptrs[r + 1]; ++e)
                if (r <= col_indices[e] && values[e] != 0.0) {
                    f.push_back(r);
                    t.push_back(col_indices[e]);
                    w.push_back(values[e]);
                }
        sc::DevGraph* g = sc::graph_from_edges(c, n_rows, f.data(), t.data(), w.data(), f.size(),
                                               node_weights);
        *out = new sc_graph{g};
    });
}

void sc_graph_destroy(sc_graph* g) {
    if (!g) return;
    delete g->g;
    delete g;
}

sc_status sc_graph_set_embedding(sc_ctx* ctx, sc_graph* g, const float* X, uint64_t n, uint64_t d) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g, "graph is NULL");
        require_same_device(c, *g->g);
        require(n == g->g->n, "embedding row count differs from the graph's node count");
        sc::graph_set_embedding(c, *g->g, X, d);
    });
}

sc_status sc_graph_info(const sc_graph* g, uint64_t* n_nodes, uint64_t* n_entries, uint64_t* edge_count,
                        double* total_weight, int32_t* any_self_loops) {
    if (!g || !g->g) return SC_E_INVALID_ARGUMENT;
    if (n_nodes) *n_nodes = g->g->n;
    if (n_entries) *n_entries = g->g->E;
    if (edge_count) *edge_count = g->g->edge_count;
    if (total_weight) *total_weight = g->g->total_weight;
    if (any_self_loops) *any_self_loops = g->g->any_self_loops ? 1 : 0;
    return SC_OK;
}

sc_status sc_graph_copy_csr(sc_ctx* ctx, const sc_graph* g, uint64_t* node_ptrs, uint32_t* neighbors,
                            float* weights) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g, "graph is NULL");
        require_same_device(c, *g->g);
        sc::graph_copy_csr(c, *g->g, node_ptrs, neighbors, weights);
    });
}

sc_status sc_graph_copy_node_data(sc_ctx* ctx, const sc_graph* g, double* node_weights, double* strengths) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g, "graph is NULL");
        require_same_device(c, *g->g);
        sc::graph_copy_node_data(c, *g->g, node_weights, strengths);
    });
}

sc_status sc_graph_validate_symmetry(sc_ctx* ctx, const sc_graph* g) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g, "graph is NULL");
        require_same_device(c, *g->g);
        sc::graph_validate_symmetry(c, *g->g);
    });
}

sc_status sc_aggregate(sc_ctx* ctx, const sc_graph* g, const uint64_t* groups, uint64_t n_groups_len,
                       sc_graph** out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && out, "graph or out is NULL");
        require_same_device(c, *g->g);
        const sc::DevGraph& G = *g->g;
        check_membership_len(n_groups_len, G.n);
        *out = nullptr;
        sc::DBuf<uint64_t> dg(c, G.n);
        sc::DBuf<uint32_t> ids(c, G.n);
        sc::h2d(c, dg.get(), groups, G.n);
        uint32_t ng = sc::renumber_u64_labels(c, dg.get(), G.n, ids.get(), nullptr);
        sc::DevGraph* a = sc::graph_aggregate(c, G, ids.get(), ng);
        *out = new sc_graph{a};
    });
}

sc_status sc_modularity(sc_ctx* ctx, const sc_graph* g, const uint64_t* labels, uint64_t n_labels,
                        double resolution, double* out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && out, "graph or out is NULL");
        require_same_device(c, *g->g);
        const sc::DevGraph& G = *g->g;
        check_membership_len(n_labels, G.n);
        sc::DBuf<uint64_t> dl(c, G.n);
        sc::DBuf<uint32_t> ids(c, G.n);
        sc::h2d(c, dl.get(), labels, G.n);
        uint32_t C = sc::renumber_u64_labels(c, dl.get(), G.n, ids.get(), nullptr);
        *out = sc::modularity(c, G, ids.get(), C, resolution);
    });
}

// No device allocation: scratch is the fixed array of sc_static.cu. The first
// call on a device also looks up that array's device address.
sc_status sc_modularity_static(sc_ctx* ctx, const sc_graph* g, const uint32_t* labels_device, uint64_t n_labels,
                               double resolution, double* out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && out, "graph or out is NULL");
        require_same_device(c, *g->g);
        const sc::DevGraph& G = *g->g;
        check_membership_len(n_labels, G.n);
        require(G.n == 0 || labels_device, "labels_device is NULL");
        *out = sc::modularity_static(c, G, labels_device, G.n, resolution);
    });
}

sc_status sc_quality(sc_ctx* ctx, const sc_graph* g, const uint64_t* membership, uint64_t n_membership,
                     int32_t objective, double resolution, double* out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && out, "graph or out is NULL");
        require(objective == SC_OBJECTIVE_RB || objective == SC_OBJECTIVE_CPM, "unknown objective");
        require_same_device(c, *g->g);
        const sc::DevGraph& G = *g->g;
        check_membership_len(n_membership, G.n);
        sc::DBuf<uint64_t> dl(c, G.n);
        sc::DBuf<uint32_t> ids(c, G.n);
        sc::h2d(c, dl.get(), membership, G.n);
        uint32_t C = sc::renumber_u64_labels(c, dl.get(), G.n, ids.get(), nullptr);
        *out = sc::quality(c, G, ids.get(), C, objective, resolution);
    });
}

sc_status sc_partition_stats(sc_ctx* ctx, const sc_graph* g, const uint64_t* membership,
                             uint64_t n_membership, uint64_t* slots_out, uint32_t* size, double* weight,
                             double* strength, double* internal, uint64_t capacity) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && slots_out, "graph or slots_out is NULL");
        require_same_device(c, *g->g);
        const sc::DevGraph& G = *g->g;
        check_membership_len(n_membership, G.n);
        uint64_t slots = 0;
        for (uint64_t i = 0; i < G.n; ++i) slots = std::max<uint64_t>(slots, membership[i] + 1);
        *slots_out = slots;
        require(slots <= capacity, "capacity is smaller than max(membership)+1");
        sc::DBuf<uint64_t> dl(c, G.n);
        sc::DBuf<uint32_t> ids(c, G.n);
        sc::h2d(c, dl.get(), membership, G.n);
        uint32_t C = sc::renumber_u64_labels(c, dl.get(), G.n, ids.get(), nullptr);
        sc::PartStats st;
        sc::partition_stats(c, G, ids.get(), C, st, internal != nullptr);
        std::vector<uint32_t> hs(C);
        std::vector<double> hw(C), hst(C), hin(C);
        sc::d2h(c, hs.data(), st.size.get(), C);
        sc::d2h(c, hw.data(), st.weight.get(), C);
        sc::d2h(c, hst.data(), st.strength.get(), C);
        sc::d2h(c, hin.data(), st.internal.get(), C);
        sc::sync(c);
        // compact id r corresponds to the r-th smallest distinct label
        std::vector<uint64_t> distinct(membership, membership + G.n);
        std::sort(distinct.begin(), distinct.end());
        distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
        if (size) std::fill(size, size + slots, 0u);
        if (weight) std::fill(weight, weight + slots, 0.0);
        if (strength) std::fill(strength, strength + slots, 0.0);
        if (internal) std::fill(internal, internal + slots, 0.0);
        for (uint64_t r = 0; r < distinct.size(); ++r) {
            uint64_t s = distinct[r];
            if (size) size[s] = hs[r];
            if (weight) weight[s] = hw[r];
            if (strength) strength[s] = hst[r];
            if (internal) internal[s] = hin[r];
        }
    });
}

sc_status sc_leiden(sc_ctx* ctx, const sc_graph* g, const sc_leiden_config* cfg, uint64_t* labels_out,
                    uint64_t* n_clusters_out) {
    return sc_leiden_from(ctx, g, cfg, nullptr, 0, labels_out, n_clusters_out);
}

sc_status sc_leiden_from(sc_ctx* ctx, const sc_graph* g, const sc_leiden_config* cfg,
                         const uint64_t* initial, uint64_t n_initial, uint64_t* labels_out,
                         uint64_t* n_clusters_out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(g && g->g && cfg && n_clusters_out, "graph, config or n_clusters_out is NULL");
        require_same_device(c, *g->g);
        const sc::DevGraph& G = *g->g;
        require(G.n == 0 || labels_out, "labels_out is NULL");
        if (initial) check_membership_len(n_initial, G.n);
        sc::DBuf<uint32_t> lab(c, G.n);
        uint64_t ncl = 0;
        sc::leiden(c, G, *cfg, initial, lab.get(), &ncl);
        sc::download_labels(c, lab.get(), G.n, labels_out);
        *n_clusters_out = ncl;
    });
}

sc_status sc_leiden_batch(sc_ctx* ctx, const sc_graph* const* graphs, const sc_leiden_config* cfgs,
                          uint64_t count, const uint64_t* label_offsets, uint64_t* labels_out,
                          uint64_t* n_clusters_out) {
    return sc_leiden_batch_ex(ctx, graphs, cfgs, count, nullptr, label_offsets, labels_out, n_clusters_out, 0);
}

sc_status sc_leiden_batch_ex(sc_ctx* ctx, const sc_graph* const* graphs, const sc_leiden_config* cfgs,
                             uint64_t count, const int64_t* warm_from, const uint64_t* label_offsets,
                             uint64_t* labels_out, uint64_t* n_clusters_out, uint32_t n_streams) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(count == 0 || (graphs && cfgs && label_offsets && labels_out && n_clusters_out),
                "batch arrays are NULL");
        for (uint64_t i = 0; i < count; ++i) {
            require(graphs[i] && graphs[i]->g, "a graph of the batch is NULL");
            require_same_device(c, *graphs[i]->g);
            if (warm_from) {
                require(warm_from[i] < (int64_t)i, "warm_from must name an earlier instance or -1");
                if (warm_from[i] >= 0)
                    require(graphs[warm_from[i]]->g->n == graphs[i]->g->n,
                            "a warm start needs an instance on a graph with the same node count");
            }
        }
        if (count == 0) return;
        uint32_t W = n_streams ? n_streams : 8u;
        if (W > count) W = (uint32_t)count;
        // dependency-ordered work list: instance i is ready once warm_from[i] is done
        std::mutex mu;
        std::condition_variable cv;
        std::vector<char> done(count, 0), taken(count, 0);
        uint64_t remaining = count;
        bool failed = false;
        sc_error_info first_err{};
        auto worker = [&]() {
            sc::Ctx w;
            sc_status st = init_ctx(w, c.device, W <= 8);
            if (st != SC_OK) {
                std::lock_guard<std::mutex> lk(mu);
                if (!failed) {
                    failed = true;
                    first_err.code = st;
                    std::snprintf(first_err.message, sizeof first_err.message, "worker context creation failed");
                }
                cv.notify_all();
                release_ctx(w);
                return;
            }
            for (;;) {
                uint64_t pick = count;
                {
                    std::unique_lock<std::mutex> lk(mu);
                    for (;;) {
                        if (failed || remaining == 0) break;
                        for (uint64_t i = 0; i < count; ++i)
                            if (!taken[i] && (!warm_from || warm_from[i] < 0 || done[warm_from[i]])) {
                                pick = i;
                                break;
                            }
                        if (pick < count) {
                            taken[pick] = 1;
                            break;
                        }
                        bool any_untaken = false;
                        for (uint64_t i = 0; i < count; ++i) any_untaken |= !taken[i];
                        if (!any_untaken) break;
                        cv.wait(lk);
                    }
                }
                if (pick == count) break;
                try {
                    const sc::DevGraph& G = *graphs[pick]->g;
                    const uint64_t* initial = nullptr;
                    if (warm_from && warm_from[pick] >= 0) initial = labels_out + label_offsets[warm_from[pick]];
                    run_instance(w, G, cfgs[pick], initial, labels_out + label_offsets[pick], n_clusters_out + pick);
                } catch (sc::Failure& f) {
                    std::lock_guard<std::mutex> lk(mu);
                    if (!failed) {
                        failed = true;
                        first_err = f.info;
                    }
                }
                {
                    std::lock_guard<std::mutex> lk(mu);
                    done[pick] = 1;
                    remaining--;
                }
                cv.notify_all();
            }
            release_ctx(w);
        };
        std::vector<std::thread> pool;
        for (uint32_t t = 0; t < W; ++t) pool.emplace_back(worker);
        for (auto& th : pool) th.join();
        if (failed) throw sc::Failure{first_err};
    });
}

sc_status sc_leiden_batch_union(sc_ctx* ctx, const sc_graph* const* graphs, const sc_leiden_config* cfgs,
                                uint64_t count, const int64_t* warm_from, const uint64_t* label_offsets,
                                uint64_t* labels_out, uint64_t* n_clusters_out, uint64_t max_union_entries) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(count == 0 || (graphs && cfgs && label_offsets && labels_out && n_clusters_out),
                "batch arrays are NULL");
        std::vector<uint32_t> depth(count, 0);
        for (uint64_t i = 0; i < count; ++i) {
            require(graphs[i] && graphs[i]->g, "a graph of the batch is NULL");
            require_same_device(c, *graphs[i]->g);
            if (warm_from) {
                require(warm_from[i] < (int64_t)i, "warm_from must name an earlier instance or -1");
                if (warm_from[i] >= 0) {
                    require(graphs[warm_from[i]]->g->n == graphs[i]->g->n,
                            "a warm start needs an instance on a graph with the same node count");
                    depth[i] = depth[warm_from[i]] + 1;
                }
            }
        }
        if (count == 0) return;
        const uint64_t cap = max_union_entries ? max_union_entries : (uint64_t(1) << 30);
        const uint32_t max_depth = *std::max_element(depth.begin(), depth.end());
        for (uint32_t d = 0; d <= max_depth; ++d) {
            // the instances whose warm start is done, in index order, packed into unions
            std::vector<uint64_t> wave;
            for (uint64_t i = 0; i < count; ++i)
                if (depth[i] == d) wave.push_back(i);
            size_t a = 0;
            while (a < wave.size()) {
                size_t b = a;
                uint64_t entries = 0, nodes = 0;
                while (b < wave.size() && b - a < 65535) {
                    const sc::DevGraph& g = *graphs[wave[b]]->g;
                    if (b > a && (entries + g.E > cap || nodes + g.n >= 0x7FFFFFFFull)) break;
                    entries += g.E;
                    nodes += g.n;
                    ++b;
                }
                const uint32_t K = (uint32_t)(b - a);
                std::vector<const sc::DevGraph*> gs(K);
                std::vector<sc_leiden_config> cf(K);
                std::vector<uint64_t> n(K), ncl(K);
                std::vector<const uint64_t*> init(K, nullptr);
                for (uint32_t t = 0; t < K; ++t) {
                    const uint64_t i = wave[a + t];
                    gs[t] = graphs[i]->g;
                    cf[t] = cfgs[i];
                    n[t] = gs[t]->n;
                    if (warm_from && warm_from[i] >= 0) init[t] = labels_out + label_offsets[warm_from[i]];
                }
                static const bool trace = std::getenv("SC_TRACE") != nullptr;
                const auto t0 = std::chrono::steady_clock::now();
                std::unique_ptr<sc::DevGraph> u(sc::graph_union(c, gs.data(), K));
                u->stream = c.stream;
                if (trace) {
                    sc::sync(c);
                    std::fprintf(stderr, "[sc] union of %u instances: n=%llu E=%llu exact=%d built in %.3f ms\n", K,
                                 (unsigned long long)u->n, (unsigned long long)u->E, (int)u->exact_w,
                                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                                     .count());
                }
                sc::DBuf<uint32_t> lab(c, std::max<uint64_t>(u->n, 1));
                sc::leiden_union(c, *u, K, n.data(), cf.data(), init.data(), lab.get(), ncl.data());
                uint64_t off = 0;
                for (uint32_t t = 0; t < K; ++t) {
                    const uint64_t i = wave[a + t];
                    sc::download_labels(c, lab.get() + off, n[t], labels_out + label_offsets[i]);
                    n_clusters_out[i] = ncl[t];
                    off += n[t];
                }
                a = b;
            }
        }
    });
}

void sc_knn_opts_default(sc_knn_opts* o) {
    if (!o) return;
    o->sigma = SC_SIGMA_MEDIAN;
    o->sym = SC_SYM_LOWER_ID;
    o->precision = SC_KNN_BF16;
    o->rerank_factor = 2;
    o->squared_kiddo = 0;
}

sc_status sc_knn_gaussian(sc_ctx* ctx, const float* X, uint64_t n, uint64_t d, uint64_t k,
                          const sc_knn_opts* opts, uint32_t* knn_index, float* knn_dist,
                          uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w, uint64_t conn_capacity,
                          uint64_t* conn_nnz, sc_graph** graph_out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(X != nullptr || n == 0, "X is NULL");
        sc_knn_opts o;
        if (opts) o = *opts;
        else sc_knn_opts_default(&o);
        sc::DevGraph* g = nullptr;
        sc::knn_gaussian(c, X, n, d, k, o, knn_index, knn_dist, conn_ptrs, conn_nbrs, conn_w, conn_capacity,
                         conn_nnz, graph_out ? &g : nullptr);
        if (graph_out) *graph_out = new sc_graph{g};
    });
}

sc_status sc_knn_search(sc_ctx* ctx, const float* X, uint64_t n, uint64_t d, uint64_t k, uint64_t q_begin,
                        uint64_t q_end, const sc_knn_opts* opts, uint32_t* knn_index, float* knn_d2) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(X != nullptr || n == 0, "X is NULL");
        sc_knn_opts o;
        if (opts) o = *opts;
        else sc_knn_opts_default(&o);
        sc::knn_search(c, X, n, d, k, q_begin, q_end, o, knn_index, knn_d2);
    });
}

sc_status sc_knn_connectivities(sc_ctx* ctx, const uint32_t* knn_index, const float* knn_d2, uint64_t n, uint64_t k,
                                const sc_knn_opts* opts, uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                                uint64_t conn_capacity, uint64_t* conn_nnz, sc_graph** graph_out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require((knn_index && knn_d2) || n == 0, "knn_index or knn_d2 is NULL");
        sc_knn_opts o;
        if (opts) o = *opts;
        else sc_knn_opts_default(&o);
        sc::DevGraph* g = nullptr;
        sc::knn_connectivities(c, knn_index, knn_d2, n, k, o, conn_ptrs, conn_nbrs, conn_w, conn_capacity, conn_nnz,
                               graph_out ? &g : nullptr);
        if (graph_out) *graph_out = new sc_graph{g};
    });
}

// ---------------------------------------------------------------- learned warm start
namespace {
// Host labels (n entries, nullable) -> compact device ids; empty buffer for NULL.
void upload_labels(sc::Ctx& c, const uint64_t* host, uint64_t n, sc::DBuf<uint32_t>& out) {
    if (!host || n == 0) return;
    sc::DBuf<uint64_t> d(c, n);
    out.alloc(c, n);
    sc::h2d(c, d.get(), host, n);
    sc::renumber_u64_labels(c, d.get(), n, out.get(), nullptr);
}
}  // namespace

uint32_t sc_mlp_param_count(void) { return sc::mlp_param_count(); }

uint32_t sc_mlp_feature_count(void) { return sc::mlp_feature_count(); }

sc_status sc_mlp_create(sc_ctx* ctx, uint64_t seed, sc_mlp** out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(out, "out is NULL");
        *out = nullptr;
        sc::Mlp* m = sc::mlp_create(c, seed);
        *out = new sc_mlp{m, c.device};
    });
}

void sc_mlp_destroy(sc_mlp* m) {
    if (!m) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(m->device);
    sc::mlp_destroy(m->m);
    cudaSetDevice(prev);
    delete m;
}

sc_status sc_mlp_get(sc_ctx* ctx, const sc_mlp* m, float* params, float* scaler, int32_t* has_scaler) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(m && m->m, "model is NULL");
        if (m->device != c.device) bad_arg("model lives on another device than the context");
        const bool has = sc::mlp_get(c, *m->m, params, scaler);
        if (has_scaler) *has_scaler = has ? 1 : 0;
    });
}

sc_status sc_mlp_set(sc_ctx* ctx, sc_mlp* m, const float* params, const float* scaler) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(m && m->m, "model is NULL");
        if (m->device != c.device) bad_arg("model lives on another device than the context");
        sc::mlp_set(c, *m->m, params, scaler);
    });
}

sc_status sc_mlp_features(sc_ctx* ctx, sc_mlp* m, const sc_graph* g, double resolution, const uint64_t* coarse,
                          const uint64_t* fine, float* feat, uint32_t* ei, uint32_t* ej, uint64_t capacity,
                          uint64_t* n_edges) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(m && m->m && g && g->g && n_edges, "model, graph or n_edges is NULL");
        if (m->device != c.device) bad_arg("model lives on another device than the context");
        require_same_device(c, *g->g);
        require(resolution > 0.0 && std::isfinite(resolution), "resolution must be positive and finite");
        sc::DBuf<uint32_t> dc, df;
        upload_labels(c, coarse, g->g->n, dc);
        upload_labels(c, fine, g->g->n, df);
        sc::mlp_features(c, *m->m, *g->g, resolution, dc.get(), df.get(), feat, ei, ej, capacity, n_edges);
    });
}

sc_status sc_mlp_train(sc_ctx* ctx, sc_mlp* m, const sc_graph* g, const uint64_t* membership, uint64_t n_membership,
                       double resolution, const uint64_t* coarse, const uint64_t* fine, uint32_t epochs, double lr,
                       double* loss_out, float* grad_out) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(m && m->m && g && g->g, "model or graph is NULL");
        if (m->device != c.device) bad_arg("model lives on another device than the context");
        require_same_device(c, *g->g);
        require(resolution > 0.0 && std::isfinite(resolution), "resolution must be positive and finite");
        require(lr >= 0.0 && std::isfinite(lr), "learning rate must be non-negative and finite");
        const sc::DevGraph& G = *g->g;
        require(membership || G.n == 0, "membership is NULL");
        check_membership_len(n_membership, G.n);
        sc::DBuf<uint64_t> dl(c, G.n);
        sc::DBuf<uint32_t> ids(c, G.n);
        sc::h2d(c, dl.get(), membership, G.n);
        if (G.n) sc::renumber_u64_labels(c, dl.get(), G.n, ids.get(), nullptr);
        sc::DBuf<uint32_t> dc, df;
        upload_labels(c, coarse, G.n, dc);
        upload_labels(c, fine, G.n, df);
        const double loss = sc::mlp_train(c, *m->m, G, ids.get(), resolution, dc.get(), df.get(), epochs, lr, grad_out);
        if (loss_out) *loss_out = loss;
    });
}

sc_status sc_mlp_propose(sc_ctx* ctx, sc_mlp* m, const sc_graph* g, double resolution, const uint64_t* coarse,
                         const uint64_t* fine, double threshold, double core_fraction, uint64_t* labels_out,
                         uint64_t* n_clusters_out, float* prob_out, uint64_t prob_capacity) {
    return guarded(ctx, [&](sc::Ctx& c) {
        require(m && m->m && g && g->g && n_clusters_out, "model, graph or n_clusters_out is NULL");
        if (m->device != c.device) bad_arg("model lives on another device than the context");
        require_same_device(c, *g->g);
        require(resolution > 0.0 && std::isfinite(resolution), "resolution must be positive and finite");
        require(std::isfinite(threshold), "threshold must be finite");
        require(core_fraction >= 0.0 && core_fraction <= 1.0, "core_fraction must lie in [0, 1]");
        const sc::DevGraph& G = *g->g;
        require(labels_out || G.n == 0, "labels_out is NULL");
        sc::DBuf<uint32_t> lab(c, G.n);
        sc::DBuf<uint32_t> dc, df;
        upload_labels(c, coarse, G.n, dc);
        upload_labels(c, fine, G.n, df);
        const uint64_t k = sc::mlp_propose(c, *m->m, G, resolution, dc.get(), df.get(), threshold, core_fraction,
                                           lab.get(), prob_out, prob_capacity);
        sc::download_labels(c, lab.get(), G.n, labels_out);
        *n_clusters_out = k;
    });
}

}  // extern "C"
