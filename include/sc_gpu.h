/*
 * sc_gpu.h — C ABI of the B200 (sm_100a) implementation of single-clustering's
 * Leiden hot path and its Gaussian kNN graph builder.
 *
 * Every entry point mirrors one Rust API of single-clustering v0.7.0; the
 * reference item each one replaces is cited beside it as `file:line` relative
 * to the single-clustering source tree.
 *
 * Conventions
 *   - Every function returns an `sc_status`. `SC_OK` is success; the codes 1..10
 *     map one-to-one onto the variants of `ClusteringError` (src/error.rs:7-68),
 *     the rest are device / argument failures the Rust API has no variant for.
 *   - Input arrays are HOST pointers owned by the caller unless the name says
 *     `_device`; the library copies them to the GPU. Outputs are host buffers
 *     the caller sized.
 *   - Ids are `uint32_t` inside the adjacency (`u32`, csr_network.rs:35-36),
 *     offsets and labels are `uint64_t` (`usize`), weights `float` in storage
 *     and `double` in every per-node quantity and every piece of arithmetic.
 *   - One `sc_ctx` per host thread. A context owns one CUDA stream, a memory
 *     pool, a device status word and the last error. Graph handles are
 *     immutable after construction and may be shared between contexts on the
 *     same device.
 *   - The library never aborts the process: device-side guards (bounded waits,
 *     bounds checks) set a status word that the host turns into SC_E_TIMEOUT /
 *     SC_E_INTERNAL.
 */
#ifndef SC_GPU_H
#define SC_GPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SC_GPU_ABI_VERSION 1

/* Status codes. 1..10 follow ClusteringError (src/error.rs:7-68) in order. */
typedef enum sc_status {
    SC_OK = 0,
    SC_E_NODE_INDEX_OUT_OF_RANGE = 1,     /* NodeIndexOutOfRange { node, n_nodes }        */
    SC_E_NON_FINITE_WEIGHT = 2,           /* NonFiniteWeight { edge }                     */
    SC_E_NEGATIVE_WEIGHT = 3,             /* NegativeWeight { edge, weight }              */
    SC_E_INVALID_NODE_WEIGHT = 4,         /* InvalidNodeWeight { node, weight }           */
    SC_E_NODE_WEIGHT_LENGTH_MISMATCH = 5, /* NodeWeightLengthMismatch { got, expected }   */
    SC_E_MEMBERSHIP_LENGTH_MISMATCH = 6,  /* MembershipLengthMismatch { got, expected }   */
    SC_E_INVALID_CONFIG = 7,              /* InvalidConfig(String)                        */
    SC_E_TOO_MANY_NODES = 8,              /* TooManyNodes { n_nodes }                     */
    SC_E_INVALID_CSR = 9,                 /* InvalidCsr(String)                           */
    SC_E_ASYMMETRIC_GRAPH = 10,           /* AsymmetricGraph { degree_sum, expected }     */
    SC_E_INVALID_ARGUMENT = 20,           /* null handle / pointer, bad enum value        */
    SC_E_CUDA = 21,                       /* a CUDA runtime call failed                   */
    SC_E_OUT_OF_MEMORY = 22,              /* device allocation failed                     */
    SC_E_TIMEOUT = 23,                    /* a bounded device wait gave up                */
    SC_E_INTERNAL = 24,                   /* an internal invariant failed (a bug)         */
    SC_E_UNSUPPORTED = 25                 /* shape outside what a kernel supports         */
} sc_status;

/* Payload of the last error, field meaning follows the ClusteringError variant. */
typedef struct sc_error_info {
    int32_t code;          /* sc_status of the failure                                */
    uint64_t node;         /* NodeIndexOutOfRange.node, InvalidNodeWeight.node        */
    uint64_t n_nodes;      /* NodeIndexOutOfRange.n_nodes, TooManyNodes.n_nodes       */
    uint64_t edge_from;    /* NonFiniteWeight/NegativeWeight .edge.0                  */
    uint64_t edge_to;      /* NonFiniteWeight/NegativeWeight .edge.1                  */
    double weight;         /* NegativeWeight.weight, InvalidNodeWeight.weight         */
    uint64_t got;          /* *LengthMismatch.got                                     */
    uint64_t expected_len; /* *LengthMismatch.expected                                */
    double degree_sum;     /* AsymmetricGraph.degree_sum                              */
    double expected;       /* AsymmetricGraph.expected                                */
    char message[256];     /* Display text of the error, NUL-terminated               */
} sc_error_info;

/* ObjectiveKind (src/community_search/leiden/objective.rs:188-199). */
typedef enum sc_objective { SC_OBJECTIVE_RB = 0, SC_OBJECTIVE_CPM = 1 } sc_objective;

/*
 * LeidenConfig (src/community_search/leiden/mod.rs:49-106), field for field.
 * `Option<T>` fields are a has_ flag plus the value.
 */
typedef struct sc_leiden_config {
    int32_t objective;              /* sc_objective                         */
    double resolution;              /* ObjectiveKind::{Rb,Cpm}.resolution   */
    int32_t has_seed;               /* seed: Option<u64>                    */
    uint64_t seed;
    uint64_t n_iterations;          /* default 2                            */
    uint64_t max_levels;            /* default 64                           */
    double tolerance;               /* default 1e-9                         */
    int32_t refine;                 /* default 1; 0 = Louvain               */
    double refine_randomness;       /* default 0.01                         */
    uint64_t patience;              /* default 2                            */
    int32_t has_max_community_weight;
    double max_community_weight;
} sc_leiden_config;

/* Per-run counters of the last sc_leiden* call on a context (host-side copy). */
typedef struct sc_run_stats {
    uint64_t passes;                /* passes actually run                        */
    uint64_t levels;                /* levels summed over passes                  */
    uint64_t local_move_sweeps;     /* local-moving sweeps summed over levels     */
    uint64_t moves;                 /* committed local moves                      */
    uint64_t kernel_launches;       /* kernels this library launched for the run  */
    double ms_local_move;           /* device time per phase, CUDA events         */
    double ms_refine;
    double ms_aggregate;
    double ms_other;
    double ms_total;
    double alg_bytes_local_move;    /* algorithmic bytes of the local-move sweeps */
    double alg_bytes_refine;
    double alg_bytes_aggregate;
} sc_run_stats;

/*
 * Launch tuning of a context (no counterpart in single-clustering). Nodes of
 * degree <= lanes8_max_degree are scored by groups of 8 lanes, <= lanes16 by 16,
 * <= lanes32 by 32, the rest by a warp, a block or (past 1024) a block with a
 * global-memory table; a batch of at most small_batch nodes of degree <= 256 is
 * scored by the warp kernel in one launch. Every routing gives the same
 * decisions (the kernels score the same candidates with the same arithmetic and
 * tie rule), so tuning changes speed only, never labels.
 * Limits: lanes8 <= 8, lanes8 <= lanes16 <= 16, lanes16 <= lanes32 <= 32.
 */
typedef struct sc_tuning {
    uint32_t lanes8_max_degree;   /* default 8  */
    uint32_t lanes16_max_degree;  /* default 16 */
    uint32_t lanes32_max_degree;  /* default 32 */
    uint32_t small_batch;         /* default 4096 */
} sc_tuning;

typedef struct sc_ctx sc_ctx;
typedef struct sc_graph sc_graph;

/* ---- context ------------------------------------------------------------ */
uint32_t sc_abi_version(void);
sc_status sc_ctx_create(int32_t device, sc_ctx** out);
void sc_ctx_destroy(sc_ctx* ctx);
/* Display text of the last error on this context ("" after success). */
const char* sc_last_error_message(const sc_ctx* ctx);
sc_status sc_last_error_info(const sc_ctx* ctx, sc_error_info* out);
sc_status sc_last_run_stats(const sc_ctx* ctx, sc_run_stats* out);
/* Blocks until all work of the context's stream is done. */
sc_status sc_ctx_synchronize(sc_ctx* ctx);
/* LeidenConfig::default() (src/community_search/leiden/mod.rs:92-106). */
void sc_leiden_config_default(sc_leiden_config* cfg);

void sc_tuning_default(sc_tuning* t);
sc_status sc_get_tuning(const sc_ctx* ctx, sc_tuning* out);
/* Validates the limits above (SC_E_INVALID_ARGUMENT otherwise). */
sc_status sc_set_tuning(sc_ctx* ctx, const sc_tuning* t);
/*
 * Bounded device waits (no counterpart in single-clustering, which has no
 * device code). Each pipeline wait of the kNN candidate kernel (a TMA copy
 * landing, an accumulator filled or drained) tries at most `limit` times, then
 * the kernel stops, waits with the library's default limit for the copies and
 * MMAs it already issued, frees its tensor memory and returns; the call then
 * fails with SC_E_TIMEOUT and the context stays usable. Default 2^26.
 */
sc_status sc_set_wait_limit(sc_ctx* ctx, uint32_t limit);
sc_status sc_get_wait_limit(const sc_ctx* ctx, uint32_t* out);
/*
 * Test hook for the bounded waits: while on, the kNN kernel's producer issues
 * the query tiles but never a point tile, so the first wait for one runs out
 * its limit (set a small one with sc_set_wait_limit) and the kNN call returns
 * SC_E_TIMEOUT without any copy or MMA left in flight. Off by default.
 */
sc_status sc_test_knn_hold_tiles(sc_ctx* ctx, int32_t on);

/*
 * Autotuner: times the first level of `cfg` (one pass, one level: the level
 * that dominates a run) on g under each candidate routing, keeps the fastest
 * on the context and returns it with its time and the default's (device time,
 * ms). n_candidates (nullable) receives how many were timed.
 */
sc_status sc_autotune(sc_ctx* ctx, const sc_graph* g, const sc_leiden_config* cfg, sc_tuning* chosen,
                      double* ms_chosen, double* ms_default, uint32_t* n_candidates);

/* ---- graph construction ------------------------------------------------- */
/*
 * CSRNetwork::from_csr_parts (src/network/csr_network.rs:185-256) followed by
 * finish (:262-351) and check_degree_sum (:712-723), computed on the GPU.
 * Each Vec of the Rust signature is a pointer plus its length, so every length
 * check of the reference is reproduced. node_weights may be NULL (= None).
 */
sc_status sc_graph_from_csr(sc_ctx* ctx,
                            const uint64_t* node_ptrs, uint64_t n_node_ptrs,
                            const uint32_t* neighbors, uint64_t n_neighbors,
                            const float* weights, uint64_t n_weights,
                            const double* node_weights, uint64_t n_node_weights,
                            sc_graph** out);

/* Same contract, inputs already in this device's memory (kNN output hand-off). */
sc_status sc_graph_from_csr_device(sc_ctx* ctx,
                                   const uint64_t* node_ptrs_device, uint64_t n_node_ptrs,
                                   const uint32_t* neighbors_device, uint64_t n_neighbors,
                                   const float* weights_device, uint64_t n_weights,
                                   const double* node_weights_device, uint64_t n_node_weights,
                                   sc_graph** out);

/*
 * CSRNetwork::from_edges / from_edges_with_node_weights
 * (src/network/csr_network.rs:104-167). Edge i is (from[i], to[i], weights[i]);
 * weights are given as double (W::to_f64) and stored `as f32`. node_weights may
 * be NULL, meaning unit weights over n_nodes nodes.
 */
sc_status sc_graph_from_edges(sc_ctx* ctx, uint64_t n_nodes,
                              const uint64_t* from, const uint64_t* to,
                              const double* weights, uint64_t n_edges,
                              const double* node_weights, sc_graph** out);

/*
 * CSRNetwork::from_csr_matrix (src/network/csr_network.rs:360-391): reads only
 * entries with row <= col and non-zero value, then from_edges.
 */
sc_status sc_graph_from_csr_matrix(sc_ctx* ctx,
                                   const uint64_t* row_ptrs, uint64_t n_rows,
                                   const uint64_t* col_indices, const double* values,
                                   uint64_t nnz, const double* node_weights,
                                   sc_graph** out);

/* Drop(CSRNetwork): waits for the device, then returns the graph's arrays to
 * the library's graph pool (kept for the next graph until the process exits). */
void sc_graph_destroy(sc_graph* g);

/* Attaches the kNN embedding the graph was built from (n x d float32,
 * row-major host memory, n = node count) for the learned warm start's
 * features: the library keeps its projection to 16 components per node (a
 * fixed sign matrix), replacing any earlier one. The reference's Leiden takes
 * no embedding; its kNN builder (src/neighborhood/mod.rs) starts from one.
 * This is the one call that changes a graph: make it before the graph is
 * shared, not while another context uses the graph. */
sc_status sc_graph_set_embedding(sc_ctx* ctx, sc_graph* g, const float* X, uint64_t n, uint64_t d);

/* node_count, stored entries, edge_count, total_weight, has_self_loops
 * (src/network/csr_network.rs:407-442, :648-652). */
sc_status sc_graph_info(const sc_graph* g, uint64_t* n_nodes, uint64_t* n_entries,
                        uint64_t* edge_count, double* total_weight, int32_t* any_self_loops);

/* to_csr_parts (src/network/csr_network.rs:484-490): node_ptrs n+1, neighbors
 * and weights n_entries each. Any pointer may be NULL to skip it. */
sc_status sc_graph_copy_csr(sc_ctx* ctx, const sc_graph* g, uint64_t* node_ptrs,
                            uint32_t* neighbors, float* weights);

/* node_weights (csr_network.rs:493-495) and strengths (:428-430), n each. */
sc_status sc_graph_copy_node_data(sc_ctx* ctx, const sc_graph* g, double* node_weights,
                                  double* strengths);

/* validate_symmetry (src/network/csr_network.rs:627-646); SC_E_INVALID_CSR on failure. */
sc_status sc_graph_validate_symmetry(sc_ctx* ctx, const sc_graph* g);

/*
 * CSRNetwork::aggregate (src/network/csr_network.rs:516-608) with the grouping
 * VectorGrouping::from_assignments(groups) (src/network/grouping.rs:154-172),
 * i.e. group ids are first renumbered by ascending rank.
 */
sc_status sc_aggregate(sc_ctx* ctx, const sc_graph* g, const uint64_t* groups,
                       uint64_t n_groups_len, sc_graph** out);

/* ---- evaluation --------------------------------------------------------- */
/* modularity (src/community_search/leiden/objective.rs:221-244). */
sc_status sc_modularity(sc_ctx* ctx, const sc_graph* g, const uint64_t* labels,
                        uint64_t n_labels, double resolution, double* out);

/*
 * Modularity for callers that cannot allocate device memory (a host framework
 * that owns the device memory pool, a fixed device-memory budget, a section
 * where cudaMalloc's implicit synchronisation is not allowed). No counterpart
 * in the reference: it is sc_modularity with the labels already on the device
 * as compact uint32 ids (< 65,536, so at most 65,536 communities; larger ids
 * return SC_E_UNSUPPORTED) and no device allocation. Its scratch is a fixed
 * 1 MiB array in the library, held by every GPU that loads the library until
 * the process exits; a call looks up that array's address for the current
 * device and CUDA context the first time it meets them. Every call ends by
 * synchronising the context's stream and reading the result back, so it must
 * not be called while that stream is being captured into a CUDA graph. Every
 * call shares the array: calls whose work overlaps on the GPU race and must be
 * serialised.
 * Bit-exact with sc_modularity when every sum of the graph's edge weights is
 * exact in f64 (all unit or f32-valued weights below 2^(52+e0) in total);
 * otherwise it may differ in the last bits.
 */
sc_status sc_modularity_static(sc_ctx* ctx, const sc_graph* g, const uint32_t* labels_device,
                               uint64_t n_labels, double resolution, double* out);

/* Partition::from_membership (partition.rs:75-112) then Rb::quality (objective.rs:108-119)
 * or Cpm::quality (:171-178). */
sc_status sc_quality(sc_ctx* ctx, const sc_graph* g, const uint64_t* membership,
                     uint64_t n_membership, int32_t objective, double resolution, double* out);

/*
 * Partition::from_membership aggregates (partition.rs:75-112): per slot
 * c < slots = max(membership)+1, size, weight, strength and internal. Any output
 * may be NULL. *slots_out receives the slot count.
 */
sc_status sc_partition_stats(sc_ctx* ctx, const sc_graph* g, const uint64_t* membership,
                             uint64_t n_membership, uint64_t* slots_out, uint32_t* size,
                             double* weight, double* strength, double* internal,
                             uint64_t capacity);

/* ---- Leiden ------------------------------------------------------------- */
/* leiden(&graph, &config) (src/community_search/leiden/mod.rs:168-204).
 * labels_out has node_count entries, consecutive from 0. */
sc_status sc_leiden(sc_ctx* ctx, const sc_graph* g, const sc_leiden_config* cfg,
                    uint64_t* labels_out, uint64_t* n_clusters_out);

/* leiden starting from `initial` labels instead of singletons: the `initial`
 * argument of run_once (src/community_search/leiden/mod.rs:207-220). */
sc_status sc_leiden_from(sc_ctx* ctx, const sc_graph* g, const sc_leiden_config* cfg,
                         const uint64_t* initial, uint64_t n_initial,
                         uint64_t* labels_out, uint64_t* n_clusters_out);

/*
 * Many independent leiden() calls in one batched launch sequence: instance i
 * runs `cfgs[i]` on `graphs[i]` (graphs may repeat) and writes labels_out at
 * label_offsets[i] (caller computes offsets; each instance needs node_count
 * entries). No reference counterpart as one call; semantically a loop over
 * leiden (src/community_search/leiden/mod.rs:168).
 */
sc_status sc_leiden_batch(sc_ctx* ctx, const sc_graph* const* graphs,
                          const sc_leiden_config* cfgs, uint64_t count,
                          const uint64_t* label_offsets, uint64_t* labels_out,
                          uint64_t* n_clusters_out);

/*
 * sc_leiden_batch with its scheduling exposed. Instances run concurrently on
 * n_streams worker streams (0 = 8), each with its own stream and state, so the
 * small kernels of coarse levels from different instances overlap. When
 * warm_from is non-NULL, instance i with warm_from[i] = j >= 0 (j < i, same
 * node count) starts from instance j's final labels — leiden with `initial`
 * (run_once, src/community_search/leiden/mod.rs:207-220) — and waits for j;
 * -1 starts from singletons. A resolution sweep chains each resolution to its
 * neighbour this way.
 */
sc_status sc_leiden_batch_ex(sc_ctx* ctx, const sc_graph* const* graphs,
                             const sc_leiden_config* cfgs, uint64_t count,
                             const int64_t* warm_from, const uint64_t* label_offsets,
                             uint64_t* labels_out, uint64_t* n_clusters_out,
                             uint32_t n_streams);

/*
 * sc_leiden_batch_ex's instances as batched device work instead of host
 * threads: instances whose warm start (warm_from, as in sc_leiden_batch_ex) is
 * done run together over the disjoint union of their graphs, every kernel
 * launch covering the nodes of all of them, with each instance's resolution,
 * seed, totals and stopping state in device arrays. Each instance takes the
 * decisions of its own leiden() run (hashes and tie rules see instance-local
 * ids, and an instance stops where its own run stops); inside the exact
 * summation regime its labels are those of sc_leiden / sc_leiden_from bit for
 * bit. All instances need one objective kind, refine setting and
 * max_community_weight. A union holds at most max_union_entries stored entries
 * (0 = 2^30) and 65,535 instances; larger waves split into several. No
 * reference counterpart as one call; semantically a loop over leiden
 * (src/community_search/leiden/mod.rs:168-220).
 */
sc_status sc_leiden_batch_union(sc_ctx* ctx, const sc_graph* const* graphs, const sc_leiden_config* cfgs,
                                uint64_t count, const int64_t* warm_from, const uint64_t* label_offsets,
                                uint64_t* labels_out, uint64_t* n_clusters_out, uint64_t max_union_entries);

/* ---- kNN graph builder --------------------------------------------------- */
typedef enum sc_knn_sigma { SC_SIGMA_MEDIAN = 0, SC_SIGMA_KTH = 1 } sc_knn_sigma;
typedef enum sc_knn_sym { SC_SYM_LOWER_ID = 0, SC_SYM_UNION = 1 } sc_knn_sym;
typedef enum sc_knn_precision { SC_KNN_FP32 = 0, SC_KNN_BF16 = 1, SC_KNN_FP8 = 2 } sc_knn_precision;

typedef struct sc_knn_opts {
    int32_t sigma;        /* sc_knn_sigma; median = reference (neighborhood/mod.rs:105-124, :480-499) */
    int32_t sym;          /* sc_knn_sym;   lower_id = reference (neighborhood/mod.rs:138-163)         */
    int32_t precision;    /* sc_knn_precision of the candidate distances: BF16 or FP8 e4m3 on the
                             tensor cores (norm-expanded contraction, FP32 accumulation), or FP32
                             on the CUDA cores (exact differences, the re-rank's arithmetic)       */
    int32_t rerank_factor;/* candidates kept per row before the exact FP32 re-rank = factor * (k+1)  */
    int32_t squared_kiddo;/* 1: kd-tree path semantics (squared distances, sigma = sqrt(median d^2)) */
} sc_knn_opts;

void sc_knn_opts_default(sc_knn_opts* opts);

/*
 * Exact pruning of the kNN search (no counterpart in single-clustering, whose
 * kd-tree prunes on the host). A search of n >= 65,536 points groups them
 * with a deterministic k-means into `clusters` clusters (0: n / 8192, within
 * 16..256), orders each cluster's points by fine cells of about 256 points,
 * and skips, per group of 256 queries, every cell that a ball or slab bound
 * proves farther than each query's (k+1)-th neighbour among its own cluster;
 * the lists equal the full scan's. 1 scans every point tile.
 * Applies to BF16 / FP8 searches of all rows (sc_knn_gaussian); row shards
 * (sc_knn_search) and FP32 candidates scan every point.
 */
sc_status sc_set_knn_clusters(sc_ctx* ctx, uint32_t clusters);

/*
 * kNN autotuner (no counterpart in single-clustering): times the exact search
 * of all n rows of X under candidate cluster counts (1 = full scan, and 32 ..
 * 256 where n allows) and keeps the fastest on the context (as
 * sc_set_knn_clusters would). Every candidate gives the same lists, so it
 * changes speed only. Outputs (each nullable): the count chosen, its device
 * time and the full scan's (ms), the number of candidates timed.
 */
sc_status sc_knn_autotune(sc_ctx* ctx, const float* X, uint64_t n, uint64_t d, uint64_t k, const sc_knn_opts* opts,
                          uint32_t* chosen_clusters, double* ms_chosen, double* ms_full, uint32_t* n_candidates);

/* Counters of the last kNN search on a context. */
typedef struct sc_knn_stats {
    uint64_t clusters;       /* point clusters of the pruned search (0: full scan)     */
    uint64_t tiles_scanned;  /* (query group, point tile) pairs the contraction ran    */
    uint64_t tiles_full;     /* the pairs of a full scan                               */
    uint64_t tiles_pass1;    /* of tiles_scanned: the own-cluster bounding pass        */
    double ms_cluster;       /* device time: k-means, sort by cluster, cluster extents */
    double ms_pass1;         /* the own-cluster pass (contraction and re-rank)         */
    double ms_bounds;        /* the bounds deciding each group's clusters              */
    double ms_pass2;         /* the final pass (contraction and re-rank)               */
} sc_knn_stats;
sc_status sc_knn_last_stats(const sc_ctx* ctx, sc_knn_stats* out);

/*
 * knn_arrayd_kiddo_gaussian / knn_arrayd_hnswlib_gaussian
 * (src/neighborhood/mod.rs:51-202, :359-578), exact on the GPU. X is row-major
 * n x d float. Outputs (host):
 *   knn_index   n*(k+1) neighbour ids per row, self first, ascending distance
 *   knn_dist    n*(k+1) distances (squared when opts.squared_kiddo), may be NULL
 * and the connectivities CSR, which is returned as a graph handle built with
 * from_csr_parts semantics when `graph_out` is non-NULL, and/or copied to host
 * when conn_ptrs is non-NULL (conn_nnz receives the entry count; conn_nbrs /
 * conn_w must then hold conn_capacity entries).
 */
sc_status sc_knn_gaussian(sc_ctx* ctx, const float* X, uint64_t n, uint64_t d, uint64_t k,
                          const sc_knn_opts* opts, uint32_t* knn_index, float* knn_dist,
                          uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                          uint64_t conn_capacity, uint64_t* conn_nnz, sc_graph** graph_out);

/* The search of sc_knn_gaussian for the query rows [q_begin, q_end) only,
 * against all n points: one shard of a build split across GPUs by query rows.
 * knn_index / knn_d2 receive (q_end - q_begin) x (k+1) entries, self first,
 * with SQUARED FP32 distances (whatever opts.squared_kiddo says). No
 * counterpart in single-clustering, whose kNN runs on one host. */
sc_status sc_knn_search(sc_ctx* ctx, const float* X, uint64_t n, uint64_t d, uint64_t k, uint64_t q_begin,
                        uint64_t q_end, const sc_knn_opts* opts, uint32_t* knn_index, float* knn_d2);

/* The connectivity step of sc_knn_gaussian from the gathered k+1 lists of all
 * n points (squared distances, as sc_knn_search writes them); outputs as in
 * sc_knn_gaussian. */
sc_status sc_knn_connectivities(sc_ctx* ctx, const uint32_t* knn_index, const float* knn_d2, uint64_t n, uint64_t k,
                                const sc_knn_opts* opts, uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                                uint64_t conn_capacity, uint64_t* conn_nnz, sc_graph** graph_out);

/* ---------------------------------------------------------------- learned warm start
 * No counterpart in single-clustering: its only warm-start hook is the
 * `initial` membership of run_once (src/community_search/leiden/mod.rs:207-220),
 * which sc_leiden_from exposes. These functions produce such a membership.
 *
 * The model is a 2-layer MLP (sc_mlp_feature_count() inputs, 128 hidden units,
 * ReLU, one logit) scoring each undirected edge with the probability that its
 * endpoints share a community, from endpoint degree/strength, the edge weight,
 * the RB null-model term at the given resolution, the endpoints' common
 * neighbourhood, when given the partitions found at a neighbouring lower
 * (`coarse`) and higher (`fine`) resolution (host label arrays of n entries,
 * each nullable) whether the endpoints share a community there and how much of
 * each endpoint's strength its neighbour-label histogram puts in the other's
 * community, and, when the graph carries an embedding
 * (sc_graph_set_embedding), the edge's length in the projected embedding
 * relative to the endpoints' local scale. A model trained with a context or an
 * embedding is meant to be used with them. The contraction runs on the tensor
 * cores (BF16 operands, features and hidden gradients split into two BF16
 * parts, FP32 accumulation); Adam updates an FP32 master copy. The features
 * that depend on neither the resolution nor a context (40 bytes per undirected
 * edge, plus the edge list: 64 bytes per edge) are computed on a graph's first
 * use and kept with the graph until sc_graph_destroy or a new
 * sc_graph_set_embedding. Parameters are laid out W1[f*128+u], b1[u],
 * w2[u], b2 (sc_mlp_param_count() floats). The feature scaler (means, then
 * inverse standard deviations, 2 * feature_count floats) is fitted on the first
 * graph the model trains on or extracts features from.
 *
 * The proposal is the connected components of the edges whose probability
 * exceeds `threshold` and whose endpoints are both core nodes (at least
 * `core_fraction` of their edges exceed the threshold), numbered 0..k-1 by
 * smallest member; other nodes stay singletons. Pass it to sc_leiden_from as
 * `initial`.
 */
typedef struct sc_mlp sc_mlp;

uint32_t sc_mlp_param_count(void);
uint32_t sc_mlp_feature_count(void);
sc_status sc_mlp_create(sc_ctx* ctx, uint64_t seed, sc_mlp** out);
void sc_mlp_destroy(sc_mlp* m);
/* Copies the parameters and/or the scaler (either may be NULL) to host;
 * *has_scaler (nullable) says whether a scaler is set. */
sc_status sc_mlp_get(sc_ctx* ctx, const sc_mlp* m, float* params, float* scaler, int32_t* has_scaler);
/* Replaces the parameters (resets the Adam state) and/or the scaler. */
sc_status sc_mlp_set(sc_ctx* ctx, sc_mlp* m, const float* params, const float* scaler);
/* The scaled edge features the model sees for g at `resolution`, edges (i < j)
 * in ascending (i, j) order: feat[e * feature_count + f], endpoints ei/ej (each
 * nullable). `capacity` is the room in edges; *n_edges receives the count. */
sc_status sc_mlp_features(sc_ctx* ctx, sc_mlp* m, const sc_graph* g, double resolution, const uint64_t* coarse,
                          const uint64_t* fine, float* feat, uint32_t* ei, uint32_t* ej, uint64_t capacity,
                          uint64_t* n_edges);
/* `epochs` full-batch Adam steps (learning rate lr) of the mean binary
 * cross-entropy against "same community in `membership`". *loss_out receives the
 * loss before the last step; grad_out (nullable, param_count floats) the last
 * gradient. epochs == 0 evaluates loss and gradient without a step. */
sc_status sc_mlp_train(sc_ctx* ctx, sc_mlp* m, const sc_graph* g, const uint64_t* membership, uint64_t n_membership,
                       double resolution, const uint64_t* coarse, const uint64_t* fine, uint32_t epochs, double lr,
                       double* loss_out, float* grad_out);
/* Initial membership for sc_leiden_from (see above); prob_out (nullable) gets
 * the edge probabilities in sc_mlp_features order, prob_capacity entries. */
sc_status sc_mlp_propose(sc_ctx* ctx, sc_mlp* m, const sc_graph* g, double resolution, const uint64_t* coarse,
                         const uint64_t* fine, double threshold, double core_fraction, uint64_t* labels_out,
                         uint64_t* n_clusters_out, float* prob_out, uint64_t prob_capacity);

#ifdef __cplusplus
}
#endif

#endif /* SC_GPU_H */
