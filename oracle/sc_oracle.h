/*
 * sc_oracle.h — CPU restatement of single-clustering v0.7.0's Leiden path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU library is compared
 * against and the timed CPU baseline; nothing in the product links it.
 *
 * Parity status: the reference is Rust and cannot be built in this
 * environment. The restatement is pinned against every golden vector the
 * reference's own tests hold for this path (karate optimum, the leidenalg /
 * igraph fixture of tests/fixtures/leidenalg_reference.json, the unit-test
 * known answers of csr_network.rs / partition.rs / objective.rs), see
 * tests/test_oracle_golden.py. The random stream is NOT the reference's
 * ChaCha8 / rand 0.9 stream (unpinned by the reference's tests too), so exact
 * labels of a seeded run are not comparable; everything given a partition is.
 *
 * Reuses the status codes and config struct of include/sc_gpu.h.
 */
#ifndef SC_ORACLE_H
#define SC_ORACLE_H

#include "../include/sc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_graph orc_graph;

/* Last error of the calling thread (payload of the ClusteringError variant). */
const sc_error_info* orc_last_error(void);

int orc_graph_from_edges(uint64_t n_nodes, const uint64_t* from, const uint64_t* to,
                         const double* w, uint64_t n_edges, const double* node_w,
                         orc_graph** out);
int orc_graph_from_csr(const uint64_t* ptr, uint64_t n_ptr, const uint32_t* nbr,
                       uint64_t n_nbr, const float* w, uint64_t n_w, const double* node_w,
                       uint64_t n_node_w, orc_graph** out);
int orc_graph_from_csr_matrix(const uint64_t* row_ptr, uint64_t n_rows, const uint64_t* col,
                              const double* val, uint64_t nnz, const double* node_w,
                              orc_graph** out);
void orc_graph_free(orc_graph* g);
void orc_graph_info(const orc_graph* g, uint64_t* n, uint64_t* entries, uint64_t* edge_count,
                    double* total_weight, int32_t* any_loops);
void orc_graph_arrays(const orc_graph* g, uint64_t* ptr, uint32_t* nbr, float* w,
                      double* node_w, double* strength);
int orc_validate_symmetry(const orc_graph* g);

int orc_aggregate(const orc_graph* g, const uint64_t* groups, uint64_t n, orc_graph** out);

/* Partition::from_membership aggregates; arrays of length `capacity` >= slots. */
int orc_partition_stats(const orc_graph* g, const uint64_t* memb, uint64_t n, uint64_t* slots,
                        uint32_t* size, double* weight, double* strength, double* internal,
                        uint64_t capacity);
int orc_quality(const orc_graph* g, const uint64_t* memb, uint64_t n, int32_t objective,
                double resolution, double* out);
int orc_modularity(const orc_graph* g, const uint64_t* labels, uint64_t n, double resolution,
                   double* out);

/* One local_move from `memb` (in/out, slot ids), as in local_move.rs:39-122. */
int orc_local_move(const orc_graph* g, uint64_t* memb, uint64_t n, int32_t objective,
                   double resolution, uint64_t seed, int32_t has_max_cw, double max_cw,
                   double* gain_out);
/* refine (refine.rs:29-103) inside `constraint`; writes refined slot ids. */
int orc_refine(const orc_graph* g, const uint32_t* constraint, uint64_t n, int32_t objective,
               double resolution, uint64_t seed, int32_t has_max_cw, double max_cw,
               double randomness, uint64_t* refined_out);

int orc_leiden(const orc_graph* g, const sc_leiden_config* cfg, const uint64_t* initial,
               uint64_t* labels, uint64_t* n_clusters);

#ifdef __cplusplus
}
#endif

#endif
