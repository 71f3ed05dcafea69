// sc_partition.cu — Partition::from_membership aggregates, RB / CPM quality and
// modularity on the GPU, with the reference's f64 results bit for bit.
//
// Per-community sums follow the reference's order (ascending node, then
// ascending neighbour). In the exact regime (see sc_graph.cu) they are taken
// with f64 atomics over all entries at once, which is exact and therefore
// order-independent; outside it one thread walks each community in order.
// The final Σ over communities is always an ordered chain: its terms are
// arbitrary doubles.
#include "sc_prims.cuh"

namespace sc {

namespace {
constexpr unsigned TB = 256;

__global__ void k_iota32(uint32_t* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

__global__ void k_heads_u64(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* head) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// rank (inclusive scan of heads, minus one) scattered back to node order
__global__ void k_scatter_rank(const uint32_t* __restrict__ order, const uint32_t* __restrict__ incl,
                               uint64_t n, uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[order[i]] = incl[i] - 1;
}

__global__ void k_mark_used(const uint32_t* __restrict__ ids, uint64_t n, uint32_t* used) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        used[ids[i]] = 1u;
}

__global__ void k_apply_rank(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ rank,
                             uint64_t n, uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = rank[ids[i]];
}

__global__ void k_starts_u32(const uint32_t* __restrict__ rows, uint64_t N, uint64_t R,
                             uint64_t* start) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = i < N ? rows[i] : R;
        uint64_t prev = i == 0 ? 0 : (uint64_t)rows[i - 1] + 1;
        for (uint64_t q = prev; q <= r && q <= R; ++q) start[q] = i;
    }
}

// Ordered per-community aggregates, one warp per community walking its members
// in ascending order (partition.rs:90-105); internal sums each member's row in
// ascending neighbour order, entries outside the rule adding +0.0 (a no-op).
__global__ void k_stats_ordered(const uint64_t* __restrict__ cstart, const uint32_t* __restrict__ members,
                                uint64_t C, const uint32_t* __restrict__ memb,
                                const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                                const float* __restrict__ w, const double* __restrict__ node_w,
                                const double* __restrict__ strength, uint32_t* size, double* weight,
                                double* stren, double* internal, int need_internal) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = warp; c < C; c += nwarps) {
        const uint64_t b = cstart[c], e = cstart[c + 1];
        const double a = warp_ordered_sum(b, e, 0.0, [&](uint64_t i) { return node_w[members[i]]; });
        const double s = warp_ordered_sum(b, e, 0.0, [&](uint64_t i) { return strength[members[i]]; });
        double in = 0.0;
        if (need_internal) {
            for (uint64_t i = b; i < e; ++i) {
                const uint32_t v = members[i];
                in = warp_ordered_sum(ptr[v], ptr[v + 1], in, [&](uint64_t j) {
                    const uint32_t u = nbr[j];
                    return (memb[u] == (uint32_t)c && (u == v || v < u)) ? (double)w[j] : 0.0;
                });
            }
        }
        if ((threadIdx.x & 31) == 0) {
            size[c] = (uint32_t)(e - b);
            weight[c] = a;
            stren[c] = s;
            internal[c] = in;
        }
    }
}

// Exact-regime aggregates: every partial sum is exact, so atomics are exact.
__global__ void k_stats_nodes_atomic(const uint32_t* __restrict__ memb, uint64_t n,
                                     const double* __restrict__ node_w,
                                     const double* __restrict__ strength, uint32_t* size,
                                     double* weight, double* stren) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = memb[v];
        atomicAdd(size + c, 1u);
        atomicAdd(weight + c, node_w[v]);
        atomicAdd(stren + c, strength[v]);
    }
}

__global__ void k_internal_atomic(const uint32_t* __restrict__ erow, const uint32_t* __restrict__ nbr,
                                  const float* __restrict__ w, uint64_t E,
                                  const uint32_t* __restrict__ memb, double* internal) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = erow[e], u = nbr[e];
        if (v <= u) {
            uint32_t c = memb[v];
            if (memb[u] == c) atomicAdd(internal + c, (double)w[e]);
        }
    }
}

// Rb::quality / Cpm::quality terms (objective.rs:108-119, :171-178)
__global__ void k_quality_terms(const double* __restrict__ weight, const double* __restrict__ stren,
                                const double* __restrict__ internal, uint64_t C, int objective,
                                double gamma, double four_m, double* terms) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < C;
         c += (uint64_t)gridDim.x * blockDim.x) {
        double t;
        if (objective == SC_OBJECTIVE_RB) {
            double k = stren[c];
            t = __dsub_rn(internal[c], __ddiv_rn(__dmul_rn(__dmul_rn(gamma, k), k), four_m));
        } else {
            double nc = weight[c];
            t = __dsub_rn(internal[c],
                          __ddiv_rn(__dmul_rn(__dmul_rn(gamma, nc), __dsub_rn(nc, 1.0)), 2.0));
        }
        terms[c] = t;
    }
}

// modularity terms (objective.rs:240-243)
__global__ void k_modularity_terms(const double* __restrict__ stren, const double* __restrict__ internal,
                                   uint64_t C, double gamma, double two_m, double* terms) {
    for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < C;
         c += (uint64_t)gridDim.x * blockDim.x) {
        double s = __ddiv_rn(stren[c], two_m);
        terms[c] = __dsub_rn(__ddiv_rn(__dmul_rn(2.0, internal[c]), two_m),
                             __dmul_rn(gamma, __dmul_rn(s, s)));
    }
}
}  // namespace

// Ascending-rank ids of arbitrary u64 labels (device); returns the distinct count.
uint32_t renumber_u64_labels(Ctx& c, const uint64_t* d_labels, uint64_t n, uint32_t* d_out,
                             uint64_t* max_label_out) {
    if (n == 0) {
        if (max_label_out) *max_label_out = 0;
        return 0;
    }
    DBuf<uint64_t> ks(c, n);
    DBuf<uint32_t> idx(c, n), order(c, n), head(c, n), incl(c, n);
    k_iota32<<<grid_for(n, TB), TB, 0, c.stream>>>(idx.get(), n);
    SC_LAUNCH_CHECK();
    sort_pairs(c, d_labels, ks.get(), idx.get(), order.get(), n, 64);
    k_heads_u64<<<grid_for(n, TB), TB, 0, c.stream>>>(ks.get(), n, head.get());
    SC_LAUNCH_CHECK();
    inclusive_sum(c, head.get(), incl.get(), n);
    k_scatter_rank<<<grid_for(n, TB), TB, 0, c.stream>>>(order.get(), incl.get(), n, d_out);
    SC_LAUNCH_CHECK();
    c.launches += 3;
    if (max_label_out) *max_label_out = to_host(c, ks.get() + n - 1);
    return to_host(c, incl.get() + n - 1);
}

// Ascending-rank renumber of u32 ids in [0, id_space) (Partition::renumber,
// partition.rs:265-296): returns the number of distinct ids.
uint32_t renumber_ids(Ctx& c, const uint32_t* d_ids, uint64_t n, uint64_t id_space, uint32_t* d_out) {
    if (n == 0) return 0;
    DBuf<uint32_t> used(c, id_space + 1), rank(c, id_space + 1);
    zero(c, used.get(), id_space + 1);
    k_mark_used<<<grid_for(n, TB), TB, 0, c.stream>>>(d_ids, n, used.get());
    SC_LAUNCH_CHECK();
    exclusive_sum(c, used.get(), rank.get(), id_space + 1);
    k_apply_rank<<<grid_for(n, TB), TB, 0, c.stream>>>(d_ids, rank.get(), n, d_out);
    SC_LAUNCH_CHECK();
    c.launches += 2;
    return to_host(c, rank.get() + id_space);
}

// from_membership aggregates over compact ids d_memb in [0, C).
void partition_stats(Ctx& c, const DevGraph& g, const uint32_t* d_memb, uint64_t C, PartStats& out,
                     bool need_internal) {
    out.slots = C;
    out.size.alloc(c, C);
    out.weight.alloc(c, C);
    out.strength.alloc(c, C);
    out.internal.alloc(c, C);
    if (C == 0) return;
    const uint64_t n = g.n;
    zero(c, out.internal.get(), C);
    if (g.exact_w && g.exact_nw) {
        zero(c, out.size.get(), C);
        zero(c, out.weight.get(), C);
        zero(c, out.strength.get(), C);
        k_stats_nodes_atomic<<<grid_for(n, TB), TB, 0, c.stream>>>(
            d_memb, n, g.node_w, g.strength, out.size.get(), out.weight.get(), out.strength.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        if (need_internal && g.E) {
            k_internal_atomic<<<grid_for(g.E, TB), TB, 0, c.stream>>>(g.erow, g.nbr, g.w, g.E, d_memb,
                                                                      out.internal.get());
            SC_LAUNCH_CHECK();
            c.launches++;
        }
        return;
    }
    DBuf<uint32_t> idx(c, n), ms(c, n), members(c, n);
    DBuf<uint64_t> cstart(c, C + 1);
    k_iota32<<<grid_for(n, TB), TB, 0, c.stream>>>(idx.get(), n);
    SC_LAUNCH_CHECK();
    sort_pairs(c, d_memb, ms.get(), idx.get(), members.get(), n, bits_for(C));
    k_starts_u32<<<grid_for(n + 1, TB), TB, 0, c.stream>>>(ms.get(), n, C, cstart.get());
    SC_LAUNCH_CHECK();
    k_stats_ordered<<<grid_for(C * 32, 256), 256, 0, c.stream>>>(
        cstart.get(), members.get(), C, d_memb, g.ptr, g.nbr, g.w, g.node_w, g.strength,
        out.size.get(), out.weight.get(), out.strength.get(), out.internal.get(),
        need_internal ? 1 : 0);
    SC_LAUNCH_CHECK();
    c.launches += 3;
}

// Rb / Cpm quality of Partition::from_membership(graph, memb) over compact ids.
// Empty slots of the reference contribute +0.0 terms: they can only turn a
// -0.0 total into +0.0, which the sign fix below reproduces.
double quality(Ctx& c, const DevGraph& g, const uint32_t* d_memb, uint64_t C, int objective,
               double gamma) {
    double four_m = 4.0 * g.total_weight;
    if (objective == SC_OBJECTIVE_RB && four_m == 0.0) return 0.0;
    PartStats st;
    partition_stats(c, g, d_memb, C, st, true);
    DBuf<double> terms(c, C);
    if (C) {
        k_quality_terms<<<grid_for(C, TB), TB, 0, c.stream>>>(st.weight.get(), st.strength.get(),
                                                              st.internal.get(), C, objective, gamma,
                                                              four_m, terms.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    double q = ordered_sum(c, terms.get(), C);
    return q;
}

double modularity(Ctx& c, const DevGraph& g, const uint32_t* d_labels, uint64_t C, double gamma) {
    double m = g.total_weight;
    if (m == 0.0) return 0.0;
    PartStats st;
    partition_stats(c, g, d_labels, C, st, true);
    double two_m = 2.0 * m;
    DBuf<double> terms(c, C);
    if (C) {
        k_modularity_terms<<<grid_for(C, TB), TB, 0, c.stream>>>(st.strength.get(), st.internal.get(),
                                                                 C, gamma, two_m, terms.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    return ordered_sum(c, terms.get(), C);
}

}  // namespace sc
