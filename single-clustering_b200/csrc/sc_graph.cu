// sc_graph.cu — device construction of CSRNetwork (csr_network.rs) on sm_100a.
//
// Parity rule: every f64 sum is taken in the reference's order. Per-row sums
// (duplicate merge, strengths) run one thread per row in ascending neighbour
// order. Cross-row sums (total_weight, Σ strength, aggregate's per-pair
// accumulators) are either provably order-independent — every term is a
// multiple of 2^e0 and the grand total is below 2^(52+e0), so every partial
// sum is exact in f64 (the "exact regime") — or are taken by an ordered chain.
#include "sc_prims.cuh"

namespace sc {

namespace {

constexpr unsigned TB = 256;

// A graph array: from the device's default stream-ordered pool for the graphs
// of a running call, from the device's graph pool for graphs handed to the user
// (see DevGraph::pooled).
template <class T>
void palloc(Ctx& c, bool pooled, T** p, uint64_t count) {
    cudaError_t e = pooled ? cudaMallocAsync((void**)p, count * sizeof(T), c.stream)
                           : cudaMallocFromPoolAsync((void**)p, count * sizeof(T), user_graph_pool(c.device),
                                                     c.stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(SC_E_OUT_OF_MEMORY, "device allocation of %llu bytes failed",
             (unsigned long long)(count * sizeof(T)));
    }
    if (e != cudaSuccess) throw_cuda(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
}

// Frees an array palloc gave out, in the order of the context's stream.
void pfree(Ctx& c, bool /*pooled*/, void* p) {
    if (p) cudaFreeAsync(p, c.stream);
}

void galloc(Ctx& c, DevGraph& g, uint64_t n, uint64_t E) {
    SC_CUDA(cudaGetDevice(&g.device));
    g.n = n;
    g.E = E;
    palloc(c, g.pooled, &g.ptr, n + 1);
    if (E) {
        palloc(c, g.pooled, &g.nbr, E);
        palloc(c, g.pooled, &g.w, E);
        palloc(c, g.pooled, &g.erow, E);
    }
    if (n) {
        palloc(c, g.pooled, &g.node_w, n);
        palloc(c, g.pooled, &g.strength, n);
        palloc(c, g.pooled, &g.self_loop, n);
    }
}

// ------------------------------------------------------------ validation
__global__ void k_first_bad_ptr(const uint64_t* __restrict__ ptr, uint64_t n,
                                unsigned long long* first) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x)
        if (ptr[v] > ptr[v + 1]) atomicMin(first, (unsigned long long)v);
}

__global__ void k_first_bad_entry(const uint32_t* __restrict__ nbr, const float* __restrict__ w,
                                  uint64_t E, uint64_t n, unsigned long long* first) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        float x = w[e];
        if ((uint64_t)nbr[e] >= n || !isfinite(x) || x < 0.0f) atomicMin(first, (unsigned long long)e);
    }
}

__global__ void k_first_bad_nodew(const double* __restrict__ nw, uint64_t n,
                                  unsigned long long* first) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        double x = nw[v];
        if (!isfinite(x) || x < 0.0) atomicMin(first, (unsigned long long)v);
    }
}

__global__ void k_first_bad_edge(const uint64_t* __restrict__ from, const uint64_t* __restrict__ to,
                                 const double* __restrict__ w, uint64_t m, uint64_t n,
                                 unsigned long long* first) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        double x = w[i];
        if (from[i] >= n || to[i] >= n || !isfinite(x) || x < 0.0)
            atomicMin(first, (unsigned long long)i);
    }
}

__global__ void k_fill_double(double* p, uint64_t n, double v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void k_lowbit_f64(const double* __restrict__ x, uint64_t n, int* min_low) {
    int best = 0x7FFFFFFF;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        best = min(best, lowbit_exp_f64(x[i]));
    for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
    if ((threadIdx.x & 31) == 0 && best != 0x7FFFFFFF) atomicMin(min_low, best);
}

// ------------------------------------------------------------ row kernels
// One warp per row writes the row id over its entries (coalesced).
__global__ void k_fill_erow(const uint64_t* __restrict__ ptr, uint64_t n, uint32_t* erow) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = warp; v < n; v += nwarps) {
        uint64_t b = ptr[v], e = ptr[v + 1];
        for (uint64_t i = b + lane; i < e; i += 32) erow[i] = (uint32_t)v;
    }
}

// dirty = 1 if some row is not strictly increasing or holds a zero weight.
__global__ void k_rows_clean(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                             const float* __restrict__ w, const uint32_t* __restrict__ erow,
                             uint64_t E, int* dirty) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        bool bad = (w[e] == 0.0f);
        if (e > 0 && erow[e - 1] == erow[e] && nbr[e - 1] >= nbr[e]) bad = true;
        if (bad) *dirty = 1;
    }
}

__global__ void k_make_row_keys(const uint32_t* __restrict__ erow, const uint32_t* __restrict__ nbr,
                                uint64_t E, uint64_t* keys) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x)
        keys[e] = ((uint64_t)erow[e] << 32) | nbr[e];
}

// Rows sorted by neighbour id (duplicates in input order): per row, count the
// distinct ids whose f64 sum is non-zero (finish, csr_network.rs:295-306).
__global__ void k_merge_count(const uint64_t* __restrict__ ptr, const uint64_t* __restrict__ keys,
                              const float* __restrict__ w, uint64_t n, uint64_t* cnt) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = ptr[v], e = ptr[v + 1], c = 0;
        while (i < e) {
            uint32_t u = (uint32_t)keys[i];
            double acc = 0.0;
            while (i < e && (uint32_t)keys[i] == u) {
                acc = __dadd_rn(acc, (double)w[i]);
                ++i;
            }
            if (acc != 0.0) ++c;
        }
        cnt[v] = c;
    }
}

__global__ void k_merge_write(const uint64_t* __restrict__ ptr_in, const uint64_t* __restrict__ keys,
                              const float* __restrict__ w_in, uint64_t n,
                              const uint64_t* __restrict__ ptr_out, uint32_t* nbr_out, float* w_out) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t i = ptr_in[v], e = ptr_in[v + 1], o = ptr_out[v];
        while (i < e) {
            uint32_t u = (uint32_t)keys[i];
            double acc = 0.0;
            while (i < e && (uint32_t)keys[i] == u) {
                acc = __dadd_rn(acc, (double)w_in[i]);
                ++i;
            }
            if (acc == 0.0) continue;
            nbr_out[o] = u;
            w_out[o] = __double2float_rn(acc);
            ++o;
        }
    }
}

// Per row of a clean CSR, one warp per row: strength (self-loop twice,
// csr_network.rs:313-320), self-loop weight, lowest set bit of the stored
// weights, any self-loop, max degree, hub count.
__global__ void k_row_stats(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                            const float* __restrict__ w, uint64_t n, double* strength,
                            double* self_loop, int* min_low, unsigned* any_loop, unsigned* max_deg) {
    // One pass per row. The strengths are folded in any order here: exact (and
    // so equal to the reference's left fold) whenever the graph turns out to be
    // in the exact regime; otherwise finalize recomputes them in order.
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    int low = 0x7FFFFFFF;
    unsigned loop = 0, mdeg = 0, hubs = 0;
    for (uint64_t v = warp; v < n; v += nwarps) {
        const uint64_t b = ptr[v], e = ptr[v + 1];
        double sl = 0.0, acc = 0.0;
        for (uint64_t i = b + lane; i < e; i += 32) {
            const float x = w[i];
            low = min(low, lowbit_exp_f32(x));
            const double st = (double)x;
            if (nbr[i] == (uint32_t)v) {
                loop = 1;
                sl = st;
                acc = __dadd_rn(acc, __dmul_rn(2.0, st));
            } else {
                acc = __dadd_rn(acc, st);
            }
        }
        for (int o = 16; o; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xFFFFFFFFu, acc, o));
        // at most one lane saw the self-loop
        for (int o = 16; o; o >>= 1) sl = fmax(sl, __shfl_xor_sync(0xFFFFFFFFu, sl, o));
        if (lane == 0) {
            strength[v] = e > b ? __dadd_rn(0.0, acc) : 0.0;
            self_loop[v] = sl;
            mdeg = max(mdeg, (unsigned)(e - b));
            hubs += (e - b) > HUB_DEGREE;
        }
    }
    for (int o = 16; o; o >>= 1) {
        low = min(low, __shfl_xor_sync(0xFFFFFFFFu, low, o));
        loop |= __shfl_xor_sync(0xFFFFFFFFu, loop, o);
        mdeg = max(mdeg, __shfl_xor_sync(0xFFFFFFFFu, mdeg, o));
        hubs += __shfl_xor_sync(0xFFFFFFFFu, hubs, o);
    }
    if (lane == 0) {
        if (low != 0x7FFFFFFF) atomicMin(min_low, low);
        if (loop) atomicOr(any_loop, 1u);
        atomicMax(max_deg, mdeg);
        if (hubs) atomicAdd(any_loop + 2, hubs);
    }
}

// Strengths as the reference folds them (csr_network.rs:313-320): left to
// right over the row in ascending-neighbour order from 0.0, a self-loop
// counted twice. For graphs outside the exact regime.
__global__ void k_row_strength_ordered(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                                       const float* __restrict__ w, uint64_t n, double* strength) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = warp; v < n; v += nwarps) {
        const uint64_t b = ptr[v], e = ptr[v + 1];
        const double s = warp_ordered_sum(b, e, 0.0, [&](uint64_t i) {
            const double st = (double)w[i];
            return nbr[i] == (uint32_t)v ? __dmul_rn(2.0, st) : st;
        });
        if ((threadIdx.x & 31u) == 0) strength[v] = s;
    }
}

// total_weight terms: stored weight of entries with row <= neighbour, else 0.
__global__ void k_upper_terms(const uint32_t* __restrict__ erow, const uint32_t* __restrict__ nbr,
                              const float* __restrict__ w, uint64_t E, double* terms,
                              uint8_t* flags) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        bool up = erow[e] <= nbr[e];
        terms[e] = up ? (double)w[e] : 0.0;
        flags[e] = up ? 1 : 0;
    }
}

__global__ void k_u8_to_u64(const uint8_t* f, uint64_t n, uint64_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = f[i];
}

// CSR offsets from keys sorted by row: start[r] = first index with row >= r.
__global__ void k_starts_from_sorted(const uint32_t* __restrict__ rows, uint64_t N, uint64_t R,
                                     uint64_t* start) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = i < N ? rows[i] : R;
        uint64_t prev = i == 0 ? 0 : (uint64_t)rows[i - 1] + 1;
        if (i == 0) prev = 0;
        for (uint64_t q = prev; q <= r && q <= R; ++q) start[q] = i;
    }
}

// ------------------------------------------------------------ totals
struct Totals {
    double total_weight;
    uint64_t edge_count;
};

// Stats, regime, totals and check_degree_sum of a graph whose rows are clean.
// Every reduction that the exact regime can use is queued first and read back
// with one synchronisation; the ordered folds of the other regime follow only
// when the regime needs them.
//   total_weight (csr_network.rs:321-324): Σ over the v <= u entries of f64(w)
//   (self-loops once), in (v asc, u asc) order; edge_count: their number.
void finalize(Ctx& c, DevGraph& g, bool check_sum) {
    const uint64_t n = g.n, E = g.E;
    DBuf<int> d_low(c, 2);
    DBuf<unsigned> d_flags(c, 3);
    DBuf<double> d_sums(c, 3);  // Σ strength, Σ node weight, Σ upper-triangle terms
    DBuf<uint64_t> d_ecount(c, 1);
    int init_low[2] = {0x7FFFFFFF, 0x7FFFFFFF};
    h2d(c, d_low.get(), init_low, 2);
    zero(c, d_flags.get(), 3);
    zero(c, d_sums.get(), 3);
    zero(c, d_ecount.get(), 1);
    if (n) {
        k_row_stats<<<grid_for(n * 32, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, n, g.strength,
                                                          g.self_loop, d_low.get(), d_flags.get(),
                                                          d_flags.get() + 1);
        SC_LAUNCH_CHECK();
        k_lowbit_f64<<<grid_for(n, TB), TB, 0, c.stream>>>(g.node_w, n, d_low.get() + 1);
        SC_LAUNCH_CHECK();
        c.launches += 2;
        device_sum(c, g.strength, d_sums.get(), n);
        device_sum(c, g.node_w, d_sums.get() + 1, n);
    }
    DBuf<double> terms;
    DBuf<uint8_t> upper;
    if (E) {
        terms.alloc(c, E);
        upper.alloc(c, E);
        k_upper_terms<<<grid_for(E, TB), TB, 0, c.stream>>>(g.erow, g.nbr, g.w, E, terms.get(), upper.get());
        SC_LAUNCH_CHECK();
        DBuf<uint64_t> f64s(c, E);
        k_u8_to_u64<<<grid_for(E, TB), TB, 0, c.stream>>>(upper.get(), E, f64s.get());
        c.launches += 2;
        device_sum(c, f64s.get(), d_ecount.get(), E);
        device_sum(c, terms.get(), d_sums.get() + 2, E);  // exact in the exact regime; unused otherwise
    }
    int low[2];
    unsigned flags[3];
    double sums[3];
    uint64_t ecount;
    {
        Mailbox mb(c);
        const int* hl = mb.get(d_low.get(), 2);
        const unsigned* hf = mb.get(d_flags.get(), 3);
        const double* hs = mb.get(d_sums.get(), 3);
        const uint64_t* he = mb.get(d_ecount.get(), 1);
        mb.wait();
        std::memcpy(low, hl, sizeof low);
        std::memcpy(flags, hf, sizeof flags);
        std::memcpy(sums, hs, sizeof sums);
        ecount = *he;
    }
    g.any_self_loops = flags[0] != 0;
    g.max_degree = flags[1];
    g.n_hubs = flags[2];
    g.e0_w = low[0];
    g.e0_nw = low[1];

    // approximate Σ strength (= 2m) decides the regime; exact inside it
    const double approx2m = n ? sums[0] : 0.0;
    const double regime2m = g.part_max_2m > 0.0 ? g.part_max_2m : approx2m;
    g.exact_w = (g.e0_w == 0x7FFFFFFF) || (regime2m < std::ldexp(1.0, 52 + g.e0_w));
    const double approx_nw = n ? sums[1] : 0.0;
    const double regime_nw = g.part_max_nw > 0.0 ? g.part_max_nw : approx_nw;
    g.exact_nw = (g.e0_nw == 0x7FFFFFFF) || (regime_nw < std::ldexp(1.0, 52 + g.e0_nw));
    // Rust-order Σ of the node weights (a fold from -0.0): in the exact regime any
    // order gives these bits, and n > 0 terms >= +0.0 never leave the -0.0 start
    if (n && !g.exact_w) {  // the strengths in the reference's order
        k_row_strength_ordered<<<grid_for(n * 32, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, n, g.strength);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    if (n == 0) g.total_node_weight = -0.0;
    else g.total_node_weight = g.exact_nw ? approx_nw : ordered_sum(c, g.node_w, n);

    g.edge_count = E ? ecount : 0;
    if (E == 0) {
        g.total_weight = 0.0;
    } else if (g.exact_w) {
        g.total_weight = sums[2];
    } else {
        DBuf<double> up(c, E);
        DBuf<uint64_t> nup(c, 1);
        select_flagged(c, terms.get(), upper.get(), up.get(), nup.get(), E);
        const uint64_t k = to_host(c, nup.get());
        g.total_weight = ordered_sum_from(c, up.get(), k, 0.0);
    }

    if (check_sum) {
        // check_degree_sum (csr_network.rs:712-723)
        double expected = 2.0 * g.total_weight;
        double tol = 1e-6 * std::max(std::fabs(expected), 1.0);
        double sum = g.exact_w ? (n ? approx2m : -0.0) : approx2m;
        if (!g.exact_w && std::fabs(sum - expected) > 0.25 * tol) sum = n ? ordered_sum(c, g.strength, n) : -0.0;
        if (std::fabs(sum - expected) > tol) {
            sc_error_info i{};
            i.code = SC_E_ASYMMETRIC_GRAPH;
            i.degree_sum = sum;
            i.expected = expected;
            fail_info(i);
        }
    }
}

// finish (csr_network.rs:262-351) on validated device arrays the graph owns.
void finish(Ctx& c, DevGraph& g) {
    const uint64_t n = g.n;
    if (g.E) {
        k_fill_erow<<<grid_for(n * 32, TB), TB, 0, c.stream>>>(g.ptr, n, g.erow);
        SC_LAUNCH_CHECK();
        c.launches++;
        DBuf<int> dirty(c, 1);
        zero(c, dirty.get(), 1);
        k_rows_clean<<<grid_for(g.E, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, g.erow, g.E,
                                                             dirty.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        if (to_host(c, dirty.get())) {
            // stable sort of every entry by (row, neighbour): duplicates keep input order
            DBuf<uint64_t> keys(c, g.E), keys_s(c, g.E);
            DBuf<float> w_s(c, g.E);
            k_make_row_keys<<<grid_for(g.E, TB), TB, 0, c.stream>>>(g.erow, g.nbr, g.E, keys.get());
            SC_LAUNCH_CHECK();
            c.launches++;
            sort_pairs(c, keys.get(), keys_s.get(), g.w, w_s.get(), g.E, 32 + bits_for(n));
            DBuf<uint64_t> cnt(c, n + 1), nptr(c, n + 1);
            k_merge_count<<<grid_for(n, TB), TB, 0, c.stream>>>(g.ptr, keys_s.get(), w_s.get(), n,
                                                                cnt.get());
            SC_LAUNCH_CHECK();
            zero(c, cnt.get() + n, 1);
            exclusive_sum(c, cnt.get(), nptr.get(), n + 1);
            uint64_t E2 = to_host(c, nptr.get() + n);
            uint32_t* nbr2 = nullptr;
            float* w2 = nullptr;
            uint32_t* erow2 = nullptr;
            if (E2) {
                palloc(c, g.pooled, &nbr2, E2);
                palloc(c, g.pooled, &w2, E2);
                palloc(c, g.pooled, &erow2, E2);
            }
            k_merge_write<<<grid_for(n, TB), TB, 0, c.stream>>>(g.ptr, keys_s.get(), w_s.get(), n,
                                                                nptr.get(), nbr2, w2);
            SC_LAUNCH_CHECK();
            c.launches += 2;
            d2d(c, g.ptr, nptr.get(), n + 1);
            pfree(c, g.pooled, g.nbr);
            pfree(c, g.pooled, g.w);
            pfree(c, g.pooled, g.erow);
            g.nbr = nbr2;
            g.w = w2;
            g.erow = erow2;
            g.E = E2;
            if (E2) {
                k_fill_erow<<<grid_for(n * 32, TB), TB, 0, c.stream>>>(g.ptr, n, g.erow);
                SC_LAUNCH_CHECK();
                c.launches++;
            }
        }
    }
    finalize(c, g, true);
}

uint64_t first_bad(Ctx& c, DBuf<unsigned long long>& d) {
    unsigned long long v = to_host(c, d.get());
    return (uint64_t)v;
}

}  // namespace

// from_csr_parts (csr_network.rs:185-256)
DevGraph* graph_from_csr(Ctx& c, const uint64_t* ptr, uint64_t n_ptr, const uint32_t* nbr,
                         uint64_t n_nbr, const float* w, uint64_t n_w, const double* node_w,
                         uint64_t n_node_w, bool device_inputs) {
    if (n_ptr == 0)
        fail(SC_E_INVALID_CSR, "malformed CSR input: node_ptrs must have at least one element");
    const uint64_t n = n_ptr - 1;
    if (n > MAX_NODES) {
        sc_error_info i{};
        i.code = SC_E_TOO_MANY_NODES;
        i.n_nodes = n;
        fail_info(i);
    }
    if (n_nbr != n_w)
        fail(SC_E_INVALID_CSR, "malformed CSR input: neighbors has %llu entries but weights has %llu",
             (unsigned long long)n_nbr, (unsigned long long)n_w);
    const cudaMemcpyKind kind = device_inputs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    std::unique_ptr<DevGraph> g(new DevGraph());
    g->pooled = false;  // the user's graph keeps out of the pool a run's temporaries cycle through
    galloc(c, *g, n, n_nbr);
    auto copy_in = [&](void* dst, const void* src, size_t bytes) {
        if (kind == cudaMemcpyHostToDevice) upload(c, dst, src, bytes);
        else if (bytes) SC_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, c.stream));
    };
    copy_in(g->ptr, ptr, n_ptr * sizeof(uint64_t));
    if (n_nbr) {
        copy_in(g->nbr, nbr, n_nbr * sizeof(uint32_t));
        copy_in(g->w, w, n_nbr * sizeof(float));
    }
    uint64_t last = to_host(c, g->ptr + n);
    if (last != n_nbr)
        fail(SC_E_INVALID_CSR, "malformed CSR input: node_ptrs ends at %llu but there are %llu entries",
             (unsigned long long)last, (unsigned long long)n_nbr);
    DBuf<unsigned long long> first(c, 1);
    const unsigned long long NOBAD = ~0ull;
    if (n) {
        h2d(c, first.get(), &NOBAD, 1);
        k_first_bad_ptr<<<grid_for(n, TB), TB, 0, c.stream>>>(g->ptr, n, first.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        uint64_t v = first_bad(c, first);
        if (v != NOBAD)
            fail(SC_E_INVALID_CSR, "malformed CSR input: node_ptrs is not non-decreasing at %llu",
                 (unsigned long long)v);
    }
    if (n_nbr) {
        h2d(c, first.get(), &NOBAD, 1);
        k_first_bad_entry<<<grid_for(n_nbr, TB), TB, 0, c.stream>>>(g->nbr, g->w, n_nbr, n,
                                                                    first.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        uint64_t e = first_bad(c, first);
        if (e != NOBAD) {
            uint32_t u;
            float x;
            d2h(c, &u, g->nbr + e, 1);
            d2h(c, &x, g->w + e, 1);
            sync(c);
            sc_error_info i{};
            if ((uint64_t)u >= n) {
                i.code = SC_E_NODE_INDEX_OUT_OF_RANGE;
                i.node = u;
                i.n_nodes = n;
            } else if (!std::isfinite(x)) {
                i.code = SC_E_NON_FINITE_WEIGHT;
                i.edge_from = 0;
                i.edge_to = u;
            } else {
                i.code = SC_E_NEGATIVE_WEIGHT;
                i.edge_from = 0;
                i.edge_to = u;
                i.weight = (double)x;
            }
            fail_info(i);
        }
    }
    if (node_w) {
        if (n_node_w != n) {
            sc_error_info i{};
            i.code = SC_E_NODE_WEIGHT_LENGTH_MISMATCH;
            i.got = n_node_w;
            i.expected_len = n;
            fail_info(i);
        }
        copy_in(g->node_w, node_w, n * sizeof(double));
        if (n) {
            h2d(c, first.get(), &NOBAD, 1);
            k_first_bad_nodew<<<grid_for(n, TB), TB, 0, c.stream>>>(g->node_w, n, first.get());
            SC_LAUNCH_CHECK();
            c.launches++;
            uint64_t v = first_bad(c, first);
            if (v != NOBAD) {
                sc_error_info i{};
                i.code = SC_E_INVALID_NODE_WEIGHT;
                i.node = v;
                d2h(c, &i.weight, g->node_w + v, 1);
                sync(c);
                fail_info(i);
            }
        }
    } else if (n) {
        k_fill_double<<<grid_for(n, TB), TB, 0, c.stream>>>(g->node_w, n, 1.0);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    finish(c, *g);
    sync(c);
    return g.release();
}

namespace {
// Expands edge i into slots 2i (from,to) and 2i+1 (to,from); loops use one slot.
__global__ void k_expand_edges(const uint64_t* __restrict__ from, const uint64_t* __restrict__ to,
                               const double* __restrict__ w, uint64_t m, uint64_t* keys, float* ws) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t a = from[i], b = to[i];
        float x = __double2float_rn(w[i]);
        keys[2 * i] = (a << 32) | b;
        ws[2 * i] = x;
        keys[2 * i + 1] = a == b ? ~0ull : ((b << 32) | a);
        ws[2 * i + 1] = x;
    }
}

__global__ void k_split_keys(const uint64_t* __restrict__ keys, uint64_t N, uint32_t* rows,
                             uint32_t* cols) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        rows[i] = (uint32_t)(keys[i] >> 32);
        cols[i] = (uint32_t)keys[i];
    }
}
}  // namespace

// from_edges_with_node_weights (csr_network.rs:120-167)
DevGraph* graph_from_edges(Ctx& c, uint64_t n, const uint64_t* from, const uint64_t* to,
                           const double* w, uint64_t m, const double* node_w) {
    std::unique_ptr<DevGraph> g(new DevGraph());
    g->pooled = false;
    DBuf<unsigned long long> first(c, 1);
    const unsigned long long NOBAD = ~0ull;
    if (n > MAX_NODES) {
        // validate_node_weights runs first (csr_network.rs:128-131)
        for (uint64_t v = 0; node_w && v < n; ++v) {
            if (!std::isfinite(node_w[v]) || node_w[v] < 0.0) {
                sc_error_info i{};
                i.code = SC_E_INVALID_NODE_WEIGHT;
                i.node = v;
                i.weight = node_w[v];
                fail_info(i);
            }
        }
        sc_error_info i{};
        i.code = SC_E_TOO_MANY_NODES;
        i.n_nodes = n;
        fail_info(i);
    }
    DBuf<double> nw(c, n);
    if (node_w) {
        h2d(c, nw.get(), node_w, n);
        if (n) {
            h2d(c, first.get(), &NOBAD, 1);
            k_first_bad_nodew<<<grid_for(n, TB), TB, 0, c.stream>>>(nw.get(), n, first.get());
            SC_LAUNCH_CHECK();
            c.launches++;
            uint64_t v = first_bad(c, first);
            if (v != NOBAD) {
                sc_error_info i{};
                i.code = SC_E_INVALID_NODE_WEIGHT;
                i.node = v;
                i.weight = node_w[v];
                fail_info(i);
            }
        }
    } else if (n) {
        k_fill_double<<<grid_for(n, TB), TB, 0, c.stream>>>(nw.get(), n, 1.0);
        c.launches++;
    }
    DBuf<uint64_t> df(c, m), dt(c, m);
    DBuf<double> dw(c, m);
    h2d(c, df.get(), from, m);
    h2d(c, dt.get(), to, m);
    h2d(c, dw.get(), w, m);
    if (m) {
        h2d(c, first.get(), &NOBAD, 1);
        k_first_bad_edge<<<grid_for(m, TB), TB, 0, c.stream>>>(df.get(), dt.get(), dw.get(), m, n,
                                                               first.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        uint64_t i0 = first_bad(c, first);
        if (i0 != NOBAD) {
            sc_error_info i{};
            uint64_t a = from[i0], b = to[i0];
            double x = w[i0];
            if (a >= n) {
                i.code = SC_E_NODE_INDEX_OUT_OF_RANGE;
                i.node = a;
                i.n_nodes = n;
            } else if (b >= n) {
                i.code = SC_E_NODE_INDEX_OUT_OF_RANGE;
                i.node = b;
                i.n_nodes = n;
            } else if (!std::isfinite(x)) {
                i.code = SC_E_NON_FINITE_WEIGHT;
                i.edge_from = a;
                i.edge_to = b;
            } else {
                i.code = SC_E_NEGATIVE_WEIGHT;
                i.edge_from = a;
                i.edge_to = b;
                i.weight = x;
            }
            fail_info(i);
        }
    }
    // scatter into both rows in edge order, then a stable sort by (row, neighbour)
    DBuf<uint64_t> keys(c, 2 * m), keys_s(c, 2 * m);
    DBuf<float> ws(c, 2 * m), ws_s(c, 2 * m);
    if (m) {
        k_expand_edges<<<grid_for(m, TB), TB, 0, c.stream>>>(df.get(), dt.get(), dw.get(), m,
                                                             keys.get(), ws.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        sort_pairs(c, keys.get(), keys_s.get(), ws.get(), ws_s.get(), 2 * m, 64);
    }
    // entries with key ~0 (the unused slots of self-loops) sort to the end
    uint64_t loops_slots = 0;
    for (uint64_t i = 0; i < m; ++i) loops_slots += from[i] == to[i];
    const uint64_t E = 2 * m - loops_slots;
    galloc(c, *g, n, E);
    d2d(c, g->node_w, nw.get(), n);
    if (E) {
        k_split_keys<<<grid_for(E, TB), TB, 0, c.stream>>>(keys_s.get(), E, g->erow, g->nbr);
        SC_LAUNCH_CHECK();
        d2d(c, g->w, ws_s.get(), E);
        k_starts_from_sorted<<<grid_for(E + 1, TB), TB, 0, c.stream>>>(g->erow, E, n, g->ptr);
        SC_LAUNCH_CHECK();
        c.launches += 2;
    } else {
        zero(c, g->ptr, n + 1);
    }
    finish(c, *g);
    sync(c);
    return g.release();
}

// ------------------------------------------------------------ aggregate
namespace {

__global__ void k_iota(uint32_t* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

// Per group, in ascending member order, one warp per group: Σ node weight
// (csr_network.rs:520-523) and Σ self-loop weight (the `self_loop_weight`
// accumulator of :549-554; members without a loop add +0.0, a no-op).
__global__ void k_group_sums(const uint64_t* __restrict__ gstart, const uint32_t* __restrict__ members,
                             uint64_t G, const double* __restrict__ node_w,
                             const double* __restrict__ self_loop, double* nw_out, double* loops_out,
                             int exact_nw, int exact_w) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t gi = warp; gi < G; gi += nwarps) {
        const uint64_t b = gstart[gi], e = gstart[gi + 1];
        const double a = warp_fold(b, e, 0.0, exact_nw, [&](uint64_t i) { return node_w[members[i]]; });
        const double l = warp_fold(b, e, 0.0, exact_w, [&](uint64_t i) { return self_loop[members[i]]; });
        if ((threadIdx.x & 31) == 0) {
            nw_out[gi] = a;
            loops_out[gi] = l;
        }
    }
}

// Entries whose neighbour's group is >= the row's group, keyed by (g, h).
__global__ void k_group_keys(const uint32_t* __restrict__ erow, const uint32_t* __restrict__ nbr,
                             const uint32_t* __restrict__ grp, uint64_t E, uint64_t G,
                             uint64_t* keys, uint8_t* flags) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t g = grp[erow[e]], h = grp[nbr[e]];
        keys[e] = g * G + h;
        flags[e] = h >= g;
    }
}

__global__ void k_seg_heads(const uint64_t* __restrict__ keys, uint64_t N, uint8_t* head) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void k_iota64(uint64_t* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = i;
}

// The (g, h) segments, 32 per warp: acc in (member asc, neighbour asc) order,
// the reference's left fold — a lane folds a short segment alone, the warp
// folds a long one together (warp_fold); then the pair rule of
// csr_network.rs:566-581 and finish's zero drop (:304).
__device__ __forceinline__ void seg_emit(uint64_t s, uint64_t b, double acc, const uint64_t* __restrict__ keys,
                                         uint64_t G, const double* __restrict__ loops, uint32_t* prow,
                                         uint32_t* pcol, float* pw, uint8_t* keep) {
    const uint64_t key = keys[b];
    const uint32_t g = (uint32_t)(key / G), h = (uint32_t)(key % G);
    float val;
    if (h == g) val = __double2float_rn(__dmul_rn(0.5, __dadd_rn(acc, loops[g])));
    else val = __double2float_rn(acc);
    prow[s] = g;
    pcol[s] = h;
    pw[s] = val;
    keep[s] = (acc > 0.0) && ((double)val != 0.0);
}

// Segments at least SEG_BLOCK long, in the exact regime, are summed in chunks
// by many blocks (k_seg_long_partial): any order gives the exact sum, and one
// warp folding a segment of a coarse community's internal entries alone takes
// milliseconds.
constexpr uint64_t SEG_BLOCK = 4096;

__global__ void k_seg_values(const uint64_t* __restrict__ seg_start, uint64_t P, uint64_t N,
                             const uint64_t* __restrict__ keys, const float* __restrict__ w,
                             uint64_t G, const double* __restrict__ loops, uint32_t* prow,
                             uint32_t* pcol, float* pw, uint8_t* keep, int exact, uint32_t* long_list,
                             uint32_t* long_count, uint32_t long_cap) {
    constexpr uint64_t SHORT = 64;
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = warp * 32; base < P; base += nwarps * 32) {
        const uint64_t s = base + lane;
        uint64_t b = 0, e = 0;
        if (s < P) {
            b = seg_start[s];
            e = s + 1 < P ? seg_start[s + 1] : N;
        }
        const bool mine = s < P && e - b <= SHORT;
        if (mine) {
            double acc = 0.0;
            for (uint64_t i = b; i < e; ++i) acc = __dadd_rn(acc, (double)w[i]);
            seg_emit(s, b, acc, keys, G, loops, prow, pcol, pw, keep);
        }
        unsigned long_mask = __ballot_sync(0xFFFFFFFFu, s < P && !mine);
        while (long_mask) {
            const int src = __ffs(long_mask) - 1;
            long_mask &= long_mask - 1;
            const uint64_t bb = __shfl_sync(0xFFFFFFFFu, b, src), ee = __shfl_sync(0xFFFFFFFFu, e, src);
            if (exact && ee - bb >= SEG_BLOCK && long_list) {  // warp-uniform
                if ((int)lane == src) {
                    const uint32_t i = atomicAdd(long_count, 1u);
                    if (i < long_cap) long_list[i] = (uint32_t)s;
                }
                continue;
            }
            const double acc = warp_fold(bb, ee, 0.0, exact, [&](uint64_t i) { return (double)w[i]; });
            if ((int)lane == src) seg_emit(s, b, acc, keys, G, loops, prow, pcol, pw, keep);
        }
    }
}

// Long segments (exact regime) in chunks of SEG_CHUNK entries spread over all
// blocks: chunk ch of listed segment li goes to block (li + ch) mod gridDim, so
// one segment of a coarse community's internal entries (hundreds of thousands
// of them) keeps the whole GPU busy instead of one block. Every partial sum is
// exact, so the atomic accumulation gives the same bits in any order.
constexpr uint64_t SEG_CHUNK = 8192;

__global__ void __launch_bounds__(256) k_seg_long_partial(const uint32_t* __restrict__ long_list,
                                                          const uint32_t* __restrict__ long_count,
                                                          uint32_t long_cap, const uint64_t* __restrict__ seg_start,
                                                          uint64_t P, uint64_t N, const float* __restrict__ w,
                                                          double* part) {
    __shared__ double red[8];
    const uint32_t cnt = min(*long_count, long_cap);
    for (uint32_t li = 0; li < cnt; ++li) {
        const uint32_t s = long_list[li];
        const uint64_t b = seg_start[s], e = s + 1 < P ? seg_start[s + 1] : N;
        const uint64_t nch = (e - b + SEG_CHUNK - 1) / SEG_CHUNK;
        uint64_t ch = (blockIdx.x + gridDim.x - (li % gridDim.x)) % gridDim.x;
        for (; ch < nch; ch += gridDim.x) {
            const uint64_t cb = b + ch * SEG_CHUNK, ce = cb + SEG_CHUNK < e ? cb + SEG_CHUNK : e;
            double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;  // four loads in flight per thread
            uint64_t i = cb + threadIdx.x;
            for (; i + 3 * blockDim.x < ce; i += 4 * blockDim.x) {
                a0 += (double)w[i];
                a1 += (double)w[i + blockDim.x];
                a2 += (double)w[i + 2 * blockDim.x];
                a3 += (double)w[i + 3 * blockDim.x];
            }
            for (; i < ce; i += blockDim.x) a0 += (double)w[i];
            double acc = (a0 + a1) + (a2 + a3);
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (unsigned k = 0; k < (blockDim.x >> 5); ++k) t += red[k];
                atomicAdd(part + li, t);
            }
            __syncthreads();
        }
    }
}

// The emission of every listed long segment from its accumulated sum.
__global__ void k_seg_long_emit(const uint32_t* __restrict__ long_list, const uint32_t* __restrict__ long_count,
                                uint32_t long_cap, const uint64_t* __restrict__ seg_start,
                                const double* __restrict__ part, const uint64_t* __restrict__ keys, uint64_t G,
                                const double* __restrict__ loops, uint32_t* prow, uint32_t* pcol, float* pw,
                                uint8_t* keep) {
    const uint32_t cnt = min(*long_count, long_cap);
    for (uint32_t li = blockIdx.x * blockDim.x + threadIdx.x; li < cnt; li += gridDim.x * blockDim.x) {
        const uint32_t s = long_list[li];
        seg_emit(s, seg_start[s], part[li], keys, G, loops, prow, pcol, pw, keep);
    }
}

// The (g, h) segments of keys sorted by (g, h) (values beside them) summed and
// emitted (seg_emit's rule): prow/pcol/pw/keep of P segments, P returned.
uint64_t segment_sums(Ctx& c, const uint64_t* keys_s, const float* w_s, uint64_t N, uint64_t G,
                      const double* loops, bool exact, DBuf<uint32_t>& prow, DBuf<uint32_t>& pcol,
                      DBuf<float>& pw, DBuf<uint8_t>& keep) {
    if (N == 0) return 0;
    DBuf<uint8_t> head(c, N);
    k_seg_heads<<<grid_for(N, TB), TB, 0, c.stream>>>(keys_s, N, head.get());
    DBuf<uint64_t> iota(c, N), seg(c, N), cnt(c, 1);
    k_iota64<<<grid_for(N, TB), TB, 0, c.stream>>>(iota.get(), N);
    SC_LAUNCH_CHECK();
    c.launches += 2;
    select_flagged(c, iota.get(), head.get(), seg.get(), cnt.get(), N);
    const uint64_t P = to_host(c, cnt.get());
    prow.alloc(c, P);
    pcol.alloc(c, P);
    pw.alloc(c, P);
    keep.alloc(c, P);
    const uint32_t long_cap = (uint32_t)(N / SEG_BLOCK + 1);
    DBuf<uint32_t> long_list(c, long_cap), long_count(c, 1);
    zero(c, long_count.get(), 1);
    k_seg_values<<<grid_for(P, TB), TB, 0, c.stream>>>(seg.get(), P, N, keys_s, w_s, G, loops, prow.get(),
                                                       pcol.get(), pw.get(), keep.get(), (int)exact,
                                                       long_list.get(), long_count.get(), long_cap);
    SC_LAUNCH_CHECK();
    c.launches++;
    if (exact) {
        DBuf<double> part(c, long_cap);
        zero(c, part.get(), long_cap);
        const unsigned pgrid = (unsigned)std::min<uint64_t>(N / SEG_CHUNK + 1, (uint64_t)c.sm_count * 4);
        k_seg_long_partial<<<pgrid, TB, 0, c.stream>>>(long_list.get(), long_count.get(), long_cap, seg.get(), P, N,
                                                       w_s, part.get());
        k_seg_long_emit<<<grid_for(long_cap, TB), TB, 0, c.stream>>>(long_list.get(), long_count.get(), long_cap,
                                                                     seg.get(), part.get(), keys_s, G, loops,
                                                                     prow.get(), pcol.get(), pw.get(), keep.get());
        SC_LAUNCH_CHECK();
        c.launches += 2;
    }
    return P;
}

// Mirror keys (h, g) of the kept off-diagonal pairs.
__global__ void k_mirror(const uint32_t* __restrict__ prow, const uint32_t* __restrict__ pcol,
                         const float* __restrict__ pw, uint64_t P, uint64_t G, uint64_t* mkeys,
                         float* mw, uint8_t* mflag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < P;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t g = prow[i], h = pcol[i];
        mkeys[i] = h * G + g;
        mw[i] = pw[i];
        mflag[i] = h != g;
    }
}

__global__ void k_key_rows(const uint64_t* __restrict__ keys, uint64_t N, uint64_t G, uint32_t* rows,
                           uint32_t* cols) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        rows[i] = (uint32_t)(keys[i] / G);
        cols[i] = (uint32_t)(keys[i] % G);
    }
}

__global__ void k_row_counts(const uint64_t* __restrict__ ls, const uint64_t* __restrict__ us,
                             uint64_t G, uint64_t* cnt) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < G;
         r += (uint64_t)gridDim.x * blockDim.x)
        cnt[r] = (ls[r + 1] - ls[r]) + (us[r + 1] - us[r]);
}

// Row r of the coarse CSR: its lower pairs (ascending g < r) then its diagonal
// and upper pairs (ascending h >= r) — already the order finish sorts to.
__global__ void k_row_assemble(const uint64_t* __restrict__ ptr, const uint64_t* __restrict__ ls,
                               const uint32_t* __restrict__ lcol, const float* __restrict__ lw,
                               const uint64_t* __restrict__ us, const uint32_t* __restrict__ ucol,
                               const float* __restrict__ uw, uint64_t G, uint32_t* nbr, float* w) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < G; r += nw) {
        uint64_t o = ptr[r];
        uint64_t l0 = ls[r], l1 = ls[r + 1], u0 = us[r], u1 = us[r + 1];
        for (uint64_t i = l0 + lane; i < l1; i += 32) {
            nbr[o + (i - l0)] = lcol[i];
            w[o + (i - l0)] = lw[i];
        }
        o += l1 - l0;
        for (uint64_t i = u0 + lane; i < u1; i += 32) {
            nbr[o + (i - u0)] = ucol[i];
            w[o + (i - u0)] = uw[i];
        }
    }
}

}  // namespace

// aggregate (csr_network.rs:516-608): d_grp holds ids already normalised to [0, G).
// ------------------------------------------------------------ aggregate, exact regime
// In the exact regime every (g, h) accumulator of aggregate (csr_network.rs:
// 516-608) is a subset sum of stored weights and exact in f64 whatever the
// order. On a graph whose stored weights are bitwise symmetric, the (h, g)
// value the reference mirrors from row h's upper part equals row g's own sum
// over its members' entries into h. So each coarse row is built from its own
// members: a hash of h -> sum per row (a warp per row up to AGG_WARP_CAP
// member entries, a block per larger row with the table in global memory),
// then the kept entries in ascending h. Same values, same order, no global
// sort of the E entries.
namespace {

constexpr uint64_t AGG_WARP_CAP = 256;
constexpr int AGG_WARPS = 4;
constexpr uint32_t AGG_EMPTY = 0xFFFFFFFFu;

// Whether every stored entry (v, u, w) has its mirror (u, v) with the same bits.
// Rows hold distinct neighbours, so mapping every upper entry (v, u > v) to its
// mirror (u, v) is one-to-one; when each mirror exists with the same bits and
// the upper and lower entries are equally many, every lower entry is some upper
// entry's mirror. So only the upper entries are searched, and the two counts
// compared afterwards (counts[0] upper, counts[1] lower).
__global__ void k_symmetric_bits(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                                 const float* __restrict__ w, const uint32_t* __restrict__ erow, uint64_t E,
                                 unsigned* bad, unsigned long long* counts) {
    unsigned long long up = 0, down = 0;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = erow[e], u = nbr[e];
        if (u < v) ++down;
        if (u <= v) continue;
        ++up;
        uint64_t lo = ptr[u], hi = ptr[u + 1];
        const uint64_t end = hi;
        while (lo < hi) {
            const uint64_t mid = (lo + hi) >> 1;
            if (nbr[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        if (!(lo < end && nbr[lo] == v && __float_as_uint(w[lo]) == __float_as_uint(w[e]))) *bad = 1u;
    }
    for (int o = 16; o; o >>= 1) {
        up += __shfl_xor_sync(0xFFFFFFFFu, up, o);
        down += __shfl_xor_sync(0xFFFFFFFFu, down, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        if (up) atomicAdd(counts, up);
        if (down) atomicAdd(counts + 1, down);
    }
}

// cap[g] = stored entries of g's members (an upper bound on its coarse row).
__global__ void k_row_caps(const uint64_t* __restrict__ gstart, const uint32_t* __restrict__ members, uint64_t G,
                           const uint64_t* __restrict__ ptr, uint64_t* cap) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = warp; g < G; g += nwarps) {
        uint64_t s = 0;
        for (uint64_t i = gstart[g] + lane; i < gstart[g + 1]; i += 32) {
            const uint32_t v = members[i];
            s += ptr[v + 1] - ptr[v];
        }
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
        if (lane == 0) cap[g] = s;
    }
}

__device__ __forceinline__ uint32_t agg_hash(uint32_t h) { return h * 0x9E3779B1u; }

// Adds x to h's slot of an open-addressing table of `size` slots (size > the
// number of distinct keys, so a free slot always exists; the probe count is
// bounded all the same).
__device__ __forceinline__ void agg_insert(uint32_t* keys, double* vals, uint64_t size, uint32_t h, double x,
                                           uint32_t* status) {
    uint64_t s = agg_hash(h) % size;
    for (uint64_t probe = 0; probe < size; ++probe) {
        const uint32_t prev = atomicCAS(keys + s, AGG_EMPTY, h);
        if (prev == AGG_EMPTY || prev == h) {
            atomicAdd(vals + s, x);
            return;
        }
        s = s + 1 == size ? 0 : s + 1;
    }
    atomicOr(status, DEV_OVERFLOW);
}

// Value and keep flag of the (g, h) entry (seg_emit's rule).
__device__ __forceinline__ float agg_value(uint32_t g, uint32_t h, double acc, const double* __restrict__ loops,
                                           bool* keep) {
    const float val = h == g ? __double2float_rn(__dmul_rn(0.5, __dadd_rn(acc, loops[g]))) : __double2float_rn(acc);
    *keep = acc > 0.0 && (double)val != 0.0;
    return val;
}

// The member entries of one group, flattened across the 32 lanes: calls
// f(j, valid) for every stored entry j of every member, in no particular
// order; every lane calls it the same number of times (valid false past the
// end), so f may use warp-collective operations.
template <class F>
__device__ __forceinline__ void warp_member_entries(const uint64_t* __restrict__ ptr,
                                                    const uint32_t* __restrict__ members, uint64_t m0, uint64_t m1,
                                                    F&& f) {
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    for (uint64_t mb = m0; mb < m1; mb += 32) {
        const uint64_t mi = mb + lane;
        uint64_t b = 0, d = 0;
        if (mi < m1) {
            const uint32_t v = members[mi];
            b = ptr[v];
            d = ptr[v + 1] - b;
        }
        uint64_t incl = d;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        const uint64_t excl = incl - d;
        const uint64_t total = __shfl_sync(FULL, incl, 31);
        for (uint64_t base = 0; base < total; base += 32) {
            const uint64_t t = base + lane;
            int L = 0;
            for (int step = 16; step; step >>= 1) {
                const uint64_t e = __shfl_sync(FULL, excl, L + step);
                if (e <= t) L += step;
            }
            const uint64_t eL = __shfl_sync(FULL, excl, L), bL = __shfl_sync(FULL, b, L);
            f(bL + (t - eL), t < total);
        }
    }
}

// The member entries of one group flattened across the whole block: members
// in chunks of blockDim, a block-wide prefix of their degrees in shared memory,
// every thread takes entries t, t + blockDim, ... and finds its member by binary
// search. f(j, valid, flat) is called by every thread of the block the same
// number of times (valid false past the end), so f may use warp-collective
// operations; flat numbers the group's entries 0, 1, ... in member order.
template <class F>
__device__ __forceinline__ void block_member_entries_at(const uint64_t* __restrict__ ptr,
                                                        const uint32_t* __restrict__ members, uint64_t m0,
                                                        uint64_t m1, uint64_t* s_pref, uint64_t* s_beg,
                                                        uint64_t* s_wsum, F&& f) {
    const unsigned tid = threadIdx.x, lane = tid & 31u, wid = tid >> 5, nw = blockDim.x >> 5;
    uint64_t flat0 = 0;  // entries of the earlier member chunks
    for (uint64_t mb = m0; mb < m1; mb += blockDim.x) {
        const uint64_t mi = mb + tid;
        uint64_t b = 0, d = 0;
        if (mi < m1) {
            const uint32_t v = members[mi];
            b = ptr[v];
            d = ptr[v + 1] - b;
        }
        uint64_t incl = d;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t t = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if ((int)lane >= o) incl += t;
        }
        if (lane == 31) s_wsum[wid] = incl;
        __syncthreads();
        uint64_t off = 0;
        for (unsigned k = 0; k < wid; ++k) off += s_wsum[k];
        s_pref[tid + 1] = off + incl;
        s_beg[tid] = b;
        if (tid == 0) s_pref[0] = 0;
        __syncthreads();
        const uint64_t nmem = (m1 - mb) < blockDim.x ? (m1 - mb) : blockDim.x;
        const uint64_t total = s_pref[nmem];
        for (uint64_t base = 0; base < total; base += blockDim.x) {
            const uint64_t t = base + tid;
            const bool valid = t < total;
            uint64_t j = 0;
            if (valid) {
                uint64_t lo = 0, hi = nmem;  // largest L with s_pref[L] <= t
                while (hi - lo > 1) {
                    const uint64_t mid = (lo + hi) >> 1;
                    if (s_pref[mid] <= t) lo = mid;
                    else hi = mid;
                }
                j = s_beg[lo] + (t - s_pref[lo]);
            }
            f(j, valid, flat0 + t);
        }
        flat0 += total;
        __syncthreads();
        (void)nw;
    }
}

// block_member_entries_at without the flattened index: f(j, valid).
template <class F>
__device__ __forceinline__ void block_member_entries(const uint64_t* __restrict__ ptr,
                                                     const uint32_t* __restrict__ members, uint64_t m0, uint64_t m1,
                                                     uint64_t* s_pref, uint64_t* s_beg, uint64_t* s_wsum, F&& f) {
    block_member_entries_at(ptr, members, m0, m1, s_pref, s_beg, s_wsum,
                            [&](uint64_t j, bool valid, uint64_t) { f(j, valid); });
}

// Warp-combined insert: lanes with the same key add their values through the
// lowest such lane, so a key hit by many lanes costs one shared atomic.
__device__ __forceinline__ void agg_insert_fix_combined(uint32_t* keys, unsigned long long* vals, uint64_t size,
                                                        uint64_t mask, bool valid, uint32_t h,
                                                        unsigned long long x, uint32_t* status) {
    const unsigned lane = threadIdx.x & 31u;
    const unsigned long long key = valid ? (unsigned long long)h : (0xFFFFFFFF00000000ull | lane);
    const unsigned mm = __match_any_sync(0xFFFFFFFFu, key);
    const unsigned long long acc = peer_sum(mm, valid ? x : 0ull);
    if (!valid || (int)lane != __ffs(mm) - 1) return;
    uint64_t slot = agg_hash(h) & mask;
    for (uint64_t probe = 0; probe < size; ++probe) {
        const uint32_t prev = atomicCAS(keys + slot, AGG_EMPTY, h);
        if (prev == AGG_EMPTY || prev == h) {
            atomicAdd(vals + slot, acc);
            return;
        }
        slot = (slot + 1) & mask;
    }
    atomicOr(status, DEV_OVERFLOW);
}

__global__ void __launch_bounds__(32 * AGG_WARPS)
    k_contract_warp(const uint64_t* __restrict__ gstart, const uint32_t* __restrict__ members, uint64_t G,
                    const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                    const float* __restrict__ w, const uint32_t* __restrict__ grp, const uint64_t* __restrict__ cap,
                    const uint64_t* __restrict__ capstart, const double* __restrict__ loops, uint32_t* tnbr,
                    float* tw, uint32_t* cnt, uint32_t* status) {
    __shared__ uint32_t s_keys[AGG_WARPS][2 * AGG_WARP_CAP];
    __shared__ double s_vals[AGG_WARPS][2 * AGG_WARP_CAP];
    __shared__ uint32_t s_lk[AGG_WARPS][AGG_WARP_CAP];
    __shared__ float s_lw[AGG_WARPS][AGG_WARP_CAP];
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* keys = s_keys[wib];
    double* vals = s_vals[wib];
    uint32_t* lk = s_lk[wib];
    float* lw = s_lw[wib];
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = warp; g < G; g += nwarps) {
        const uint64_t cg = cap[g];
        if (cg > AGG_WARP_CAP) continue;  // warp-uniform: a block-kernel row
        uint64_t size = 64;
        while (size < 2 * cg) size <<= 1;
        for (uint64_t s = lane; s < size; s += 32) {
            keys[s] = AGG_EMPTY;
            vals[s] = 0.0;
        }
        __syncwarp();
        warp_member_entries(ptr, members, gstart[g], gstart[g + 1], [&](uint64_t j, bool valid) {
            uint32_t h = 0;
            double x = 0.0;
            if (valid) {
                h = grp[nbr[j]];
                x = (double)w[j];
            }
            // lanes with the same key add through the lowest one (exact regime: any grouping)
            const unsigned long long key = valid ? (unsigned long long)h : (0xFFFFFFFF00000000ull | (unsigned)lane);
            const unsigned mm = __match_any_sync(FULL, key);
            const double acc = peer_sum(mm, x);
            if (valid && lane == __ffs(mm) - 1) agg_insert(keys, vals, size, h, acc, status);
        });
        __syncwarp();
        uint32_t nk = 0;
        for (uint64_t s0 = 0; s0 < size; s0 += 32) {
            const uint64_t s = s0 + lane;
            const uint32_t h = keys[s];
            bool keep = false;
            float val = 0.0f;
            if (h != AGG_EMPTY) val = agg_value((uint32_t)g, h, vals[s], loops, &keep);
            const unsigned bal = __ballot_sync(FULL, keep);
            if (keep) {
                const uint32_t pos = nk + __popc(bal & ((1u << lane) - 1u));
                lk[pos] = h;
                lw[pos] = val;
            }
            nk += __popc(bal);
        }
        __syncwarp();
        const uint64_t o = capstart[g];
        for (uint32_t i = lane; i < nk; i += 32) {
            const uint32_t h = lk[i];
            uint32_t r = 0;
            for (uint32_t j = 0; j < nk; ++j) r += lk[j] < h;
            tnbr[o + r] = h;
            tw[o + r] = lw[i];
        }
        if (lane == 0) cnt[g] = nk;
        __syncwarp();
    }
}

// Rows too large for a shared table (the "big" rows): every member entry as a
// (g, h) key and its weight, row i's entries at loff[i] .., one block per row.
__global__ void __launch_bounds__(256)
    k_big_row_keys(const uint32_t* __restrict__ rows, uint64_t nrows, const uint64_t* __restrict__ loff,
                   const uint64_t* __restrict__ gstart, const uint32_t* __restrict__ members,
                   const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr, const float* __restrict__ w,
                   const uint32_t* __restrict__ grp, uint64_t G, uint64_t* keys, float* vals) {
    __shared__ uint64_t s_pref[257], s_beg[256], s_wsum[8];
    for (uint64_t i = blockIdx.x; i < nrows; i += gridDim.x) {
        const uint32_t g = rows[i];
        const uint64_t o = loff[i];
        block_member_entries_at(ptr, members, gstart[g], gstart[g + 1], s_pref, s_beg, s_wsum,
                                [&](uint64_t j, bool valid, uint64_t t) {
                                    if (!valid) return;
                                    keys[o + t] = (uint64_t)g * G + grp[nbr[j]];
                                    vals[o + t] = w[j];
                                });
    }
}

// The kept (g, h, w) of the big rows, sorted by (g, h) with row starts kstart,
// into each row's slot range: one block per big row.
__global__ void k_place_big_rows(const uint32_t* __restrict__ rows, uint64_t nrows,
                                 const uint64_t* __restrict__ kstart, const uint32_t* __restrict__ kcol,
                                 const float* __restrict__ kw, const uint64_t* __restrict__ capstart, uint32_t* tnbr,
                                 float* tw, uint32_t* cnt) {
    for (uint64_t i = blockIdx.x; i < nrows; i += gridDim.x) {
        const uint32_t g = rows[i];
        const uint64_t b = kstart[g], e = kstart[g + 1], o = capstart[g];
        for (uint64_t t = b + threadIdx.x; t < e; t += blockDim.x) {
            tnbr[o + (t - b)] = kcol[t];
            tw[o + (t - b)] = kw[t];
        }
        if (threadIdx.x == 0) cnt[g] = (uint32_t)(e - b);
    }
}

constexpr uint64_t AGG_SMEM_SLOTS = 4096;  // shared table of the block kernel (48 KB)
constexpr uint64_t AGG_SMALL_GRAPH = 1u << 16;  // entries up to which the hash path is always taken
// The share of the entries in rows past the warp kernel, as 1/AGG_SORT_SHARE,
// above which the whole graph takes the sort path (0: never). Measured on the
// kNN graphs of a run: never taking it (big rows sorted on their own, below)
// made aggregation twice as slow; a tenth is the best of the rules tried.
constexpr uint64_t AGG_SORT_SHARE = 10;
constexpr uint64_t AGG_SMEM_KEEP = AGG_SMEM_SLOTS / 2;

// A row has at most min(cap, G) distinct neighbour groups; its table needs twice that.
__device__ __forceinline__ uint64_t agg_slots(uint64_t cap, uint64_t G) {
    const uint64_t d = cap < G ? cap : G;
    uint64_t s = 64;
    while (s < 2 * d) s <<= 1;
    return s;
}

// mid: rows past the warp kernel whose table fits the block kernel's shared
// memory; big: the rest (their entries are sorted, k_big_row_keys).
__global__ void k_flag_large(const uint64_t* __restrict__ cap, uint64_t G, uint8_t* mid, uint8_t* big,
                             uint64_t* lcap) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < G;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const bool large = cap[g] > AGG_WARP_CAP;
        const bool m = large && agg_slots(cap[g], G) <= AGG_SMEM_SLOTS;
        mid[g] = m;
        big[g] = large && !m;
        lcap[g] = large ? cap[g] : 0;
    }
}

// One block per row of the mid list: integer fixed-point sums (exact in this
// regime: every weight is a multiple of 2^e0 and every sum below 2^(52+e0)) in
// a shared table, kept entries sorted by neighbour with a block bitonic sort.
__global__ void __launch_bounds__(256)
    k_contract_smem(const uint32_t* __restrict__ rows, uint64_t nrows, uint64_t G,
                    const uint64_t* __restrict__ gstart, const uint32_t* __restrict__ members,
                    const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                    const float* __restrict__ w, const uint32_t* __restrict__ grp, const uint64_t* __restrict__ cap,
                    const uint64_t* __restrict__ capstart, const double* __restrict__ loops, double inv_scale,
                    double scale, uint32_t* tnbr, float* tw, uint32_t* cnt, uint32_t* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* vals = (unsigned long long*)smem_raw;          // AGG_SMEM_SLOTS
    uint32_t* keys = (uint32_t*)(vals + AGG_SMEM_SLOTS);               // AGG_SMEM_SLOTS
    uint32_t* sk = keys + AGG_SMEM_SLOTS;                              // AGG_SMEM_KEEP
    float* sv = (float*)(sk + AGG_SMEM_KEEP);                          // AGG_SMEM_KEEP
    __shared__ uint32_t s_n;
    __shared__ uint64_t s_pref[257], s_beg[256], s_wsum[8];
    for (uint64_t i = blockIdx.x; i < nrows; i += gridDim.x) {
        const uint32_t g = rows[i];
        const uint64_t size = agg_slots(cap[g], G);
        const uint64_t mask = size - 1;
        for (uint64_t s2 = threadIdx.x; s2 < size; s2 += blockDim.x) {
            keys[s2] = AGG_EMPTY;
            vals[s2] = 0ull;
        }
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        block_member_entries(ptr, members, gstart[g], gstart[g + 1], s_pref, s_beg, s_wsum,
                             [&](uint64_t j, bool valid) {
                                 uint32_t h = 0;
                                 unsigned long long x = 0;
                                 if (valid) {
                                     h = grp[nbr[j]];
                                     x = (unsigned long long)__double2ll_rn(__dmul_rn((double)w[j], inv_scale));
                                 }
                                 agg_insert_fix_combined(keys, vals, size, mask, valid, h, x, status);
                             });
        for (uint64_t s2 = threadIdx.x; s2 < size; s2 += blockDim.x) {
            const uint32_t h = keys[s2];
            if (h == AGG_EMPTY) continue;
            bool keep;
            const double acc = __dmul_rn(__ll2double_rn((long long)vals[s2]), scale);
            const float val = agg_value(g, h, acc, loops, &keep);
            if (keep) {
                const uint32_t pos = atomicAdd(&s_n, 1u);
                if (pos < AGG_SMEM_KEEP) {
                    sk[pos] = h;
                    sv[pos] = val;
                } else {
                    atomicOr(status, DEV_OVERFLOW);
                }
            }
        }
        __syncthreads();
        const uint32_t nk = s_n < AGG_SMEM_KEEP ? s_n : (uint32_t)AGG_SMEM_KEEP;
        uint32_t P = 1;
        while (P < nk) P <<= 1;
        for (uint32_t t = nk + threadIdx.x; t < P; t += blockDim.x) sk[t] = AGG_EMPTY;
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1)
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t t = threadIdx.x; t < P; t += blockDim.x) {
                    const uint32_t o = t ^ j;
                    if (o > t) {
                        const bool up = (t & k) == 0;
                        const uint32_t a = sk[t], b = sk[o];
                        if ((a > b) == up) {
                            sk[t] = b;
                            sk[o] = a;
                            const float va = sv[t];
                            sv[t] = sv[o];
                            sv[o] = va;
                        }
                    }
                }
                __syncthreads();
            }
        const uint64_t o = capstart[g];
        for (uint32_t t = threadIdx.x; t < nk; t += blockDim.x) {
            tnbr[o + t] = sk[t];
            tw[o + t] = sv[t];
        }
        if (threadIdx.x == 0) cnt[g] = nk;
        __syncthreads();
    }
}

__global__ void k_gather_u64(const uint32_t* __restrict__ idx, uint64_t n, const uint64_t* __restrict__ src,
                             uint64_t* dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

// Final rows: ptr from the kept counts, entries copied from the row slots.
__global__ void k_pack_rows(const uint64_t* __restrict__ optr, const uint64_t* __restrict__ capstart, uint64_t G,
                            const uint32_t* __restrict__ tnbr, const float* __restrict__ tw, uint32_t* nbr,
                            float* w) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = warp; g < G; g += nwarps) {
        const uint64_t o = optr[g], len = optr[g + 1] - o, src = capstart[g];
        for (uint64_t j = lane; j < len; j += 32) {
            nbr[o + j] = tnbr[src + j];
            w[o + j] = tw[src + j];
        }
    }
}

__global__ void k_u32_to_u64(const uint32_t* __restrict__ a, uint64_t n, uint64_t* b) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = i < n ? a[i] : 0;
}

}  // namespace

// Whether g's stored weights are bitwise symmetric (cached on the graph).
bool graph_bitwise_symmetric(Ctx& c, const DevGraph& g) {
    int st = g.sym_state.load(std::memory_order_relaxed);
    if (st != 0) return st == 1;
    DBuf<unsigned> bad(c, 1);
    DBuf<unsigned long long> counts(c, 2);
    zero(c, bad.get(), 1);
    zero(c, counts.get(), 2);
    if (g.E) {
        k_symmetric_bits<<<grid_for(g.E, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, g.erow, g.E, bad.get(),
                                                                counts.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    Mailbox mb(c);
    const unsigned* hb = mb.get(bad.get(), 1);
    const unsigned long long* hc = mb.get(counts.get(), 2);
    mb.wait();
    const bool sym = *hb == 0 && hc[0] == hc[1];
    g.sym_state.store(sym ? 1 : 2, std::memory_order_relaxed);
    return sym;
}

namespace {

DevGraph* contract_exact(Ctx& c, const DevGraph& g, const uint32_t* d_grp, uint64_t G, const uint64_t* gstart,
                         const uint32_t* members, const double* nw_new, const double* loops) {
    std::unique_ptr<DevGraph> out(new DevGraph());
    out->part_max_2m = g.part_max_2m;  // aggregation keeps every instance's totals
    out->part_max_nw = g.part_max_nw;
    DBuf<uint64_t> cap(c, G + 1), capstart(c, G + 1);
    zero(c, cap.get() + G, 1);
    if (G) {
        k_row_caps<<<grid_for(G * 32, TB), TB, 0, c.stream>>>(gstart, members, G, g.ptr, cap.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    exclusive_sum(c, cap.get(), capstart.get(), G + 1);  // capstart[G] = E
    DBuf<uint32_t> tnbr(c, g.E), cnt(c, G + 1);
    DBuf<float> tw(c, g.E);
    zero(c, cnt.get(), G + 1);
    // rows past the warp kernel: shared-table rows (mid) and global-table rows (large)
    DBuf<uint8_t> fmid(c, G), flag(c, G);
    DBuf<uint64_t> lcap(c, G), nl(c, 3);
    DBuf<uint32_t> iota(c, G), rows(c, G), mrows(c, G);
    uint64_t nlarge = 0, nmid = 0;
    if (G) {
        k_flag_large<<<grid_for(G, TB), TB, 0, c.stream>>>(cap.get(), G, fmid.get(), flag.get(), lcap.get());
        k_iota<<<grid_for(G, TB), TB, 0, c.stream>>>(iota.get(), G);
        SC_LAUNCH_CHECK();
        c.launches += 2;
        select_flagged(c, iota.get(), flag.get(), rows.get(), nl.get(), G);
        select_flagged(c, iota.get(), fmid.get(), mrows.get(), nl.get() + 1, G);
        device_sum(c, lcap.get(), nl.get() + 2, G);
        uint64_t counts[3];
        {
            Mailbox mb(c);
            const uint64_t* hc = mb.get(nl.get(), 3);
            mb.wait();
            std::memcpy(counts, hc, sizeof counts);
        }
        nlarge = counts[0];
        nmid = counts[1];
        // Rows past the warp kernel are served by one block each; when they hold
        // more than a tenth of the entries the sort path is faster (measured on
        // kNN graphs at every level of a run), except on small graphs, where the
        // sort path's extra launches and read-backs cost more than any block.
        if (AGG_SORT_SHARE && counts[2] * AGG_SORT_SHARE > g.E && g.E > AGG_SMALL_GRAPH) return nullptr;
    }
    if (nmid) {
        const size_t smem = AGG_SMEM_SLOTS * (sizeof(unsigned long long) + sizeof(uint32_t)) +
                            AGG_SMEM_KEEP * (sizeof(uint32_t) + sizeof(float));
        SC_CUDA(cudaFuncSetAttribute(k_contract_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const double scale = std::ldexp(1.0, g.e0_w), inv = std::ldexp(1.0, -g.e0_w);
        const unsigned grid = (unsigned)std::min<uint64_t>(nmid, (uint64_t)c.sm_count * 3);
        k_contract_smem<<<grid, 256, smem, c.stream>>>(mrows.get(), nmid, G, gstart, members, g.ptr, g.nbr, g.w,
                                                       d_grp, cap.get(), capstart.get(), loops, inv, scale,
                                                       tnbr.get(), tw.get(), cnt.get(), c.d_status);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    if (G) {
        const unsigned grid = grid_for(G * 32, 32 * AGG_WARPS, 148u * 16u);
        k_contract_warp<<<grid, 32 * AGG_WARPS, 0, c.stream>>>(gstart, members, G, g.ptr, g.nbr, g.w, d_grp,
                                                               cap.get(), capstart.get(), loops, tnbr.get(), tw.get(),
                                                               cnt.get(), c.d_status);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    if (nlarge) {
        // big rows: their member entries as (g, h) keys, sorted, summed per
        // segment and placed into their rows (sorted by neighbour already)
        DBuf<uint64_t> lc(c, nlarge + 1), loff(c, nlarge + 1);
        k_gather_u64<<<grid_for(nlarge, TB), TB, 0, c.stream>>>(rows.get(), nlarge, cap.get(), lc.get());
        zero(c, lc.get() + nlarge, 1);
        exclusive_sum(c, lc.get(), loff.get(), nlarge + 1);
        c.launches++;
        const uint64_t L = to_host(c, loff.get() + nlarge);
        DBuf<uint64_t> keys(c, L), keys_s(c, L);
        DBuf<float> vals(c, L), vals_s(c, L);
        const unsigned grid = (unsigned)std::min<uint64_t>(nlarge, (uint64_t)c.sm_count * 4);
        k_big_row_keys<<<grid, 256, 0, c.stream>>>(rows.get(), nlarge, loff.get(), gstart, members, g.ptr, g.nbr,
                                                   g.w, d_grp, G, keys.get(), vals.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        sort_pairs(c, keys.get(), keys_s.get(), vals.get(), vals_s.get(), L, bits_for((uint64_t)G * G - 1));
        keys.release();
        vals.release();
        DBuf<uint32_t> prow, pcol;
        DBuf<float> pw;
        DBuf<uint8_t> keep;
        const uint64_t P = segment_sums(c, keys_s.get(), vals_s.get(), L, G, loops, true, prow, pcol, pw, keep);
        keys_s.release();
        vals_s.release();
        if (P) {
            DBuf<uint32_t> krow(c, P), kcol(c, P);
            DBuf<float> kw(c, P);
            DBuf<uint64_t> kc(c, 1), kstart(c, (uint64_t)G + 1);
            select_flagged(c, prow.get(), keep.get(), krow.get(), kc.get(), P);
            select_flagged(c, pcol.get(), keep.get(), kcol.get(), kc.get(), P);
            select_flagged(c, pw.get(), keep.get(), kw.get(), kc.get(), P);
            const uint64_t K = to_host(c, kc.get());
            k_starts_from_sorted<<<grid_for(K + 1, TB), TB, 0, c.stream>>>(krow.get(), K, G, kstart.get());
            k_place_big_rows<<<grid, 256, 0, c.stream>>>(rows.get(), nlarge, kstart.get(), kcol.get(), kw.get(),
                                                         capstart.get(), tnbr.get(), tw.get(), cnt.get());
            SC_LAUNCH_CHECK();
            c.launches += 2;
        }
    }
    // assemble (the status word of the contraction kernels is read with the size)
    DBuf<uint64_t> cnt64(c, G + 1), optr(c, G + 1);
    k_u32_to_u64<<<grid_for(G + 1, TB), TB, 0, c.stream>>>(cnt.get(), G + 1, cnt64.get());
    exclusive_sum(c, cnt64.get(), optr.get(), G + 1);
    uint64_t E2;
    {
        Mailbox mb(c);
        const uint32_t* hs = mb.get(c.d_status, 1);
        const uint64_t* he = mb.get(optr.get() + G, 1);
        mb.wait();
        const uint32_t st = *hs;
        E2 = *he;
        raise_device_status(c, st);
    }
    galloc(c, *out, G, E2);
    d2d(c, out->ptr, optr.get(), G + 1);
    d2d(c, out->node_w, nw_new, G);
    if (E2) {
        k_pack_rows<<<grid_for(G * 32, TB), TB, 0, c.stream>>>(optr.get(), capstart.get(), G, tnbr.get(), tw.get(),
                                                               out->nbr, out->w);
        k_fill_erow<<<grid_for(G * 32, TB), TB, 0, c.stream>>>(out->ptr, G, out->erow);
        SC_LAUNCH_CHECK();
        c.launches += 2;
    }
    c.launches++;
    return out.release();
}

// One instance's arrays inside a union graph.
struct UnionPart {
    const uint64_t* ptr;
    const uint32_t* nbr;
    const float* w;
    const uint32_t* erow;
    const double* node_w;
    uint64_t n, E, noff, eoff;
};

// Copies instance blockIdx.y into the union: ids shift by its node offset,
// entry offsets by its entry offset. Blocks along x stride over its entries
// and nodes.
__global__ void k_union_copy(const UnionPart* __restrict__ parts, uint64_t* ptr, uint32_t* nbr, float* w,
                             uint32_t* erow, double* node_w) {
    const UnionPart pt = parts[blockIdx.y];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < pt.E; e += stride) {
        nbr[pt.eoff + e] = pt.nbr[e] + (uint32_t)pt.noff;
        erow[pt.eoff + e] = pt.erow[e] + (uint32_t)pt.noff;
        w[pt.eoff + e] = pt.w[e];
    }
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < pt.n; v += stride) {
        ptr[pt.noff + v] = pt.ptr[v] + pt.eoff;
        node_w[pt.noff + v] = pt.node_w[v];
    }
}

}  // namespace

// The disjoint union of graphs (instance i's nodes follow instance i-1's):
// one graph whose rows are the instances' rows, ids shifted, with its own
// statistics (from the default pool, like the graphs of a run).
DevGraph* graph_union(Ctx& c, const DevGraph* const* gs, uint64_t count) {
    if (count == 0 || count > 65535) fail(SC_E_INVALID_ARGUMENT, "a union takes 1..65535 graphs");
    std::vector<UnionPart> parts(count);
    uint64_t n = 0, E = 0;
    for (uint64_t i = 0; i < count; ++i) {
        const DevGraph& g = *gs[i];
        parts[i] = UnionPart{g.ptr, g.nbr, g.w, g.erow, g.node_w, g.n, g.E, n, E};
        n += g.n;
        E += g.E;
    }
    if (n >= 0x7FFFFFFFull) fail(SC_E_TOO_MANY_NODES, "a union of %llu nodes exceeds 2^31 - 1", (unsigned long long)n);
    std::unique_ptr<DevGraph> u(new DevGraph());
    u->pooled = true;
    // sums never cross instances: the heaviest instance decides the regime
    for (uint64_t i = 0; i < count; ++i) {
        const DevGraph& g = *gs[i];
        u->part_max_2m = std::max(u->part_max_2m, std::max(g.part_max_2m, 2.0 * g.total_weight));
        u->part_max_nw = std::max(u->part_max_nw, std::max(g.part_max_nw, g.total_node_weight));
    }
    if (u->part_max_2m == 0.0) u->part_max_2m = -1.0;  // no edges: the union's own (zero) totals decide
    if (u->part_max_nw == 0.0) u->part_max_nw = -1.0;
    galloc(c, *u, n, E);
    DBuf<UnionPart> d_parts(c, count);
    h2d(c, d_parts.get(), parts.data(), count);
    uint64_t most = 0;
    for (const UnionPart& pt : parts) most = std::max(most, std::max(pt.E, pt.n));
    const unsigned gx = grid_for(most, TB, 148u * 8u);
    k_union_copy<<<dim3(gx, (unsigned)count), TB, 0, c.stream>>>(d_parts.get(), u->ptr, u->nbr, u->w, u->erow,
                                                                  u->node_w);
    SC_LAUNCH_CHECK();
    c.launches++;
    SC_CUDA(cudaMemcpyAsync(u->ptr + n, &E, sizeof(uint64_t), cudaMemcpyHostToDevice, c.stream));
    finalize(c, *u, false);
    sync(c);  // the host value of E above must outlive the copy
    return u.release();
}

// Stats and checks of an aggregated graph; its rows mirror each other exactly.
void finish_aggregate(Ctx& c, DevGraph& out) {
    // aggregate cannot fail in the reference (csr_network.rs:605-607)
    try {
        finalize(c, out, true);
    } catch (Failure& f) {
        if (f.info.code == SC_E_ASYMMETRIC_GRAPH) {
            f.info.code = SC_E_INTERNAL;
            std::snprintf(f.info.message, sizeof f.info.message,
                          "aggregate produced a graph failing the degree-sum check");
        }
        throw;
    }
    out.sym_state.store(1, std::memory_order_relaxed);
}

DevGraph* graph_aggregate(Ctx& c, const DevGraph& g, const uint32_t* d_grp, uint32_t G) {
    const uint64_t n = g.n, E = g.E;
    std::unique_ptr<DevGraph> out(new DevGraph());
    out->part_max_2m = g.part_max_2m;  // aggregation keeps every instance's totals
    out->part_max_nw = g.part_max_nw;
    // members of each group in ascending node order
    DBuf<uint32_t> idx(c, n), grp_s(c, n), members(c, n);
    DBuf<uint64_t> gstart(c, (uint64_t)G + 1);
    DBuf<double> nw_new(c, G), loops(c, G);
    if (n) {
        k_iota<<<grid_for(n, TB), TB, 0, c.stream>>>(idx.get(), n);
        c.launches++;
        sort_pairs(c, d_grp, grp_s.get(), idx.get(), members.get(), n, bits_for(G));
        k_starts_from_sorted<<<grid_for(n + 1, TB), TB, 0, c.stream>>>(grp_s.get(), n, G, gstart.get());
        k_group_sums<<<grid_for((uint64_t)G * 32, TB), TB, 0, c.stream>>>(gstart.get(), members.get(), G, g.node_w,
                                                           g.self_loop, nw_new.get(), loops.get(),
                                                           (int)g.exact_nw, (int)g.exact_w);
        SC_LAUNCH_CHECK();
        c.launches += 2;
    }
    idx.release();
    grp_s.release();
    if (g.exact_w && graph_bitwise_symmetric(c, g)) {
        std::unique_ptr<DevGraph> fast(contract_exact(c, g, d_grp, G, gstart.get(), members.get(), nw_new.get(),
                                                      loops.get()));
        if (fast) {
            members.release();
            gstart.release();
            finish_aggregate(c, *fast);
            return fast.release();
        }
    }
    members.release();
    gstart.release();

    // (g, h >= g) entries in CSR order, stably sorted by (g, h)
    uint64_t N = 0;
    DBuf<uint64_t> ukeys, ukeys_s;
    DBuf<float> uw, uw_s;
    if (E) {
        DBuf<uint64_t> keys(c, E);
        DBuf<uint8_t> flags(c, E);
        k_group_keys<<<grid_for(E, TB), TB, 0, c.stream>>>(g.erow, g.nbr, d_grp, E, G, keys.get(),
                                                           flags.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        ukeys.alloc(c, E);
        uw.alloc(c, E);
        DBuf<uint64_t> cnt(c, 1);
        select_flagged(c, keys.get(), flags.get(), ukeys.get(), cnt.get(), E);
        select_flagged(c, g.w, flags.get(), uw.get(), cnt.get(), E);
        N = to_host(c, cnt.get());
        ukeys_s.alloc(c, N);
        uw_s.alloc(c, N);
        sort_pairs(c, ukeys.get(), ukeys_s.get(), uw.get(), uw_s.get(), N,
                   bits_for((uint64_t)G * G - 1));
        ukeys.release();
        uw.release();
    }
    // segments = distinct (g, h)
    DBuf<uint32_t> prow, pcol;
    DBuf<float> pw;
    DBuf<uint8_t> keep;
    const uint64_t P = segment_sums(c, ukeys_s.get(), uw_s.get(), N, G, loops.get(), g.exact_w, prow, pcol, pw,
                                    keep);
    ukeys_s.release();
    uw_s.release();
    // kept pairs, still in (g, h) order: the upper triangle incl. diagonal
    uint64_t K = 0;
    DBuf<uint32_t> krow, kcol;
    DBuf<float> kw;
    if (P) {
        krow.alloc(c, P);
        kcol.alloc(c, P);
        kw.alloc(c, P);
        DBuf<uint64_t> cnt(c, 1);
        select_flagged(c, prow.get(), keep.get(), krow.get(), cnt.get(), P);
        select_flagged(c, pcol.get(), keep.get(), kcol.get(), cnt.get(), P);
        select_flagged(c, pw.get(), keep.get(), kw.get(), cnt.get(), P);
        K = to_host(c, cnt.get());
    }
    prow.release();
    pcol.release();
    pw.release();
    keep.release();
    // lower triangle: mirrored off-diagonal pairs sorted by (h, g)
    uint64_t L = 0;
    DBuf<uint32_t> lrow, lcol;
    DBuf<float> lw;
    if (K) {
        DBuf<uint64_t> mk(c, K), mk_c(c, K), mk_s(c, K);
        DBuf<float> mw(c, K), mw_c(c, K);
        DBuf<uint8_t> mf(c, K);
        k_mirror<<<grid_for(K, TB), TB, 0, c.stream>>>(krow.get(), kcol.get(), kw.get(), K, G,
                                                       mk.get(), mw.get(), mf.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        DBuf<uint64_t> cnt(c, 1);
        select_flagged(c, mk.get(), mf.get(), mk_c.get(), cnt.get(), K);
        select_flagged(c, mw.get(), mf.get(), mw_c.get(), cnt.get(), K);
        L = to_host(c, cnt.get());
        lw.alloc(c, L);
        sort_pairs(c, mk_c.get(), mk_s.get(), mw_c.get(), lw.get(), L,
                   bits_for((uint64_t)G * G - 1));
        lrow.alloc(c, L);
        lcol.alloc(c, L);
        if (L) {
            k_key_rows<<<grid_for(L, TB), TB, 0, c.stream>>>(mk_s.get(), L, G, lrow.get(), lcol.get());
            SC_LAUNCH_CHECK();
            c.launches++;
        }
    }
    // assemble
    const uint64_t E2 = K + L;
    galloc(c, *out, G, E2);
    d2d(c, out->node_w, nw_new.get(), G);
    {
        DBuf<uint64_t> us(c, (uint64_t)G + 1), ls(c, (uint64_t)G + 1), cnt(c, (uint64_t)G + 1);
        k_starts_from_sorted<<<grid_for(K + 1, TB), TB, 0, c.stream>>>(krow.get(), K, G, us.get());
        k_starts_from_sorted<<<grid_for(L + 1, TB), TB, 0, c.stream>>>(lrow.get(), L, G, ls.get());
        SC_LAUNCH_CHECK();
        k_row_counts<<<grid_for(G, TB), TB, 0, c.stream>>>(ls.get(), us.get(), G, cnt.get());
        zero(c, cnt.get() + G, 1);
        exclusive_sum(c, cnt.get(), out->ptr, (uint64_t)G + 1);
        if (E2) {
            k_row_assemble<<<grid_for((uint64_t)G * 32, TB), TB, 0, c.stream>>>(
                out->ptr, ls.get(), lcol.get(), lw.get(), us.get(), kcol.get(), kw.get(), G,
                out->nbr, out->w);
            SC_LAUNCH_CHECK();
            k_fill_erow<<<grid_for((uint64_t)G * 32, TB), TB, 0, c.stream>>>(out->ptr, G, out->erow);
            SC_LAUNCH_CHECK();
            c.launches += 2;
        }
        c.launches += 3;
    }
    finish_aggregate(c, *out);
    return out.release();
}

// ------------------------------------------------------------ symmetry
namespace {
// validate_symmetry (csr_network.rs:627-646) with edge_weight's shorter-row
// search (:465-478): first failing stored entry, as its index.
__global__ void k_symmetry(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                           const float* __restrict__ w, const uint32_t* __restrict__ erow,
                           uint64_t E, unsigned long long* first) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < E;
         e += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = erow[e], u = nbr[e];
        double x = (double)w[e];
        // edge_weight(u, v)
        uint64_t du = ptr[u + 1] - ptr[u], dv = ptr[v + 1] - ptr[v];
        uint32_t s = du <= dv ? u : v, t = du <= dv ? v : u;
        uint64_t lo = ptr[s], hi = ptr[s + 1];
        while (lo < hi) {
            uint64_t mid = (lo + hi) >> 1;
            if (nbr[mid] < t) lo = mid + 1;
            else hi = mid;
        }
        bool found = lo < ptr[s + 1] && nbr[lo] == t;
        bool ok = found && fabs((double)w[lo] - x) <= 1e-6 * fmax(fabs(x), 1.0);
        if (!ok) atomicMin(first, (unsigned long long)e);
    }
}
}  // namespace

void graph_validate_symmetry(Ctx& c, const DevGraph& g) {
    if (g.E == 0) return;
    DBuf<unsigned long long> first(c, 1);
    const unsigned long long NOBAD = ~0ull;
    h2d(c, first.get(), &NOBAD, 1);
    k_symmetry<<<grid_for(g.E, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, g.erow, g.E, first.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    uint64_t e = first_bad(c, first);
    if (e == NOBAD) return;
    // re-derive the message on the host from the few values involved
    uint32_t v, u;
    float x;
    d2h(c, &v, g.erow + e, 1);
    d2h(c, &u, g.nbr + e, 1);
    d2h(c, &x, g.w + e, 1);
    uint64_t pu[2], pv[2];
    sync(c);
    d2h(c, pu, g.ptr + u, 2);
    d2h(c, pv, g.ptr + v, 2);
    sync(c);
    uint64_t du = pu[1] - pu[0], dv = pv[1] - pv[0];
    uint32_t s = du <= dv ? u : v, t = du <= dv ? v : u;
    uint64_t lo = du <= dv ? pu[0] : pv[0], hi = du <= dv ? pu[1] : pv[1];
    std::vector<uint32_t> row(hi - lo);
    std::vector<float> rw(hi - lo);
    d2h(c, row.data(), g.nbr + lo, hi - lo);
    d2h(c, rw.data(), g.w + lo, hi - lo);
    sync(c);
    (void)s;
    auto it = std::lower_bound(row.begin(), row.end(), t);
    if (it == row.end() || *it != t)
        fail(SC_E_INVALID_CSR,
             "malformed CSR input: edge (%u, %u) is present but (%u, %u) is missing", v, u, u, v);
    double back = (double)rw[it - row.begin()];
    fail(SC_E_INVALID_CSR, "malformed CSR input: edge (%u, %u) has weight %s but (%u, %u) has %s", v,
         u, fmt_f64((double)x).c_str(), u, v, fmt_f64(back).c_str());
}

void graph_copy_csr(Ctx& c, const DevGraph& g, uint64_t* ptr, uint32_t* nbr, float* w) {
    if (ptr) d2h(c, ptr, g.ptr, g.n + 1);
    if (nbr) d2h(c, nbr, g.nbr, g.E);
    if (w) d2h(c, w, g.w, g.E);
    sync(c);
}

void graph_copy_node_data(Ctx& c, const DevGraph& g, double* node_w, double* strength) {
    if (node_w) d2h(c, node_w, g.node_w, g.n);
    if (strength) d2h(c, strength, g.strength, g.n);
    sync(c);
}

}  // namespace sc
