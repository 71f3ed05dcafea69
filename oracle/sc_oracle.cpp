// sc_oracle.cpp — CPU restatement of single-clustering v0.7.0's Leiden path.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline). Built with
// -O2 -ffp-contract=off and no fast-math, so every double operation is the
// IEEE-754 round-to-nearest operation Rust performs, in the same order.
//
// Each function names the reference item it restates as `file:line` relative
// to the single-clustering source tree. Deliberate differences:
//   * RNG: xoshiro256** seeded through splitmix64 instead of ChaCha8Rng /
//     rand 0.9 (mod.rs:172-175, partition.rs:512-530, refine.rs:144). The
//     reference's own tests only pin in-process determinism, so the stream is
//     unpinned either way; the call structure (one rng per leiden, a fresh
//     level rng per pass, one shuffle per local_move / refine, one f64 draw
//     per randomised select) is kept.
//   * finish sorts each row with a stable sort where the reference uses
//     sort_unstable; equal neighbour ids (duplicates) are then summed in input
//     order. The two agree whenever the f64 sum of a duplicate run is exact,
//     which holds for every input in the reference's tests.
#include "sc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <limits>
#include <string>
#include <vector>

namespace {

using std::size_t;
using std::vector;

constexpr uint32_t UNASSIGNED = 0xFFFFFFFFu;      // partition.rs:22
constexpr uint64_t MAX_NODES = 0xFFFFFFFFull;     // csr_network.rs:36
constexpr double MIN_GAIN_RELATIVE = 1e-12;       // local_move.rs:22
constexpr size_t MAX_MOVES_PER_NODE = 100;        // local_move.rs:32

thread_local sc_error_info g_err;

int fail(int code) {
    g_err.code = code;
    return code;
}

void clear_err() { std::memset(&g_err, 0, sizeof(g_err)); }

// Rust's `Iterator::sum` for f64 folds from -0.0 (edition 2024 toolchains).
template <class It>
double rust_sum(It b, It e) {
    double s = -0.0;
    for (; b != e; ++b) s += *b;
    return s;
}

// ---------------------------------------------------------------- RNG
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; ++i) {
            x += 0x9E3779B97F4A7C15ull;
            uint64_t z = x;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            s[i] = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next_u64() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double next_f64() { return (double)(next_u64() >> 11) * 0x1.0p-53; }
    // unbiased integer in [0, n) (Lemire's multiply-and-reject)
    uint64_t below(uint64_t n) {
        uint64_t x = next_u64();
        __uint128_t m = (__uint128_t)x * n;
        uint64_t l = (uint64_t)m;
        if (l < n) {
            uint64_t t = (0 - n) % n;
            while (l < t) {
                x = next_u64();
                m = (__uint128_t)x * n;
                l = (uint64_t)m;
            }
        }
        return (uint64_t)(m >> 64);
    }
    // Fisher-Yates from the back, like SliceRandom::shuffle
    void shuffle(vector<size_t>& a) {
        for (size_t i = a.size(); i > 1; --i) {
            size_t j = (size_t)below(i);
            std::swap(a[i - 1], a[j]);
        }
    }
};

// ---------------------------------------------------------------- graph
// CSRNetworkData (csr_network.rs:38-60)
struct Graph {
    vector<uint64_t> ptr;
    vector<uint32_t> nbr;
    vector<float> w;
    vector<double> node_w;
    vector<double> strength;
    double total_weight = 0.0;
    uint64_t edge_count = 0;
    bool any_self_loops = false;

    size_t n() const { return node_w.size(); }
    // self_loop_weight (csr_network.rs:452-462)
    double self_loop(size_t v) const {
        if (!any_self_loops) return 0.0;
        auto b = nbr.begin() + ptr[v], e = nbr.begin() + ptr[v + 1];
        auto it = std::lower_bound(b, e, (uint32_t)v);
        if (it != e && *it == (uint32_t)v) return (double)w[it - nbr.begin()];
        return 0.0;
    }
    // total_node_weight (csr_network.rs:446-448)
    double total_node_weight() const { return rust_sum(node_w.begin(), node_w.end()); }
};

// validate_node_weights (csr_network.rs:666-673)
bool validate_node_weights(const vector<double>& nw) {
    for (size_t v = 0; v < nw.size(); ++v) {
        double x = nw[v];
        if (!std::isfinite(x) || x < 0.0) {
            g_err.node = v;
            g_err.weight = x;
            fail(SC_E_INVALID_NODE_WEIGHT);
            return false;
        }
    }
    return true;
}

// check_edge (csr_network.rs:676-696)
bool check_edge(uint64_t from, uint64_t to, double w, uint64_t n) {
    if (from >= n) {
        g_err.node = from;
        g_err.n_nodes = n;
        fail(SC_E_NODE_INDEX_OUT_OF_RANGE);
        return false;
    }
    if (to >= n) {
        g_err.node = to;
        g_err.n_nodes = n;
        fail(SC_E_NODE_INDEX_OUT_OF_RANGE);
        return false;
    }
    if (!std::isfinite(w)) {
        g_err.edge_from = from;
        g_err.edge_to = to;
        fail(SC_E_NON_FINITE_WEIGHT);
        return false;
    }
    if (w < 0.0) {
        g_err.edge_from = from;
        g_err.edge_to = to;
        g_err.weight = w;
        fail(SC_E_NEGATIVE_WEIGHT);
        return false;
    }
    return true;
}

// check_degree_sum (csr_network.rs:712-723)
bool check_degree_sum(const Graph& g) {
    double sum = rust_sum(g.strength.begin(), g.strength.end());
    double expected = 2.0 * g.total_weight;
    double tol = 1e-6 * std::max(std::fabs(expected), 1.0);
    if (std::fabs(sum - expected) > tol) {
        g_err.degree_sum = sum;
        g_err.expected = expected;
        fail(SC_E_ASYMMETRIC_GRAPH);
        return false;
    }
    return true;
}

// finish (csr_network.rs:262-351)
bool finish(vector<uint64_t> ptr, vector<uint32_t> nbr, vector<float> w, vector<double> node_w,
            Graph& out) {
    const size_t n = ptr.size() - 1;
    vector<std::pair<uint32_t, float>> row;
    vector<double> strength(n, 0.0);
    double total = 0.0;
    uint64_t edge_count = 0;
    size_t write = 0;
    bool any_loops = false;
    for (size_t v = 0; v < n; ++v) {
        size_t lo = ptr[v], hi = ptr[v + 1];
        ptr[v] = write;
        row.clear();
        for (size_t i = lo; i < hi; ++i) row.emplace_back(nbr[i], w[i]);
        std::stable_sort(row.begin(), row.end(),
                         [](const auto& a, const auto& b) { return a.first < b.first; });
        size_t i = 0;
        while (i < row.size()) {
            uint32_t u = row[i].first;
            double acc = 0.0;
            while (i < row.size() && row[i].first == u) {
                acc += (double)row[i].second;
                ++i;
            }
            if (acc == 0.0) continue;  // an explicit zero is not an edge
            nbr[write] = u;
            w[write] = (float)acc;
            ++write;
            double stored = (double)(float)acc;
            if ((size_t)u == v) {
                any_loops = true;
                strength[v] += 2.0 * stored;
            } else {
                strength[v] += stored;
            }
            if (v <= (size_t)u) {
                total += stored;
                ++edge_count;
            }
        }
    }
    ptr[n] = write;
    nbr.resize(write);
    w.resize(write);
    out.ptr = std::move(ptr);
    out.nbr = std::move(nbr);
    out.w = std::move(w);
    out.node_w = std::move(node_w);
    out.strength = std::move(strength);
    out.total_weight = total;
    out.edge_count = edge_count;
    out.any_self_loops = any_loops;
    return check_degree_sum(out);
}

// from_edges_with_node_weights (csr_network.rs:120-167)
bool from_edges(const uint64_t* from, const uint64_t* to, const double* wt, size_t m,
                vector<double> node_w, Graph& out) {
    const size_t n = node_w.size();
    if (!validate_node_weights(node_w)) return false;
    if (n > MAX_NODES) {
        g_err.n_nodes = n;
        fail(SC_E_TOO_MANY_NODES);
        return false;
    }
    vector<uint64_t> counts(n, 0);
    for (size_t i = 0; i < m; ++i) {
        if (!check_edge(from[i], to[i], wt[i], n)) return false;
        counts[from[i]] += 1;
        if (from[i] != to[i]) counts[to[i]] += 1;
    }
    vector<uint64_t> ptr(n + 1, 0);
    for (size_t v = 0; v < n; ++v) ptr[v + 1] = ptr[v] + counts[v];
    size_t slots = ptr[n];
    vector<uint32_t> nbr(slots, 0);
    vector<float> w(slots, 0.0f);
    vector<uint64_t> cursor(ptr.begin(), ptr.end() - 1);
    for (size_t i = 0; i < m; ++i) {
        float x = (float)wt[i];
        uint64_t a = from[i], b = to[i];
        nbr[cursor[a]] = (uint32_t)b;
        w[cursor[a]] = x;
        cursor[a]++;
        if (a != b) {
            nbr[cursor[b]] = (uint32_t)a;
            w[cursor[b]] = x;
            cursor[b]++;
        }
    }
    return finish(std::move(ptr), std::move(nbr), std::move(w), std::move(node_w), out);
}

// from_csr_parts (csr_network.rs:185-256)
bool from_csr_parts(vector<uint64_t> ptr, vector<uint32_t> nbr, vector<float> w,
                    const double* node_w, size_t n_node_w, Graph& out) {
    char buf[200];
    if (ptr.empty()) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "malformed CSR input: node_ptrs must have at least one element");
        fail(SC_E_INVALID_CSR);
        return false;
    }
    size_t n = ptr.size() - 1;
    if (n > MAX_NODES) {
        g_err.n_nodes = n;
        fail(SC_E_TOO_MANY_NODES);
        return false;
    }
    if (nbr.size() != w.size()) {
        std::snprintf(buf, sizeof buf, "neighbors has %zu entries but weights has %zu", nbr.size(),
                      w.size());
        std::snprintf(g_err.message, sizeof g_err.message, "malformed CSR input: %s", buf);
        fail(SC_E_INVALID_CSR);
        return false;
    }
    if (ptr[n] != nbr.size()) {
        std::snprintf(buf, sizeof buf, "node_ptrs ends at %llu but there are %zu entries",
                      (unsigned long long)ptr[n], nbr.size());
        std::snprintf(g_err.message, sizeof g_err.message, "malformed CSR input: %s", buf);
        fail(SC_E_INVALID_CSR);
        return false;
    }
    for (size_t v = 0; v < n; ++v) {
        if (ptr[v] > ptr[v + 1]) {
            std::snprintf(g_err.message, sizeof g_err.message,
                          "malformed CSR input: node_ptrs is not non-decreasing at %zu", v);
            fail(SC_E_INVALID_CSR);
            return false;
        }
    }
    for (size_t i = 0; i < nbr.size(); ++i) {
        uint32_t u = nbr[i];
        float x = w[i];
        if ((size_t)u >= n) {
            g_err.node = u;
            g_err.n_nodes = n;
            fail(SC_E_NODE_INDEX_OUT_OF_RANGE);
            return false;
        }
        if (!std::isfinite(x)) {
            g_err.edge_from = 0;
            g_err.edge_to = u;
            fail(SC_E_NON_FINITE_WEIGHT);
            return false;
        }
        if (x < 0.0f) {
            g_err.edge_from = 0;
            g_err.edge_to = u;
            g_err.weight = (double)x;
            fail(SC_E_NEGATIVE_WEIGHT);
            return false;
        }
    }
    vector<double> nw;
    if (node_w) {
        if (n_node_w != n) {
            g_err.got = n_node_w;
            g_err.expected_len = n;
            fail(SC_E_NODE_WEIGHT_LENGTH_MISMATCH);
            return false;
        }
        nw.assign(node_w, node_w + n);
        if (!validate_node_weights(nw)) return false;
    } else {
        nw.assign(n, 1.0);
    }
    return finish(std::move(ptr), std::move(nbr), std::move(w), std::move(nw), out);
}

// VectorGrouping::from_assignments + normalize_groups (grouping.rs:154-172, :226-254)
vector<size_t> normalize_groups(const uint64_t* input, size_t n, size_t* group_count) {
    size_t max_group = 0;
    for (size_t i = 0; i < n; ++i) max_group = std::max<size_t>(max_group, input[i]);
    size_t gc = max_group + 1;
    vector<size_t> sizes(gc, 0);
    for (size_t i = 0; i < n; ++i) sizes[input[i]]++;
    vector<size_t> new_ids(gc);
    size_t next = 0;
    for (size_t c = 0; c < gc; ++c) new_ids[c] = sizes[c] == 0 ? SIZE_MAX : next++;
    vector<size_t> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = new_ids[input[i]];
    *group_count = next;
    return out;
}

// aggregate (csr_network.rs:516-608)
Graph aggregate(const Graph& g, const vector<size_t>& group, size_t n_groups) {
    const size_t n = g.n();
    vector<double> new_nw(n_groups, 0.0);
    for (size_t v = 0; v < n; ++v) new_nw[group[v]] += g.node_w[v];
    vector<size_t> starts(n_groups + 1, 0);
    for (size_t v = 0; v < n; ++v) starts[group[v] + 1]++;
    for (size_t c = 0; c < n_groups; ++c) starts[c + 1] += starts[c];
    vector<uint32_t> members(n);
    {
        vector<size_t> cursor(starts.begin(), starts.end() - 1);
        for (size_t v = 0; v < n; ++v) members[cursor[group[v]]++] = (uint32_t)v;
    }
    vector<double> acc(n_groups, 0.0);
    vector<size_t> touched;
    vector<uint64_t> counts(n_groups, 0);
    struct Pair {
        uint32_t a, b;
        float w;
    };
    vector<Pair> pairs;
    for (size_t c = 0; c < n_groups; ++c) {
        double loops = 0.0;
        for (size_t mi = starts[c]; mi < starts[c + 1]; ++mi) {
            size_t v = members[mi];
            for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
                size_t u = g.nbr[e];
                double x = (double)g.w[e];
                if (u == v) loops += x;
                size_t h = group[u];
                if (h < c) continue;
                if (acc[h] == 0.0) touched.push_back(h);
                acc[h] += x;
            }
        }
        for (size_t h : touched) {
            double x = acc[h];
            acc[h] = 0.0;
            if (x <= 0.0) continue;
            if (h == c) {
                pairs.push_back({(uint32_t)c, (uint32_t)c, (float)(0.5 * (x + loops))});
                counts[c]++;
            } else {
                pairs.push_back({(uint32_t)c, (uint32_t)h, (float)x});
                counts[c]++;
                counts[h]++;
            }
        }
        touched.clear();
    }
    vector<uint64_t> ptr(n_groups + 1, 0);
    for (size_t c = 0; c < n_groups; ++c) ptr[c + 1] = ptr[c] + counts[c];
    vector<uint32_t> nbr(ptr[n_groups]);
    vector<float> w(ptr[n_groups]);
    vector<uint64_t> cursor(ptr.begin(), ptr.end() - 1);
    for (const Pair& p : pairs) {
        nbr[cursor[p.a]] = p.b;
        w[cursor[p.a]] = p.w;
        cursor[p.a]++;
        if (p.a != p.b) {
            nbr[cursor[p.b]] = p.a;
            w[cursor[p.b]] = p.w;
            cursor[p.b]++;
        }
    }
    Graph out;
    finish(std::move(ptr), std::move(nbr), std::move(w), std::move(new_nw), out);
    return out;
}

// ---------------------------------------------------------------- partition
// Partition (partition.rs:26-333)
struct Partition {
    vector<uint32_t> memb;
    vector<uint32_t> size;
    vector<double> weight, strength, internal;
    vector<size_t> free;
    double total_weight = 0.0, total_node_weight = 0.0;

    size_t slots() const { return size.size(); }
    size_t community_count() const { return size.size() - free.size(); }
    size_t membership(size_t v) const { return memb[v]; }
    size_t sz(size_t c) const { return c < size.size() ? size[c] : 0; }
    double wt(size_t c) const { return c < weight.size() ? weight[c] : 0.0; }
    double st(size_t c) const { return c < strength.size() ? strength[c] : 0.0; }
    double in(size_t c) const { return c < internal.size() ? internal[c] : 0.0; }
    size_t empty_community() const { return free.empty() ? size.size() : free.back(); }

    // singleton (partition.rs:53-69)
    static Partition singleton(const Graph& g) {
        Partition p;
        size_t n = g.n();
        p.memb.resize(n);
        p.size.assign(n, 1);
        p.weight.resize(n);
        p.strength.resize(n);
        p.internal.resize(n);
        for (size_t v = 0; v < n; ++v) {
            p.memb[v] = (uint32_t)v;
            p.weight[v] = g.node_w[v];
            p.strength[v] = g.strength[v];
            p.internal[v] = g.self_loop(v);
        }
        p.total_weight = g.total_weight;
        p.total_node_weight = g.total_node_weight();
        return p;
    }

    // from_membership (partition.rs:75-112)
    static Partition from_membership(const Graph& g, const vector<size_t>& m) {
        Partition p;
        size_t slots = 0;
        for (size_t c : m) slots = std::max(slots, c + 1);
        p.memb.resize(m.size());
        for (size_t v = 0; v < m.size(); ++v) p.memb[v] = (uint32_t)m[v];
        p.size.assign(slots, 0);
        p.weight.assign(slots, 0.0);
        p.strength.assign(slots, 0.0);
        p.internal.assign(slots, 0.0);
        p.total_weight = g.total_weight;
        p.total_node_weight = g.total_node_weight();
        for (size_t v = 0; v < m.size(); ++v) {
            size_t c = m[v];
            p.size[c] += 1;
            p.weight[c] += g.node_w[v];
            p.strength[c] += g.strength[v];
        }
        for (size_t v = 0; v < m.size(); ++v) {
            size_t c = m[v];
            for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
                size_t u = g.nbr[e];
                if (m[u] != c) continue;
                if (u == v || v < u) p.internal[c] += (double)g.w[e];
            }
        }
        for (size_t c = slots; c-- > 0;)
            if (p.size[c] == 0) p.free.push_back(c);
        return p;
    }

    // remove_node (partition.rs:201-224)
    size_t remove_node(size_t v, const Graph& g, double w_own) {
        size_t c = memb[v];
        size[c] -= 1;
        weight[c] -= g.node_w[v];
        strength[c] -= g.strength[v];
        internal[c] -= w_own + g.self_loop(v);
        if (size[c] == 0) {
            weight[c] = 0.0;
            strength[c] = 0.0;
            internal[c] = 0.0;
            free.push_back(c);
        }
        memb[v] = UNASSIGNED;
        return c;
    }

    // insert_node (partition.rs:230-260)
    void insert_node(size_t v, size_t c, const Graph& g, double w_to) {
        if (c == size.size()) {
            size.push_back(0);
            weight.push_back(0.0);
            strength.push_back(0.0);
            internal.push_back(0.0);
        } else if (size[c] == 0) {
            for (size_t i = free.size(); i-- > 0;) {
                if (free[i] == c) {
                    free[i] = free.back();
                    free.pop_back();
                    break;
                }
            }
        }
        size[c] += 1;
        weight[c] += g.node_w[v];
        strength[c] += g.strength[v];
        internal[c] += w_to + g.self_loop(v);
        memb[v] = (uint32_t)c;
    }

    // renumber (partition.rs:265-296)
    void renumber() {
        size_t slots_n = size.size();
        vector<size_t> new_id(slots_n, SIZE_MAX);
        size_t next = 0;
        for (size_t c = 0; c < slots_n; ++c)
            if (size[c] > 0) new_id[c] = next++;
        for (size_t c = 0; c < slots_n; ++c) {
            size_t t = new_id[c];
            if (t == SIZE_MAX || t == c) continue;
            size[t] = size[c];
            weight[t] = weight[c];
            strength[t] = strength[c];
            internal[t] = internal[c];
        }
        size.resize(next);
        weight.resize(next);
        strength.resize(next);
        internal.resize(next);
        free.clear();
        for (auto& m : memb)
            if (m != UNASSIGNED) m = (uint32_t)new_id[m];
    }

    vector<size_t> membership_vec() const { return vector<size_t>(memb.begin(), memb.end()); }
};

// ---------------------------------------------------------------- objectives
// InsertContext (objective.rs:22-41)
struct InsertContext {
    double node_strength, node_weight, self_loop;
    static InsertContext for_node(const Graph& g, size_t v) {
        return {g.strength[v], g.node_w[v], g.self_loop(v)};
    }
};

// Rb / Cpm (objective.rs:89-184)
struct Objective {
    int kind;
    double gamma;
    double delta_insert(const Partition& p, const InsertContext& ctx, size_t c, double w) const {
        if (kind == SC_OBJECTIVE_RB) {
            double four_m = 4.0 * p.total_weight;
            if (four_m == 0.0) return 0.0;
            double k_c = p.st(c);
            double k = ctx.node_strength;
            return (w + ctx.self_loop) - gamma * k * (2.0 * k_c + k) / four_m;
        }
        double n_c = p.wt(c);
        double a = ctx.node_weight;
        return (w + ctx.self_loop) - gamma * a * (2.0 * n_c + a - 1.0) / 2.0;
    }
    double quality(const Partition& p) const {
        vector<double> terms(p.slots());
        if (kind == SC_OBJECTIVE_RB) {
            double four_m = 4.0 * p.total_weight;
            if (four_m == 0.0) return 0.0;
            for (size_t c = 0; c < p.slots(); ++c) {
                double k_c = p.st(c);
                terms[c] = p.in(c) - gamma * k_c * k_c / four_m;
            }
        } else {
            for (size_t c = 0; c < p.slots(); ++c) {
                double n_c = p.wt(c);
                terms[c] = p.in(c) - gamma * n_c * (n_c - 1.0) / 2.0;
            }
        }
        return rust_sum(terms.begin(), terms.end());
    }
};

// modularity (objective.rs:221-244)
double modularity(const Graph& g, const uint64_t* labels, double gamma) {
    double m = g.total_weight;
    if (m == 0.0) return 0.0;
    size_t n_comms = 0;
    for (size_t v = 0; v < g.n(); ++v) n_comms = std::max<size_t>(n_comms, labels[v] + 1);
    vector<double> internal(n_comms, 0.0), strength(n_comms, 0.0);
    for (size_t v = 0; v < g.n(); ++v) {
        size_t c = labels[v];
        strength[c] += g.strength[v];
        for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
            size_t u = g.nbr[e];
            if (labels[u] == c && (u == v || v < u)) internal[c] += (double)g.w[e];
        }
    }
    double two_m = 2.0 * m;
    vector<double> terms(n_comms);
    for (size_t c = 0; c < n_comms; ++c) {
        double s = strength[c] / two_m;
        terms[c] = 2.0 * internal[c] / two_m - gamma * (s * s);
    }
    return rust_sum(terms.begin(), terms.end());
}

// ---------------------------------------------------------------- scratch
// NeighborWeights (partition.rs:343-484)
struct NeighborWeights {
    struct Slot {
        uint64_t stamp = 0;
        double weight = 0.0;
    };
    vector<Slot> slots;
    uint64_t generation = 0;
    vector<size_t> touched;

    void ensure_capacity(size_t n) {
        if (slots.size() < n) slots.resize(n);
    }
    void begin() {
        touched.clear();
        if (generation == UINT64_MAX) {
            for (auto& s : slots) s.stamp = 0;
            generation = 1;
        } else {
            generation++;
        }
    }
    void add(size_t c, double w) {
        if (c >= slots.size()) slots.resize(c + 1);
        Slot& s = slots[c];
        if (s.stamp != generation) {
            s.stamp = generation;
            s.weight = w;
            touched.push_back(c);
        } else {
            s.weight += w;
        }
    }
    void collect(const Graph& g, const vector<uint32_t>& memb, size_t v) {
        begin();
        for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
            size_t u = g.nbr[e];
            if (u == v) continue;
            uint32_t c = memb[u];
            if (c == UNASSIGNED) continue;
            add(c, (double)g.w[e]);
        }
    }
    void collect_constrained(const Graph& g, const vector<uint32_t>& memb, size_t v,
                             const uint32_t* constraint) {
        begin();
        uint32_t own = constraint[v];
        for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
            size_t u = g.nbr[e];
            if (u == v || constraint[u] != own) continue;
            uint32_t c = memb[u];
            if (c == UNASSIGNED) continue;
            add(c, (double)g.w[e]);
        }
    }
    double weight_to(size_t c) const {
        if (c < slots.size() && slots[c].stamp == generation) return slots[c].weight;
        return 0.0;
    }
};

// MoveScratch (partition.rs:491-551)
struct MoveScratch {
    NeighborWeights weights;
    vector<size_t> order;
    std::deque<size_t> queue;
    vector<char> queued;

    MoveScratch(size_t, size_t slots) { weights.slots.resize(slots); }
    void seed_queue(size_t n, Rng& rng) {
        order.resize(n);
        for (size_t i = 0; i < n; ++i) order[i] = i;
        rng.shuffle(order);
        queue.assign(order.begin(), order.end());
        queued.assign(n, 1);
    }
    const vector<size_t>& shuffled_order(size_t n, Rng& rng) {
        order.resize(n);
        for (size_t i = 0; i < n; ++i) order[i] = i;
        rng.shuffle(order);
        return order;
    }
    bool pop(size_t* v) {
        if (queue.empty()) return false;
        *v = queue.front();
        queue.pop_front();
        queued[*v] = 0;
        return true;
    }
    void push(size_t v) {
        if (!queued[v]) {
            queued[v] = 1;
            queue.push_back(v);
        }
    }
};

// ---------------------------------------------------------------- local moving
// local_move (local_move.rs:39-122)
double local_move(const Graph& g, Partition& p, const Objective& obj, MoveScratch& s, Rng& rng,
                  bool has_limit, double limit) {
    size_t n = g.n();
    if (n == 0) return 0.0;
    s.seed_queue(n, rng);
    double threshold = MIN_GAIN_RELATIVE * std::max(std::fabs(p.total_weight), 1.0);
    double total_gain = 0.0;
    size_t moves = 0;
    size_t budget = n > SIZE_MAX / MAX_MOVES_PER_NODE ? SIZE_MAX : n * MAX_MOVES_PER_NODE;
    size_t v;
    while (s.pop(&v)) {
        InsertContext ctx = InsertContext::for_node(g, v);
        s.weights.ensure_capacity(p.slots() + 1);
        s.weights.collect(g, p.memb, v);
        size_t old = p.membership(v);
        double w_old = s.weights.weight_to(old);
        p.remove_node(v, g, w_old);
        double base = obj.delta_insert(p, ctx, old, w_old);
        size_t best = old;
        double best_gain = base;
        auto fits = [&](size_t c) { return !has_limit || p.wt(c) + ctx.node_weight <= limit; };
        for (size_t i = 0; i < s.weights.touched.size(); ++i) {
            size_t c = s.weights.touched[i];
            if (c == old || !fits(c)) continue;
            double gain = obj.delta_insert(p, ctx, c, s.weights.weight_to(c));
            if (gain > best_gain || (gain == best_gain && c < best)) {
                best = c;
                best_gain = gain;
            }
        }
        size_t empty = p.empty_community();
        if (empty != old && fits(empty)) {
            double gain = obj.delta_insert(p, ctx, empty, 0.0);
            if (gain > best_gain || (gain == best_gain && empty < best)) {
                best = empty;
                best_gain = gain;
            }
        }
        bool accept = best != old && best_gain - base > threshold && moves < budget;
        size_t target = accept ? best : old;
        p.insert_node(v, target, g, s.weights.weight_to(target));
        if (!accept) continue;
        total_gain += best_gain - base;
        moves++;
        for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
            size_t u = g.nbr[e];
            if (u != v && !s.queued[u] && p.membership(u) != target) s.push(u);
        }
    }
    return total_gain;
}

// ---------------------------------------------------------------- refinement
// select (refine.rs:110-153)
bool select_candidate(const vector<std::pair<size_t, double>>& cands, double best_rel,
                      double randomness, Rng& rng, vector<double>& wbuf, size_t* out) {
    if (cands.empty()) return false;
    auto argmax = [&]() {
        size_t best = SIZE_MAX;
        for (const auto& c : cands)
            if (c.second >= best_rel) best = std::min(best, c.first);
        return best;
    };
    if (randomness <= 0.0) {
        *out = argmax();
        return true;
    }
    wbuf.clear();
    for (const auto& c : cands) wbuf.push_back(std::exp((c.second - best_rel) / randomness));
    double total = rust_sum(wbuf.begin(), wbuf.end());
    if (!std::isfinite(total) || total <= 0.0) {
        *out = argmax();
        return true;
    }
    double threshold = rng.next_f64() * total;
    for (size_t i = 0; i < cands.size(); ++i) {
        threshold -= wbuf[i];
        if (threshold <= 0.0) {
            *out = cands[i].first;
            return true;
        }
    }
    *out = cands.back().first;
    return true;
}

// refine (refine.rs:29-103)
Partition refine(const Graph& g, const uint32_t* constraint, const Objective& obj, MoveScratch& s,
                 Rng& rng, bool has_limit, double limit, double randomness) {
    size_t n = g.n();
    Partition r = Partition::singleton(g);
    if (n == 0) return r;
    double mean_edge = g.edge_count > 0 ? g.total_weight / (double)g.edge_count : 1.0;
    randomness = randomness * mean_edge;
    vector<size_t> order = s.shuffled_order(n, rng);
    vector<std::pair<size_t, double>> cands;
    vector<double> wbuf;
    for (size_t v : order) {
        size_t own = r.membership(v);
        if (r.sz(own) != 1) continue;
        InsertContext ctx = InsertContext::for_node(g, v);
        s.weights.ensure_capacity(r.slots() + 1);
        s.weights.collect_constrained(g, r.memb, v, constraint);
        double w_own = s.weights.weight_to(own);
        r.remove_node(v, g, w_own);
        double base = obj.delta_insert(r, ctx, own, w_own);
        cands.clear();
        double best_rel = 0.0;
        for (size_t i = 0; i < s.weights.touched.size(); ++i) {
            size_t c = s.weights.touched[i];
            if (c == own) continue;
            if (has_limit && r.wt(c) + ctx.node_weight > limit) continue;
            double rel = obj.delta_insert(r, ctx, c, s.weights.weight_to(c)) - base;
            if (rel >= 0.0) {
                cands.emplace_back(c, rel);
                best_rel = std::max(best_rel, rel);
            }
        }
        size_t target = own;
        size_t chosen;
        if (select_candidate(cands, best_rel, randomness, rng, wbuf, &chosen)) target = chosen;
        r.insert_node(v, target, g, s.weights.weight_to(target));
    }
    return r;
}

// ---------------------------------------------------------------- driver
// LeidenConfig::validate (mod.rs:117-153)
bool validate_config(const sc_leiden_config& c) {
    double r = c.resolution;
    if (c.objective != SC_OBJECTIVE_RB && c.objective != SC_OBJECTIVE_CPM) {
        std::snprintf(g_err.message, sizeof g_err.message, "invalid configuration: unknown objective");
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    if (!std::isfinite(r) || r < 0.0) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "invalid configuration: resolution must be finite and non-negative, got %g", r);
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    if (c.n_iterations == 0) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "invalid configuration: n_iterations must be at least 1");
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    if (c.max_levels == 0) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "invalid configuration: max_levels must be at least 1");
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    if (c.patience == 0) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "invalid configuration: patience must be at least 1");
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    if (!std::isfinite(c.refine_randomness) || c.refine_randomness < 0.0) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "invalid configuration: refine_randomness must be finite and non-negative, got %g",
                      c.refine_randomness);
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    if (c.has_max_community_weight &&
        (!std::isfinite(c.max_community_weight) || c.max_community_weight <= 0.0)) {
        std::snprintf(g_err.message, sizeof g_err.message,
                      "invalid configuration: max_community_weight must be finite and positive, got %g",
                      c.max_community_weight);
        fail(SC_E_INVALID_CONFIG);
        return false;
    }
    return true;
}

struct PassResult {
    vector<size_t> labels;
    size_t n_clusters;
    double improvement;
};

// run_once (mod.rs:214-289)
PassResult run_once(const Graph& graph, const Objective& obj, Rng& rng,
                    const sc_leiden_config& cfg, const vector<size_t>& initial) {
    size_t n = graph.n();
    Rng level_rng(rng.next_u64());
    const Graph* level = &graph;
    Graph owned;
    Partition p = Partition::from_membership(*level, initial);
    MoveScratch scratch(n, std::max(p.slots(), n) + 1);
    double total_improvement = 0.0;
    vector<size_t> node_at_level(n);
    for (size_t i = 0; i < n; ++i) node_at_level[i] = i;
    bool has_limit = cfg.has_max_community_weight != 0;
    for (uint64_t lvl = 0; lvl < cfg.max_levels; ++lvl) {
        total_improvement += local_move(*level, p, obj, scratch, level_rng, has_limit,
                                        cfg.max_community_weight);
        Partition collapse = cfg.refine
                                 ? refine(*level, p.memb.data(), obj, scratch, level_rng, has_limit,
                                          cfg.max_community_weight, cfg.refine_randomness)
                                 : p;
        collapse.renumber();  // renumber_into_grouping (partition.rs:303-306)
        vector<size_t> grp = collapse.membership_vec();
        size_t n_groups = 0;
        vector<uint64_t> grp64(grp.begin(), grp.end());
        vector<size_t> norm = normalize_groups(grp64.data(), grp64.size(), &n_groups);
        Graph coarse = aggregate(*level, norm, n_groups);
        if (coarse.n() >= level->n()) break;
        vector<size_t> coarse_memb(coarse.n(), 0);
        for (size_t v = 0; v < level->n(); ++v) coarse_memb[collapse.membership(v)] = p.membership(v);
        for (auto& slot : node_at_level) slot = collapse.membership(slot);
        owned = std::move(coarse);
        level = &owned;
        p = Partition::from_membership(*level, coarse_memb);
    }
    p.renumber();
    PassResult r;
    r.labels.resize(n);
    for (size_t i = 0; i < n; ++i) r.labels[i] = p.membership(node_at_level[i]);
    r.n_clusters = p.community_count();
    r.improvement = total_improvement;
    return r;
}

struct OGraphBox {
    Graph g;
};

}  // namespace

struct orc_graph {
    Graph g;
};

extern "C" {

const sc_error_info* orc_last_error(void) { return &g_err; }

int orc_graph_from_edges(uint64_t n_nodes, const uint64_t* from, const uint64_t* to,
                         const double* w, uint64_t n_edges, const double* node_w,
                         orc_graph** out) {
    clear_err();
    vector<double> nw = node_w ? vector<double>(node_w, node_w + n_nodes)
                               : vector<double>(n_nodes, 1.0);
    auto* box = new orc_graph();
    if (!from_edges(from, to, w, n_edges, std::move(nw), box->g)) {
        delete box;
        return g_err.code;
    }
    *out = box;
    return SC_OK;
}

int orc_graph_from_csr(const uint64_t* ptr, uint64_t n_ptr, const uint32_t* nbr, uint64_t n_nbr,
                       const float* w, uint64_t n_w, const double* node_w, uint64_t n_node_w,
                       orc_graph** out) {
    clear_err();
    auto* box = new orc_graph();
    if (!from_csr_parts(vector<uint64_t>(ptr, ptr + n_ptr), vector<uint32_t>(nbr, nbr + n_nbr),
                        vector<float>(w, w + n_w), node_w, n_node_w, box->g)) {
        delete box;
        return g_err.code;
    }
    *out = box;
    return SC_OK;
}

// from_csr_matrix_with_node_weights (csr_network.rs:368-391)
int orc_graph_from_csr_matrix(const uint64_t* row_ptr, uint64_t n_rows, const uint64_t* col,
                              const double* val, uint64_t, const double* node_w,
                              orc_graph** out) {
    clear_err();
    vector<uint64_t> f, t;
    vector<double> ww;
    for (uint64_t r = 0; r < n_rows; ++r)
        for (uint64_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e)
            if (r <= col[e] && val[e] != 0.0) {
                f.push_back(r);
                t.push_back(col[e]);
                ww.push_back(val[e]);
            }
    return orc_graph_from_edges(n_rows, f.data(), t.data(), ww.data(), f.size(), node_w, out);
}

void orc_graph_free(orc_graph* g) { delete g; }

void orc_graph_info(const orc_graph* b, uint64_t* n, uint64_t* entries, uint64_t* edge_count,
                    double* total_weight, int32_t* any_loops) {
    const Graph& g = b->g;
    if (n) *n = g.n();
    if (entries) *entries = g.nbr.size();
    if (edge_count) *edge_count = g.edge_count;
    if (total_weight) *total_weight = g.total_weight;
    if (any_loops) *any_loops = g.any_self_loops ? 1 : 0;
}

void orc_graph_arrays(const orc_graph* b, uint64_t* ptr, uint32_t* nbr, float* w, double* node_w,
                      double* strength) {
    const Graph& g = b->g;
    if (ptr) std::copy(g.ptr.begin(), g.ptr.end(), ptr);
    if (nbr) std::copy(g.nbr.begin(), g.nbr.end(), nbr);
    if (w) std::copy(g.w.begin(), g.w.end(), w);
    if (node_w) std::copy(g.node_w.begin(), g.node_w.end(), node_w);
    if (strength) std::copy(g.strength.begin(), g.strength.end(), strength);
}

// validate_symmetry (csr_network.rs:627-646) with edge_weight (:465-478)
int orc_validate_symmetry(const orc_graph* b) {
    clear_err();
    const Graph& g = b->g;
    auto edge_weight = [&](size_t from, size_t to, double* out) {
        size_t df = g.ptr[from + 1] - g.ptr[from], dt = g.ptr[to + 1] - g.ptr[to];
        size_t s = df <= dt ? from : to, t = df <= dt ? to : from;
        auto bb = g.nbr.begin() + g.ptr[s], ee = g.nbr.begin() + g.ptr[s + 1];
        auto it = std::lower_bound(bb, ee, (uint32_t)t);
        if (it != ee && *it == (uint32_t)t) {
            *out = (double)g.w[it - g.nbr.begin()];
            return true;
        }
        return false;
    };
    for (size_t v = 0; v < g.n(); ++v) {
        for (uint64_t e = g.ptr[v]; e < g.ptr[v + 1]; ++e) {
            size_t u = g.nbr[e];
            double x = (double)g.w[e], back;
            if (!edge_weight(u, v, &back)) {
                std::snprintf(g_err.message, sizeof g_err.message,
                              "malformed CSR input: edge (%zu, %zu) is present but (%zu, %zu) is missing",
                              v, u, u, v);
                return fail(SC_E_INVALID_CSR);
            }
            if (!(std::fabs(back - x) <= 1e-6 * std::max(std::fabs(x), 1.0))) {
                std::snprintf(g_err.message, sizeof g_err.message,
                              "malformed CSR input: edge (%zu, %zu) has weight %g but (%zu, %zu) has %g",
                              v, u, x, u, v, back);
                return fail(SC_E_INVALID_CSR);
            }
        }
    }
    return SC_OK;
}

int orc_aggregate(const orc_graph* b, const uint64_t* groups, uint64_t n, orc_graph** out) {
    clear_err();
    if (n != b->g.n()) {
        g_err.got = n;
        g_err.expected_len = b->g.n();
        return fail(SC_E_MEMBERSHIP_LENGTH_MISMATCH);
    }
    size_t n_groups = 0;
    vector<size_t> norm = n ? normalize_groups(groups, n, &n_groups) : vector<size_t>();
    auto* box = new orc_graph();
    box->g = aggregate(b->g, norm, n_groups);
    *out = box;
    return SC_OK;
}

int orc_partition_stats(const orc_graph* b, const uint64_t* memb, uint64_t n, uint64_t* slots,
                        uint32_t* size, double* weight, double* strength, double* internal,
                        uint64_t capacity) {
    clear_err();
    if (n != b->g.n()) {
        g_err.got = n;
        g_err.expected_len = b->g.n();
        return fail(SC_E_MEMBERSHIP_LENGTH_MISMATCH);
    }
    Partition p = Partition::from_membership(b->g, vector<size_t>(memb, memb + n));
    *slots = p.slots();
    if (p.slots() > capacity) return fail(SC_E_INVALID_ARGUMENT);
    for (size_t c = 0; c < p.slots(); ++c) {
        if (size) size[c] = p.size[c];
        if (weight) weight[c] = p.weight[c];
        if (strength) strength[c] = p.strength[c];
        if (internal) internal[c] = p.internal[c];
    }
    return SC_OK;
}

int orc_quality(const orc_graph* b, const uint64_t* memb, uint64_t n, int32_t objective,
                double resolution, double* out) {
    clear_err();
    if (n != b->g.n()) {
        g_err.got = n;
        g_err.expected_len = b->g.n();
        return fail(SC_E_MEMBERSHIP_LENGTH_MISMATCH);
    }
    Partition p = Partition::from_membership(b->g, vector<size_t>(memb, memb + n));
    Objective obj{objective, resolution};
    *out = obj.quality(p);
    return SC_OK;
}

int orc_modularity(const orc_graph* b, const uint64_t* labels, uint64_t n, double resolution,
                   double* out) {
    clear_err();
    if (n != b->g.n()) {
        g_err.got = n;
        g_err.expected_len = b->g.n();
        return fail(SC_E_MEMBERSHIP_LENGTH_MISMATCH);
    }
    *out = modularity(b->g, labels, resolution);
    return SC_OK;
}

int orc_local_move(const orc_graph* b, uint64_t* memb, uint64_t n, int32_t objective,
                   double resolution, uint64_t seed, int32_t has_max_cw, double max_cw,
                   double* gain_out) {
    clear_err();
    const Graph& g = b->g;
    if (n != g.n()) return fail(SC_E_MEMBERSHIP_LENGTH_MISMATCH);
    Partition p = Partition::from_membership(g, vector<size_t>(memb, memb + n));
    MoveScratch s(n, std::max(p.slots(), (size_t)n) + 1);
    Rng rng(seed);
    Objective obj{objective, resolution};
    double gain = local_move(g, p, obj, s, rng, has_max_cw != 0, max_cw);
    for (size_t v = 0; v < n; ++v) memb[v] = p.memb[v];
    if (gain_out) *gain_out = gain;
    return SC_OK;
}

int orc_refine(const orc_graph* b, const uint32_t* constraint, uint64_t n, int32_t objective,
               double resolution, uint64_t seed, int32_t has_max_cw, double max_cw,
               double randomness, uint64_t* refined_out) {
    clear_err();
    const Graph& g = b->g;
    if (n != g.n()) return fail(SC_E_MEMBERSHIP_LENGTH_MISMATCH);
    MoveScratch s(n, n + 1);
    Rng rng(seed);
    Objective obj{objective, resolution};
    Partition r = refine(g, constraint, obj, s, rng, has_max_cw != 0, max_cw, randomness);
    for (size_t v = 0; v < n; ++v) refined_out[v] = r.memb[v];
    return SC_OK;
}

// leiden (mod.rs:168-204)
int orc_leiden(const orc_graph* b, const sc_leiden_config* cfg, const uint64_t* initial,
               uint64_t* labels_out, uint64_t* n_clusters) {
    clear_err();
    if (!validate_config(*cfg)) return g_err.code;
    const Graph& g = b->g;
    Objective obj{cfg->objective, cfg->resolution};
    Rng rng(cfg->has_seed ? cfg->seed : 0x5eed5eed5eedull);
    size_t n = g.n();
    if (n == 0) {
        *n_clusters = 0;
        return SC_OK;
    }
    vector<size_t> labels(n);
    if (initial) {
        for (size_t i = 0; i < n; ++i) labels[i] = initial[i];
    } else {
        for (size_t i = 0; i < n; ++i) labels[i] = i;
    }
    size_t clusters = n;
    size_t stagnant = 0;
    for (uint64_t it = 0; it < cfg->n_iterations; ++it) {
        PassResult r = run_once(g, obj, rng, *cfg, labels);
        labels = std::move(r.labels);
        clusters = r.n_clusters;
        double scale = std::max(std::fabs(g.total_weight), 1.0);
        if (r.improvement <= cfg->tolerance * scale) {
            stagnant++;
            if (stagnant >= cfg->patience) break;
        } else {
            stagnant = 0;
        }
    }
    for (size_t i = 0; i < n; ++i) labels_out[i] = labels[i];
    *n_clusters = clusters;
    return SC_OK;
}

}  // extern "C"
