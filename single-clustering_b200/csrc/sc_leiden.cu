// sc_leiden.cu — parallel Leiden on sm_100a: local moving, refinement and the
// level / pass driver of src/community_search/leiden/mod.rs:168-289.
//
// Local moving (local_move.rs:39-122) becomes synchronous sweeps over the
// active nodes, split into B hash batches. Inside a batch every node scores
// its candidates against a snapshot (decide kernels), then one kernel commits
// the moves (apply). A move into a singleton community whose sole member is
// moving in the same batch is cancelled — for a mutual pair the lower seeded
// priority yields — so two singletons never swap past each other.
//
// Community aggregates (K_c, node weight n_c, size) are int64 fixed point:
// integer atomics are associative, so a fixed seed gives bit-identical runs.
// In the exact regime the fixed-point values are the f64 values themselves.
//
// Degree buckets: a group of G = 8 / 16 / 32 lanes per node for degree <= G
// (neighbour communities merged with __match_any_sync, no shared memory);
// one 256-thread block per node above that, with an open-addressing hash in
// shared memory (global memory past its capacity).
#include <random>

#include "sc_prims.cuh"

namespace sc {

namespace {

constexpr unsigned TB = 256;
constexpr int NBUCKET = 6;          // G8, G16, G32, warp (shared hash), block (shared hash), hub (global hash)
constexpr uint32_t WARP_DEGREE = 256;  // largest degree of the warp-per-node bucket
constexpr int WCAP = 2 * WARP_DEGREE;  // per-warp shared hash entries
constexpr int WARPS_PER_BLOCK = 4;
constexpr int HCAP_SMEM = 2 * HUB_DEGREE;  // shared hash entries per block (u32 key + i64 val): 24 KB
constexpr int LM_BATCHES = 2;
constexpr int RF_BATCHES = 8;
constexpr int MAX_SLOTS = 64;  // (batch, bucket) counters, cursors and offsets are sized for this
static_assert(LM_BATCHES * NBUCKET <= MAX_SLOTS && RF_BATCHES * NBUCKET <= MAX_SLOTS,
              "batch x bucket slots exceed the fixed counter arrays");
constexpr int MAX_SWEEPS = 100;
constexpr uint32_t EMPTYK = 0xFFFFFFFFu;

struct Params {
    // graph
    const uint64_t* ptr;
    const uint32_t* nbr;
    const float* w;
    const double* strength;
    const double* node_w;
    const double* self_loop;
    // partition being changed (working partition or refined partition)
    uint32_t* memb;
    long long* Kf;
    long long* Wf;
    uint32_t* csize;
    // refinement only: the constraint (working membership)
    const uint32_t* constraint;
    // decisions
    uint32_t* tgt;
    uint32_t* hint;
    uint32_t* from;
    long long* dgain;
    uint32_t* epoch;
    uint32_t cur;
    uint64_t S0;           // fresh-community id base (local moving)
    // objective
    int objective;
    double gamma, four_m, thr;
    double scale, inv_scale;    // 2^F, 2^-F for edge-weight quantities
    double nscale, inv_nscale;  // same for node weights
    int has_limit;
    double limit;
    int need_nc;                // community node weights are read (CPM, or a weight cap)
    double theta;               // refinement randomness (<= 0: argmax)
    uint64_t seed;
    uint32_t* status;
    unsigned long long* counters;  // [0] moves, [1] Σdeg, [2] Σcand, [3] nodes
    long long* gain_acc;
    // max_community_weight: one joiner per target community per batch (the
    // highest claim key wins), so a community never passes the cap
    unsigned long long* claim;
    uint32_t* moved;  // epoch in which the node last committed a move
    // batched runs over a disjoint union of instances (nullptr: one instance,
    // the scalars above): each node's instance, the instances' settings, and
    // each instance's gain accumulator
    const uint32_t* inst;
    const struct InstCfg* icfg;
    long long* gain_inst;
};

// Settings of one instance of a batched run, for the current level.
struct InstCfg {
    double gamma, four_m, thr, theta;
    uint64_t seed;    // the instance's seed for this level (local moving or refinement)
    uint32_t base;    // the instance's first node id in the union at this level
    uint32_t frozen;  // 1: the instance takes no decisions (it stopped, as its own run would)
};

// What a node's decisions read: the run's scalars, or its instance's. Hashes
// and tie rules see instance-local ids (node id - base), so a node of a batched
// run draws exactly what it draws in its instance's own run.
struct NodeCfg {
    double gamma, four_m, thr, theta;
    uint64_t seed;
    uint32_t base;
};

template <bool MULTI>
__device__ __forceinline__ NodeCfg node_cfg(const Params& p, uint32_t v) {
    if (!MULTI) return NodeCfg{p.gamma, p.four_m, p.thr, p.theta, p.seed, 0u};
    const InstCfg& c = p.icfg[p.inst[v]];
    return NodeCfg{c.gamma, c.four_m, c.thr, c.theta, c.seed, c.base};
}

__device__ __forceinline__ long long to_fix(double x, double inv) { return __double2ll_rn(__dmul_rn(x, inv)); }
__device__ __forceinline__ double from_fix(long long q, double s) { return __dmul_rn(__ll2double_rn(q), s); }

// Rb::delta_insert (objective.rs:91-106) / Cpm::delta_insert (:158-169)
__device__ __forceinline__ double gain_of(const Params& p, const NodeCfg& q, double wto, double sl, double k,
                                          double kc, double a, double nc) {
    if (p.objective == SC_OBJECTIVE_RB) {
        if (q.four_m == 0.0) return 0.0;
        return __dsub_rn(__dadd_rn(wto, sl),
                         __ddiv_rn(__dmul_rn(__dmul_rn(q.gamma, k), __dadd_rn(__dmul_rn(2.0, kc), k)),
                                   q.four_m));
    }
    return __dsub_rn(__dadd_rn(wto, sl),
                     __ddiv_rn(__dmul_rn(__dmul_rn(q.gamma, a),
                                         __dsub_rn(__dadd_rn(__dmul_rn(2.0, nc), a), 1.0)),
                               2.0));
}

__device__ __forceinline__ bool better(double g, uint32_t c, double bg, uint32_t bc) {
    return g > bg || (g == bg && c < bc);
}

__device__ __forceinline__ uint64_t prio(uint64_t seed, uint32_t ep, uint32_t v) {
    return hash3(seed ^ 0xA5A5A5A5DEADBEEFull, ep, v);
}

// Whether node x's move (decided in epoch p.cur) is cancelled. x and the
// member h of its target are nodes of the same instance.
template <bool MULTI>
__device__ __forceinline__ bool cancelled(const Params& p, uint32_t x) {
    uint32_t h = p.hint[x];
    if (h == NONE32) return false;
    if (p.epoch[h] != p.cur) return false;  // the target's member is not moving
    if (p.hint[h] == x) {                   // mutual: the lower priority yields
        const NodeCfg q = node_cfg<MULTI>(p, x);
        uint64_t px = prio(q.seed, p.cur, x - q.base), ph = prio(q.seed, p.cur, h - q.base);
        return px < ph || (px == ph && x < h);
    }
    return true;
}

template <bool MULTI>
__device__ __forceinline__ unsigned long long claim_key(const Params& p, uint32_t v) {
    const NodeCfg q = node_cfg<MULTI>(p, v);
    return ((unsigned long long)p.cur << 40) | ((prio(q.seed ^ 0x77ull, p.cur, v - q.base) & 0xFFull) << 32) | v;
}

// Whether node x's move is dropped: cancelled, or beaten to a capped community.
template <bool MULTI>
__device__ __forceinline__ bool lost(const Params& p, uint32_t x) {
    if (cancelled<MULTI>(p, x)) return true;
    return p.has_limit && p.claim[p.tgt[x]] != claim_key<MULTI>(p, x);
}

__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t a, uint64_t b) {
    return (double)(hash3(seed ^ 0x5151515151515151ull, a, b) >> 11) * 0x1.0p-53;
}

// Refinement's randomised choice (refine.rs:110-153) draws candidate c with
// probability exp(rel_c / theta) / sum. Gumbel-max draws from the same
// distribution: argmax_c rel_c / theta + G_c with G_c = -log(-log U_c), U_c
// uniform in (0, 1) from a hash of (seed, epoch, node, c). The result does not
// depend on the order candidates are visited in, so no candidate list or sort
// is needed. theta <= 0 is the deterministic argmax (ties to the lower id).
// v and c are instance-local ids (refined community ids are node ids).
__device__ __forceinline__ double refine_key(const Params& p, const NodeCfg& q, double rel, uint32_t v,
                                             uint32_t c) {
    if (q.theta <= 0.0) return rel;
    uint64_t h = hash3(q.seed ^ 0x5151515151515151ull, ((uint64_t)p.cur << 32) | v, c);
    double u = ((double)(h >> 11) + 0.5) * 0x1.0p-53;
    return __dadd_rn(__ddiv_rn(rel, q.theta), -log(-log(u)));
}

// Read-only load (ld.global.nc): the decide kernels never write the graph, the
// membership or the community aggregates they read; only the commit kernels do.
template <class T>
__device__ __forceinline__ T ro(const T* a) {
    return __ldg(a);
}

// Warp-aggregated counter add.
__device__ __forceinline__ void warp_add(unsigned long long* ctr, unsigned long long x) {
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(ctr, x);
}

// ------------------------------------------------------------ small-degree decide
// REFINE=false: local moving. REFINE=true: refinement (singletons only, inside
// the constraint, randomised choice among non-negative candidates).
template <int G, bool REFINE, bool MULTI>
__global__ void __launch_bounds__(TB, 4) k_decide_small(Params p, const uint32_t* __restrict__ list,
                                                        const uint64_t* __restrict__ lbeg,
                                                        const uint32_t* __restrict__ ldeg, uint32_t count) {
    const unsigned FULL = 0xFFFFFFFFu;
    __shared__ unsigned long long s_acc[TB];
    const int lane = threadIdx.x & 31;
    const int sub = lane & (G - 1);
    const int gw = lane / G;  // group within warp
    const int gbase = gw * G;
    const unsigned gmask = (G == 32) ? FULL : (((1u << G) - 1u) << gbase);
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const int per_warp = 32 / G;
    unsigned long long sdeg = 0, scand = 0, snodes = 0;

    // Software pipeline: the list entry and this lane's neighbour id / weight of
    // the group's next node are loaded one iteration ahead, so their round trip
    // overlaps the current node's membership gathers and scoring.
    const uint64_t step = nwarps * per_warp;
    uint32_t nv = 0, nu = 0;
    uint64_t nb = 0;
    int ndeg = 0;
    float nwt = 0.0f;
    auto fetch = [&](uint64_t w0) {
        const uint64_t i = w0 + gw;
        nv = 0, nu = 0, nb = 0, ndeg = 0, nwt = 0.0f;
        if (i < count) {
            nv = ro(list + i);
            nb = ro(lbeg + i);
            ndeg = (int)ro(ldeg + i);
            if (sub < ndeg) {
                nu = ro(p.nbr + (nb + sub));
                nwt = ro(p.w + (nb + sub));
            }
        }
    };
    fetch(warp * per_warp);
    for (uint64_t wb = warp * per_warp; wb < count; wb += step) {
        const uint64_t i = wb + gw;
        const bool have = i < count;
        const uint32_t v = nv;
        const int deg = ndeg;
        const uint32_t u_next = nu;
        const float wt_next = nwt;
        fetch(wb + step);
        const NodeCfg q = node_cfg<MULTI>(p, v);
        const uint32_t own = have ? ro(p.memb + (v)) : 0;
        bool eligible = have;
        if (REFINE && have) eligible = ro(p.csize + (own)) == 1;  // refine.rs:60-62
        bool valid = eligible && sub < deg;
        const uint32_t u = valid ? u_next : 0;
        const float wt = valid ? wt_next : 0.0f;
        valid = valid && u != v;
        if (REFINE && valid) valid = ro(p.constraint + (u)) == ro(p.constraint + (v));
        const uint32_t cu = valid ? ro(p.memb + (u)) : NONE32;
        const long long wf = valid ? to_fix((double)wt, p.inv_scale) : 0;
        const uint64_t key = valid ? (((uint64_t)gw << 32) | cu) : (0xFFFFFFFF00000000ull | (uint64_t)lane);
        const unsigned mm = __match_any_sync(FULL, key);
        const bool leader = valid && (__ffs(mm) - 1 == lane);
        // per-community sums: every lane adds into its group leader's shared slot
        // (integer adds, so the order does not matter); only leaders read theirs
        s_acc[threadIdx.x] = 0ull;
        __syncwarp();
        if (valid) atomicAdd(&s_acc[(threadIdx.x & ~31u) + (unsigned)(__ffs(mm) - 1)], (unsigned long long)wf);
        __syncwarp();
        const long long acc = (long long)s_acc[threadIdx.x];
        __syncwarp();
        // node quantities (identical in all lanes of the group)
        long long kf = 0, af = 0;
        double sl = 0.0;
        if (eligible) {
            kf = to_fix(ro(p.strength + (v)), p.inv_scale);
            af = to_fix(ro(p.node_w + (v)), p.inv_nscale);
            sl = ro(p.self_loop + (v));
        }
        const double k = from_fix(kf, p.scale), a = from_fix(af, p.nscale);
        // weight to the own community
        unsigned ob = __ballot_sync(FULL, leader && cu == own) & gmask;
        long long wof = __shfl_sync(FULL, acc, ob ? (__ffs(ob) - 1) : lane);
        if (!ob) wof = 0;
        double base = 0.0;
        if (eligible) {
            base = gain_of(p, q, from_fix(wof, p.scale), sl, k, from_fix(ro(p.Kf + (own)) - kf, p.scale), a,
                           (p.need_nc ? from_fix(ro(p.Wf + (own)) - af, p.nscale) : 0.0));
        }
        // candidates held by leader lanes
        double g = -INFINITY;
        uint32_t c = NONE32, cu_member = NONE32;
        bool cand = false;
        if (leader && cu != own) {
            double nc = (p.need_nc ? from_fix(ro(p.Wf + (cu)), p.nscale) : 0.0);
            if (!p.has_limit || __dadd_rn(nc, a) <= p.limit) {
                g = gain_of(p, q, from_fix(acc, p.scale), sl, k, from_fix(ro(p.Kf + (cu)), p.scale), a, nc);
                if (REFINE) {
                    double rel = __dsub_rn(g, base);
                    if (rel >= 0.0) {  // `>=` takes ties (refine.rs:91-95)
                        cand = true;
                        g = refine_key(p, q, rel, v - q.base, cu - q.base);
                    } else {
                        g = -INFINITY;
                    }
                } else {
                    cand = true;
                }
                if (cand) {
                    c = cu;
                    cu_member = u;
                }
            }
        }
        if (sub == 0 && eligible) {
            snodes += 1;
            sdeg += (unsigned long long)deg;
        }
        scand += (leader && cu != own) ? 1ull : 0ull;
        // argmax over the group: higher key, then lower id
#pragma unroll
        for (int o = G / 2; o; o >>= 1) {
            double og = __shfl_xor_sync(FULL, g, o);
            uint32_t oc = __shfl_xor_sync(FULL, c, o);
            uint32_t om = __shfl_xor_sync(FULL, cu_member, o);
            if (better(og, oc, g, c)) {
                g = og;
                c = oc;
                cu_member = om;
            }
        }
        if (!REFINE) {
            if (sub == 0 && eligible) {
                uint32_t best = own;
                double bg = base;
                if (c != NONE32 && better(g, c, bg, best)) {
                    best = c;
                    bg = g;
                }
                // one empty community per node (local_move.rs:92-100)
                const uint32_t fresh = (uint32_t)(p.S0 + v);
                if (fresh != own && ro(p.csize + (own)) > 1 && ro(p.csize + (fresh)) == 0 &&
                    (!p.has_limit || a <= p.limit)) {
                    double ge = gain_of(p, q, 0.0, sl, k, 0.0, a, 0.0);
                    if (better(ge, fresh, bg, best)) {
                        best = fresh;
                        bg = ge;
                    }
                }
                double d = __dsub_rn(bg, base);
                if (best != own && d > q.thr) {
                    p.tgt[v] = best;
                    p.from[v] = own;
                    p.dgain[v] = to_fix(d, p.inv_scale);
                    p.hint[v] = (best != fresh && ro(p.csize + (best)) == 1) ? cu_member : NONE32;
                    p.epoch[v] = p.cur;
                }
            }
        } else if (sub == 0 && eligible && c != NONE32) {
            p.tgt[v] = c;
            p.from[v] = own;
            p.dgain[v] = 0;
            p.hint[v] = (ro(p.csize + (c)) == 1) ? cu_member : NONE32;
            p.epoch[v] = p.cur;
        }
    }
    warp_add(p.counters + 1, sdeg);
    warp_add(p.counters + 2, scand);
    warp_add(p.counters + 3, snodes);
}

// ------------------------------------------------------------ large-degree decide
__device__ __forceinline__ uint32_t hslot(uint32_t c, uint32_t mask) {
    return (c * 0x9E3779B1u) & mask;
}

__device__ bool hinsert(uint32_t* keys, long long* vals, uint32_t mask, uint32_t c, long long x,
                        uint32_t* status) {
    uint32_t h = hslot(c, mask);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        uint32_t k = keys[h];
        if (k == c) {
            atomicAdd((unsigned long long*)(vals + h), (unsigned long long)x);
            return true;
        }
        if (k == EMPTYK) {
            uint32_t prev = atomicCAS(keys + h, EMPTYK, c);
            if (prev == EMPTYK || prev == c) {
                atomicAdd((unsigned long long*)(vals + h), (unsigned long long)x);
                return true;
            }
        }
        h = (h + 1) & mask;
    }
    atomicOr(status, DEV_OVERFLOW);
    return false;
}

// hinsert that also appends every slot it claims to `list` (the distinct keys,
// in no particular order; the caller sized `list` for all of them).
__device__ void hinsert_listed(uint32_t* keys, long long* vals, uint32_t mask, uint32_t c, long long x,
                               uint32_t* status, uint32_t* list, uint32_t* count, uint32_t list_cap) {
    uint32_t h = hslot(c, mask);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        uint32_t k = keys[h];
        if (k == EMPTYK) {
            const uint32_t prev = atomicCAS(keys + h, EMPTYK, c);
            if (prev == EMPTYK) {
                const uint32_t i = atomicAdd(count, 1u);
                if (i < list_cap) list[i] = h;
                else atomicOr(status, DEV_OVERFLOW);
            }
            k = prev == EMPTYK ? c : prev;
        }
        if (k == c) {
            atomicAdd((unsigned long long*)(vals + h), (unsigned long long)x);
            return;
        }
        h = (h + 1) & mask;
    }
    atomicOr(status, DEV_OVERFLOW);
}

__device__ long long hlookup(const uint32_t* keys, const long long* vals, uint32_t mask, uint32_t c) {
    uint32_t h = hslot(c, mask);
    for (uint32_t probe = 0; probe <= mask; ++probe) {
        uint32_t k = keys[h];
        if (k == c) return vals[h];
        if (k == EMPTYK) return 0;
        h = (h + 1) & mask;
    }
    return 0;
}

// Block-wide argmax of (g, c) with ties to the lower id.
__device__ void block_argmax(double& g, uint32_t& c, double* sg, uint32_t* sc) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o; o >>= 1) {
        double og = __shfl_xor_sync(0xFFFFFFFFu, g, o);
        uint32_t oc = __shfl_xor_sync(0xFFFFFFFFu, c, o);
        if (better(og, oc, g, c)) {
            g = og;
            c = oc;
        }
    }
    if (lane == 0) {
        sg[wid] = g;
        sc[wid] = c;
    }
    __syncthreads();
    if (wid == 0) {
        int nw = blockDim.x >> 5;
        g = lane < nw ? sg[lane] : -INFINITY;
        c = lane < nw ? sc[lane] : NONE32;
        for (int o = 16; o; o >>= 1) {
            double og = __shfl_xor_sync(0xFFFFFFFFu, g, o);
            uint32_t oc = __shfl_xor_sync(0xFFFFFFFFu, c, o);
            if (better(og, oc, g, c)) {
                g = og;
                c = oc;
            }
        }
        if (lane == 0) {
            sg[0] = g;
            sc[0] = c;
        }
    }
    __syncthreads();
    g = sg[0];
    c = sc[0];
    __syncthreads();
}

// One warp per node of degree 33..WARP_DEGREE: an open-addressing hash of
// neighbour communities in this warp's slice of shared memory, gains scored
// by every lane over its slots, warp argmax.
template <bool REFINE, bool MULTI>
__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK) k_decide_warp(Params p, const uint32_t* __restrict__ list,
                                                                      const uint64_t* __restrict__ lbeg,
                                                                      const uint32_t* __restrict__ ldeg,
                                                                      uint32_t count) {
    __shared__ uint32_t s_keys[WARPS_PER_BLOCK][WCAP];
    __shared__ long long s_vals[WARPS_PER_BLOCK][WCAP];
    __shared__ uint32_t s_list[WARPS_PER_BLOCK][WARP_DEGREE];  // claimed slots: the distinct communities
    __shared__ uint32_t s_cnt[WARPS_PER_BLOCK];
    const unsigned FULL = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    uint32_t* keys = s_keys[wib];
    long long* vals = s_vals[wib];
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long sdeg = 0, scand = 0, snodes = 0;
    // Software pipeline: the next node's list entry is loaded at the top of an
    // iteration, its first 32 neighbour ids / weights once this node's entries
    // are in the table; both round trips overlap this node's work.
    uint32_t nv = 0, nu = 0, ndeg = 0;
    uint64_t nb = 0;
    float nw = 0.0f;
    auto fetch_head = [&](uint64_t i) {
        nv = 0, nb = 0, ndeg = 0;
        if (i < count) {
            nv = ro(list + i);
            nb = ro(lbeg + i);
            ndeg = ro(ldeg + i);
        }
    };
    auto fetch_chunk = [&]() {
        nu = 0, nw = 0.0f;
        if ((uint32_t)lane < ndeg) {
            nu = ro(p.nbr + (nb + lane));
            nw = ro(p.w + (nb + lane));
        }
    };
    fetch_head(warp);
    fetch_chunk();
    for (uint64_t i = warp; i < count; i += nwarps) {
        const uint32_t v = nv;
        const uint64_t b = nb, e = b + ndeg;
        const uint32_t deg = ndeg;
        const uint32_t u_first = nu;
        const float w_first = nw;
        fetch_head(i + nwarps);
        const NodeCfg q = node_cfg<MULTI>(p, v);
        const uint32_t own = ro(p.memb + (v));
        if (REFINE && ro(p.csize + (own)) != 1) {  // warp-uniform
            fetch_chunk();
            continue;
        }
        uint32_t cap = 64;
        while (cap < 2 * deg) cap <<= 1;
        if (cap > (uint32_t)WCAP) {  // not this bucket's node
            if (lane == 0) atomicOr(p.status, DEV_OVERFLOW);
            fetch_chunk();
            continue;
        }
        const uint32_t mask = cap - 1;
        for (uint32_t s = lane; s < cap; s += 32) {
            keys[s] = EMPTYK;
            vals[s] = 0;
        }
        if (lane == 0) s_cnt[wib] = 0;
        __syncwarp();
        const uint32_t cv = REFINE ? ro(p.constraint + (v)) : 0;
        for (uint64_t base0 = b; base0 < e; base0 += 32) {  // warp-uniform trip count
            const uint64_t j = base0 + lane;
            const bool first = base0 == b;
            bool ok = j < e;
            uint32_t u = 0;
            float wj = 0.0f;
            if (ok) {
                u = first ? u_first : ro(p.nbr + (j));
                wj = first ? w_first : ro(p.w + (j));
            }
            ok = ok && u != v;
            if (REFINE && ok) ok = ro(p.constraint + (u)) == cv;
            const uint32_t cu = ok ? ro(p.memb + (u)) : 0u;
            const uint64_t key = ok ? (uint64_t)cu : (0xFFFFFFFF00000000ull | lane);
            const unsigned peers = __match_any_sync(FULL, key);
            const long long x = peer_sum(peers, ok ? to_fix((double)wj, p.inv_scale) : 0ll);
            if (ok && __ffs(peers) - 1 == lane)
                hinsert_listed(keys, vals, mask, cu, x, p.status, s_list[wib], &s_cnt[wib], WARP_DEGREE);
        }
        fetch_chunk();
        __syncwarp();
        const uint32_t ndist = min(s_cnt[wib], WARP_DEGREE);
        const long long kf = to_fix(ro(p.strength + (v)), p.inv_scale);
        const long long af = to_fix(ro(p.node_w + (v)), p.inv_nscale);
        const double k = from_fix(kf, p.scale), a = from_fix(af, p.nscale), sl = ro(p.self_loop + (v));
        const long long wof = hlookup(keys, vals, mask, own);
        const double base = gain_of(p, q, from_fix(wof, p.scale), sl, k, from_fix(ro(p.Kf + (own)) - kf, p.scale), a,
                                    (p.need_nc ? from_fix(ro(p.Wf + (own)) - af, p.nscale) : 0.0));
        double g = -INFINITY;
        uint32_t c = NONE32;
        uint32_t lc = 0;
        for (uint32_t t = lane; t < ndist; t += 32) {  // the distinct communities only
            const uint32_t s = s_list[wib][t];
            const uint32_t cu = keys[s];
            if (cu == own) continue;
            lc++;
            const double nc = (p.need_nc ? from_fix(ro(p.Wf + (cu)), p.nscale) : 0.0);
            if (p.has_limit && __dadd_rn(nc, a) > p.limit) continue;
            double gg = gain_of(p, q, from_fix(vals[s], p.scale), sl, k, from_fix(ro(p.Kf + (cu)), p.scale), a, nc);
            if (REFINE) {
                const double rel = __dsub_rn(gg, base);
                if (!(rel >= 0.0)) continue;
                gg = refine_key(p, q, rel, v - q.base, cu - q.base);
            }
            if (better(gg, cu, g, c)) {
                g = gg;
                c = cu;
            }
        }
        for (int o = 16; o; o >>= 1) {
            const double og = __shfl_xor_sync(FULL, g, o);
            const uint32_t oc = __shfl_xor_sync(FULL, c, o);
            if (better(og, oc, g, c)) {
                g = og;
                c = oc;
            }
        }
        scand += lc;
        uint32_t target = NONE32;
        long long dg = 0;
        if (!REFINE) {
            uint32_t best = own;
            double bg = base;
            if (c != NONE32 && better(g, c, bg, best)) {
                best = c;
                bg = g;
            }
            const uint32_t fresh = (uint32_t)(p.S0 + v);
            if (fresh != own && ro(p.csize + (own)) > 1 && ro(p.csize + (fresh)) == 0 && (!p.has_limit || a <= p.limit)) {
                const double ge = gain_of(p, q, 0.0, sl, k, 0.0, a, 0.0);
                if (better(ge, fresh, bg, best)) {
                    best = fresh;
                    bg = ge;
                }
            }
            const double d = __dsub_rn(bg, base);
            if (best != own && d > q.thr) {
                target = best;
                dg = to_fix(d, p.inv_scale);
            }
        } else {
            target = c;
        }
        // the member of a singleton target, for conflict detection
        uint32_t member = NONE32;
        if (target != NONE32 && ro(p.csize + (target)) == 1) {
            for (uint64_t base0 = b; base0 < e; base0 += 32) {
                const uint64_t j = base0 + lane;
                const uint32_t u = j < e ? ro(p.nbr + (j)) : v;
                const bool hit = u != v && ro(p.memb + (u)) == target;
                if (hit) member = u;
                if (__ballot_sync(FULL, hit)) break;
            }
            for (int o = 16; o; o >>= 1) member = min(member, __shfl_xor_sync(FULL, member, o));
        }
        if (lane == 0) {
            snodes += 1;
            sdeg += deg;
            if (target != NONE32) {
                p.tgt[v] = target;
                p.from[v] = own;
                p.dgain[v] = dg;
                p.hint[v] = member;
                p.epoch[v] = p.cur;
            }
        }
        __syncwarp();
    }
    warp_add(p.counters + 1, sdeg);
    warp_add(p.counters + 2, scand);
    warp_add(p.counters + 3, snodes);
}

// One block per node. HUB = false: degree <= HUB_DEGREE, hash table in shared
// memory. HUB = true: the table lives in this block's slice of the global
// scratch (gcap entries), which the host sized for the largest degree; the
// grid never exceeds the number of slices.
template <bool REFINE, bool HUB, bool MULTI>
__global__ void __launch_bounds__(TB) k_decide_block(Params p, const uint32_t* __restrict__ list,
                                                     const uint64_t* __restrict__ lbeg,
                                                     const uint32_t* __restrict__ ldeg, uint32_t count,
                                                     uint32_t* gkeys, long long* gvals, uint64_t gcap) {
    extern __shared__ __align__(16) unsigned char smem[];
    long long* s_vals = (long long*)smem;
    uint32_t* s_keys = (uint32_t*)(smem + HCAP_SMEM * sizeof(long long));
    __shared__ double red_g[32];
    __shared__ uint32_t red_c[32];
    __shared__ uint32_t s_member, s_target;

    unsigned long long sdeg = 0, scand = 0, snodes = 0;
    for (uint64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t v = ro(list + (i));
        const NodeCfg q = node_cfg<MULTI>(p, v);
        const uint64_t b = ro(lbeg + i), e = b + ro(ldeg + i);
        const uint32_t deg = (uint32_t)(e - b);
        const uint32_t own = ro(p.memb + (v));
        if (REFINE && ro(p.csize + (own)) != 1) continue;  // uniform over the block
        uint32_t cap = 64;
        while (cap < 2 * deg) cap <<= 1;
        uint32_t* keys;
        long long* vals;
        if (!HUB) {
            if (cap > (uint32_t)HCAP_SMEM) {  // not this bucket's node: skip it, flag it
                if (threadIdx.x == 0) atomicOr(p.status, DEV_OVERFLOW);
                continue;
            }
            keys = s_keys;
            vals = s_vals;
        } else {
            if (cap > gcap) {
                if (threadIdx.x == 0) atomicOr(p.status, DEV_OVERFLOW);
                continue;
            }
            keys = gkeys + (uint64_t)blockIdx.x * gcap;
            vals = gvals + (uint64_t)blockIdx.x * gcap;
        }
        const uint32_t mask = cap - 1;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            keys[s] = EMPTYK;
            vals[s] = 0;
        }
        __syncthreads();
        const uint32_t cv = REFINE ? ro(p.constraint + (v)) : 0;
        {
            const unsigned lane = threadIdx.x & 31u;
            // each warp walks its own 32-entry chunks: trip counts are warp-uniform
            for (uint64_t base0 = b + (threadIdx.x & ~31u); base0 < e; base0 += blockDim.x) {
                const uint64_t j = base0 + lane;
                bool ok = j < e;
                const uint32_t u = ok ? ro(p.nbr + (j)) : 0u;
                ok = ok && u != v;
                if (REFINE && ok) ok = ro(p.constraint + (u)) == cv;
                const uint32_t cu = ok ? ro(p.memb + (u)) : 0u;
                const uint64_t key = ok ? (uint64_t)cu : (0xFFFFFFFF00000000ull | lane);
                const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
                const long long x = peer_sum(peers, ok ? to_fix((double)ro(p.w + (j)), p.inv_scale) : 0ll);
                if (ok && __ffs(peers) - 1 == (int)lane) hinsert(keys, vals, mask, cu, x, p.status);
            }
        }
        __syncthreads();
        const long long kf = to_fix(ro(p.strength + (v)), p.inv_scale);
        const long long af = to_fix(ro(p.node_w + (v)), p.inv_nscale);
        const double k = from_fix(kf, p.scale), a = from_fix(af, p.nscale), sl = ro(p.self_loop + (v));
        const long long wof = hlookup(keys, vals, mask, own);
        const double base = gain_of(p, q, from_fix(wof, p.scale), sl, k, from_fix(ro(p.Kf + (own)) - kf, p.scale),
                                    a, (p.need_nc ? from_fix(ro(p.Wf + (own)) - af, p.nscale) : 0.0));
        double g = -INFINITY;
        uint32_t c = NONE32;
        uint32_t lc = 0;
        for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) {
            uint32_t cu = keys[s];
            if (cu == EMPTYK || cu == own) continue;
            lc++;
            double nc = (p.need_nc ? from_fix(ro(p.Wf + (cu)), p.nscale) : 0.0);
            if (p.has_limit && __dadd_rn(nc, a) > p.limit) continue;
            double gg = gain_of(p, q, from_fix(vals[s], p.scale), sl, k, from_fix(ro(p.Kf + (cu)), p.scale), a, nc);
            if (REFINE) {
                double rel = __dsub_rn(gg, base);
                if (!(rel >= 0.0)) continue;
                gg = refine_key(p, q, rel, v - q.base, cu - q.base);
            }
            if (better(gg, cu, g, c)) {
                g = gg;
                c = cu;
            }
        }
        scand += lc;
        if (threadIdx.x == 0) {
            snodes += 1;
            sdeg += deg;
        }
        block_argmax(g, c, red_g, red_c);
        if (threadIdx.x == 0) {
            uint32_t best = own;
            double bg = base;
            if (!REFINE) {
                if (c != NONE32 && better(g, c, bg, best)) {
                    best = c;
                    bg = g;
                }
                const uint32_t fresh = (uint32_t)(p.S0 + v);
                if (fresh != own && ro(p.csize + (own)) > 1 && ro(p.csize + (fresh)) == 0 &&
                    (!p.has_limit || a <= p.limit)) {
                    double ge = gain_of(p, q, 0.0, sl, k, 0.0, a, 0.0);
                    if (better(ge, fresh, bg, best)) {
                        best = fresh;
                        bg = ge;
                    }
                }
                double d = __dsub_rn(bg, base);
                s_target = (best != own && d > q.thr) ? best : NONE32;
                if (s_target != NONE32) p.dgain[v] = to_fix(d, p.inv_scale);
            } else {
                s_target = c;  // NONE32 when no candidate has rel >= 0
                p.dgain[v] = 0;
            }
            if (s_target != NONE32) {
                p.tgt[v] = s_target;
                p.from[v] = own;
                p.epoch[v] = p.cur;
            }
            s_member = NONE32;
        }
        __syncthreads();
        // the member of a singleton target, for conflict detection
        const uint32_t target = s_target;
        if (target != NONE32) {
            if (ro(p.csize + (target)) == 1) {
                for (uint64_t j = b + threadIdx.x; j < e; j += blockDim.x) {
                    uint32_t u = ro(p.nbr + (j));
                    if (u != v && ro(p.memb + (u)) == target) s_member = u;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) p.hint[v] = s_member;
        }
        __syncthreads();
    }
    // block-level counter flush (thread 0 holds the node and degree counts)
    atomicAdd(p.counters + 2, scand);
    if (threadIdx.x == 0) {
        atomicAdd(p.counters + 1, sdeg);
        atomicAdd(p.counters + 3, snodes);
    }
}

// ------------------------------------------------------------ commit
template <bool REFINE, bool MULTI>
__global__ void k_apply(Params p, const uint32_t* __restrict__ list, uint32_t count) {
    unsigned long long nmoves = 0;
    long long gsum = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = list[i];
        if (p.epoch[v] != p.cur) continue;
        if (lost<MULTI>(p, v)) continue;
        const uint32_t t = p.tgt[v], old = p.from[v];
        const long long kf = to_fix(p.strength[v], p.inv_scale);
        p.memb[v] = t;
        atomicAdd((unsigned long long*)(p.Kf + old), (unsigned long long)(-kf));
        atomicAdd((unsigned long long*)(p.Kf + t), (unsigned long long)kf);
        if (p.need_nc) {  // community node weights: read only by CPM and the weight cap
            const long long af = to_fix(p.node_w[v], p.inv_nscale);
            atomicAdd((unsigned long long*)(p.Wf + old), (unsigned long long)(-af));
            atomicAdd((unsigned long long*)(p.Wf + t), (unsigned long long)af);
        }
        atomicSub(p.csize + old, 1u);
        atomicAdd(p.csize + t, 1u);
        nmoves++;
        if (MULTI) {
            if (p.dgain[v]) atomicAdd((unsigned long long*)(p.gain_inst + p.inst[v]), (unsigned long long)p.dgain[v]);
        } else {
            gsum += p.dgain[v];
        }
        if (!REFINE) p.moved[v] = p.cur;
    }
    warp_add(p.counters + 0, nmoves);
    for (int o = 16; o; o >>= 1) gsum += __shfl_xor_sync(0xFFFFFFFFu, gsum, o);
    if ((threadIdx.x & 31) == 0 && gsum) atomicAdd((unsigned long long*)p.gain_acc, (unsigned long long)gsum);
}

// Re-queue the neighbours of every node that moved in this batch and now sits
// in a different community from them (local_move.rs:113-118). Runs after the
// commit, so every membership it reads is final.
// A node enters the next sweep's list once: its stamp is raised to `mark` (the
// next sweep's number + 1) and only the lane that raised it appends it.
// Half a warp per node (k-NN rows hold 10-30 entries, so a whole warp per row
// would leave most lanes idle); both halves walk max(their chunk counts) chunks
// so that the ballot and the shuffle see every lane.
__global__ void k_activate(Params p, const uint32_t* __restrict__ list, uint32_t count, uint32_t* stamp,
                           uint32_t mark, uint32_t* next_list, uint32_t* next_count) {
    const unsigned FULL = 0xFFFFFFFFu;
    const unsigned lane = threadIdx.x & 31u, half = lane >> 4, sub = lane & 15u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i0 = warp * 2; i0 < count; i0 += nwarps * 2) {  // warp-uniform
        const uint64_t i = i0 + half;
        uint32_t v = 0, t = 0;
        uint64_t b = 0, e = 0;
        if (i < count) {
            v = list[i];
            if (p.moved[v] == p.cur) {
                t = p.memb[v];
                b = p.ptr[v];
                e = p.ptr[v + 1];
            }
        }
        const uint64_t my_chunks = (e - b + 15) >> 4;
        const uint64_t chunks = max(my_chunks, __shfl_xor_sync(FULL, my_chunks, 16));
        for (uint64_t ch = 0; ch < chunks; ++ch) {
            const uint64_t j = b + ch * 16 + sub;
            uint32_t u = 0;
            bool add = false;
            if (j < e) {
                u = p.nbr[j];
                // a plain read first: a node already queued for the next sweep
                // (the common case once many of its neighbours moved) costs no atomic
                add = u != v && p.memb[u] != t && stamp[u] < mark && atomicMax(stamp + u, mark) < mark;
            }
            const unsigned bal = __ballot_sync(FULL, add);
            if (bal) {
                const int leader = __ffs(bal) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(next_count, (uint32_t)__popc(bal));
                base = __shfl_sync(FULL, base, leader);
                if (add) next_list[base + __popc(bal & ((1u << lane) - 1u))] = u;
            }
        }
    }
}

template <bool MULTI>
__global__ void k_claim(Params p, const uint32_t* __restrict__ list, uint32_t count) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = list[i];
        if (p.epoch[v] != p.cur || cancelled<MULTI>(p, v)) continue;
        atomicMax(p.claim + p.tgt[v], claim_key<MULTI>(p, v));
    }
}

// ------------------------------------------------------------ bucketing
// Degree buckets; the lane-group limits come from the context's tuning
// (lanes8 <= 8 <= ..., each at most its group size). Any routing gives the same
// decisions: every decide kernel scores the same candidates with the same
// arithmetic and tie rule.
struct Route {
    uint32_t g8, g16, g32;
};

__device__ __forceinline__ int bucket_of(uint32_t deg, Route r) {
    return deg <= r.g8 ? 0 : deg <= r.g16 ? 1 : deg <= r.g32 ? 2 : deg <= WARP_DEGREE ? 3 : deg <= HUB_DEGREE ? 4 : 5;
}

// The hash batch of node v in a sweep, or -1 for a node of a frozen instance.
template <bool MULTI>
__device__ __forceinline__ int batch_of(uint64_t seed, uint32_t sweep, uint64_t v, int B, const uint32_t* inst,
                                        const InstCfg* icfg) {
    if (!MULTI) return (int)(hash3(seed, sweep, v) % (uint64_t)B);
    const InstCfg& c = icfg[inst[v]];
    if (c.frozen) return -1;
    return (int)(hash3(c.seed, sweep, v - c.base) % (uint64_t)B);
}

// The nodes of a sweep: alist[0 .. *acount) or, with alist == nullptr, all n.
template <bool MULTI>
__global__ void k_bucket_count(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ alist,
                               const uint32_t* __restrict__ acount, uint64_t n, uint64_t seed, uint32_t sweep, int B,
                               Route route, uint32_t* counts, const uint32_t* inst, const InstCfg* icfg) {
    __shared__ uint32_t sc[64];
    for (int t = threadIdx.x; t < B * NBUCKET; t += blockDim.x) sc[t] = 0;
    __syncthreads();
    const uint64_t m = alist ? *acount : n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t v = alist ? alist[i] : i;
        const int b = batch_of<MULTI>(seed, sweep, v, B, inst, icfg);
        if (b < 0) continue;
        int k = bucket_of((uint32_t)(ptr[v + 1] - ptr[v]), route);
        atomicAdd(&sc[b * NBUCKET + k], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < B * NBUCKET; t += blockDim.x)
        if (sc[t]) atomicAdd(counts + t, sc[t]);
}

// One warp-aggregated atomic per distinct (batch, bucket) per warp.
template <bool MULTI>
__global__ void k_bucket_scatter(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ alist,
                                 const uint32_t* __restrict__ acount, uint64_t n, uint64_t seed, uint32_t sweep,
                                 int B, Route route, uint32_t* cursor, uint32_t* list, uint64_t* lbeg,
                                 uint32_t* ldeg, const uint32_t* inst, const InstCfg* icfg) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t m = alist ? *acount : n;
    for (uint64_t base = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) - lane; base < m; base += stride) {
        const uint64_t i = base + lane;
        const uint64_t v = i < m ? (alist ? alist[i] : i) : 0;
        int slot = -1;
        uint64_t rb = 0;
        uint32_t deg = 0;
        if (i < m) {
            const int b = batch_of<MULTI>(seed, sweep, v, B, inst, icfg);
            if (b >= 0) {
                rb = ptr[v];
                deg = (uint32_t)(ptr[v + 1] - rb);
                int k = bucket_of(deg, route);
                slot = b * NBUCKET + k;
            }
        }
        const unsigned mm = __match_any_sync(0xFFFFFFFFu, slot < 0 ? 1000 + (int)lane : slot);
        const int leader = __ffs(mm) - 1;
        uint32_t pos0 = 0;
        if (slot >= 0 && (int)lane == leader) pos0 = atomicAdd(cursor + slot, (uint32_t)__popc(mm));
        pos0 = __shfl_sync(0xFFFFFFFFu, pos0, leader);
        if (slot >= 0) {
            const uint32_t pos = pos0 + __popc(mm & ((1u << lane) - 1u));
            list[pos] = (uint32_t)v;
            lbeg[pos] = rb;
            ldeg[pos] = deg;
        }
    }
}

// ------------------------------------------------------------ partition state
__global__ void k_init_comm(const uint32_t* __restrict__ memb, uint64_t n, const double* __restrict__ strength,
                            const double* __restrict__ node_w, double inv_scale, double inv_nscale,
                            long long* Kf, long long* Wf, uint32_t* csize) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = memb[v];
        atomicAdd((unsigned long long*)(Kf + c), (unsigned long long)to_fix(strength[v], inv_scale));
        if (Wf) atomicAdd((unsigned long long*)(Wf + c), (unsigned long long)to_fix(node_w[v], inv_nscale));
        atomicAdd(csize + c, 1u);
    }
}

__global__ void k_identity(uint32_t* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

__global__ void k_scatter_coarse(const uint32_t* __restrict__ grp, const uint32_t* __restrict__ memb,
                                 uint64_t n, uint32_t* cmemb) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x)
        cmemb[grp[v]] = memb[v];
}

__global__ void k_gather(const uint32_t* __restrict__ map, uint32_t* x, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        x[i] = map[x[i]];
}

// ------------------------------------------------------------ host side
struct Scales {
    double scale, inv, nscale, ninv;
};

Scales scales_for(const DevGraph& g) {
    Scales s;
    int F;
    if (g.exact_w) F = (g.e0_w == 0x7FFFFFFF) ? 0 : g.e0_w;
    else F = (int)std::ceil(std::log2(std::max(2.0 * g.total_weight, 1e-300))) + 1 - 61;
    int Fn;
    if (g.exact_nw) Fn = (g.e0_nw == 0x7FFFFFFF) ? 0 : g.e0_nw;
    else Fn = (int)std::ceil(std::log2(std::max(g.total_node_weight, 1e-300))) + 1 - 61;
    s.scale = std::ldexp(1.0, F);
    s.inv = std::ldexp(1.0, -F);
    s.nscale = std::ldexp(1.0, Fn);
    s.ninv = std::ldexp(1.0, -Fn);
    return s;
}

struct Workspace {
    DBuf<uint32_t> tgt, hint, from, epoch, list, moved;
    DBuf<uint64_t> lbeg;  // row start of each list entry (written by the bucket scatter)
    DBuf<uint32_t> ldeg;  // degree of each list entry
    DBuf<long long> dgain;
    DBuf<uint32_t> alist, nlist;    // this sweep's active nodes, the next sweep's
    DBuf<uint32_t> acount, ncount;  // their counts (device)
    DBuf<uint32_t> stamp;           // per node: 1 + the last sweep it was queued for
    DBuf<uint32_t> counts;
    DBuf<uint32_t> cursor;  // scatter cursors of the (batch, bucket) lists
    DBuf<unsigned long long> counters;
    DBuf<long long> gain_acc;
    DBuf<uint32_t> gkeys;
    DBuf<long long> gvals;
    uint64_t gcap = 0;
    int nblk_large = 0;
    uint64_t cap = 0;  // nodes the per-node arrays hold (the largest level seen)
};

// Phase times of a run: events recorded around each phase on the context's
// stream, read after the run's last synchronisation, so timing adds none.
class PhaseClock {
   public:
    explicit PhaseClock(Ctx& c) : c_(c) {}
    PhaseClock(const PhaseClock&) = delete;
    PhaseClock& operator=(const PhaseClock&) = delete;
    ~PhaseClock() {
        for (Span& s : spans_) {
            cudaEventDestroy(s.a);
            cudaEventDestroy(s.b);
        }
    }
    size_t start() {
        Span s{};
        SC_CUDA(cudaEventCreate(&s.a));
        if (cudaEventCreate(&s.b) != cudaSuccess) {
            cudaEventDestroy(s.a);
            SC_CUDA(cudaErrorMemoryAllocation);
        }
        spans_.push_back(s);
        SC_CUDA(cudaEventRecord(s.a, c_.stream));
        return spans_.size() - 1;
    }
    // the span's time is added to *into when collect() runs
    void stop(size_t i, double* into) {
        SC_CUDA(cudaEventRecord(spans_[i].b, c_.stream));
        spans_[i].into = into;
    }
    // waits for every stopped span and adds its time to its target
    void collect() {
        for (Span& s : spans_) {
            if (!s.into) continue;
            SC_CUDA(cudaEventSynchronize(s.b));
            float ms = 0.0f;
            SC_CUDA(cudaEventElapsedTime(&ms, s.a, s.b));
            *s.into += ms;
            s.into = nullptr;
        }
    }

   private:
    struct Span {
        cudaEvent_t a, b;
        double* into;
    };
    Ctx& c_;
    std::vector<Span> spans_;
};

// One workspace serves every level of a run: the per-node arrays are sized by
// the first (largest) level and only their prefix is used below it, which
// spares each level some twenty allocations (the bulk of a small level's host
// time). The hub scratch grows when a level needs more.
void prepare_workspace(Ctx& c, Workspace& ws, const DevGraph& g) {
    const uint64_t n = g.n;
    if (ws.cap < n || ws.cap == 0) {
        const uint64_t m = std::max<uint64_t>(n, 1);
        ws.tgt.alloc(c, m);
        ws.hint.alloc(c, m);
        ws.from.alloc(c, m);
        ws.epoch.alloc(c, m);
        ws.moved.alloc(c, m);
        ws.list.alloc(c, m);
        ws.lbeg.alloc(c, m);
        ws.ldeg.alloc(c, m);
        ws.dgain.alloc(c, m);
        ws.alist.alloc(c, m);
        ws.nlist.alloc(c, m);
        ws.acount.alloc(c, 1);
        ws.ncount.alloc(c, 1);
        ws.stamp.alloc(c, m);
        ws.counts.alloc(c, 64);
        ws.cursor.alloc(c, 64);
        ws.counters.alloc(c, 4);
        ws.gain_acc.alloc(c, 1);
        ws.cap = m;
    }
    zero(c, ws.epoch.get(), n);
    zero(c, ws.moved.get(), n);
    zero(c, ws.hint.get(), n);
    // global hash / candidate scratch, one slice per block, for the hubs only
    ws.nblk_large = 0;
    ws.gcap = 0;
    if (g.n_hubs) {
        uint64_t cap = 64;
        while (cap < 2ull * g.max_degree) cap <<= 1;
        int nblk = (int)std::min<uint64_t>((uint64_t)c.sm_count * 2, g.n_hubs);
        const uint64_t budget = 1ull << 31;  // bytes of hub scratch at most
        while (nblk > 1 && (uint64_t)nblk * cap * 12 > budget) nblk >>= 1;
        ws.nblk_large = nblk;
        ws.gcap = cap;
        if (ws.gkeys.n < (uint64_t)nblk * cap) {
            ws.gkeys.alloc(c, (uint64_t)nblk * cap);
            ws.gvals.alloc(c, (uint64_t)nblk * cap);
        }
    }
}

template <bool REFINE, bool MULTI>
void launch_decide(Ctx& c, Params& p, Workspace& ws, int k, uint32_t off, uint32_t cnt,
                   cudaStream_t st = nullptr) {
    if (!cnt) return;
    if (!st) st = c.stream;
    const uint32_t* list = ws.list.get() + off;
    const uint64_t* lbeg = ws.lbeg.get() + off;
    const uint32_t* ldeg = ws.ldeg.get() + off;
    if (k == 0) {
        unsigned warps = (cnt + 3) / 4;
        k_decide_small<8, REFINE, MULTI><<<grid_for((uint64_t)warps * 32, TB, 148u * 64u), TB, 0, st>>>(p, list, lbeg, ldeg, cnt);
    } else if (k == 1) {
        unsigned warps = (cnt + 1) / 2;
        k_decide_small<16, REFINE, MULTI><<<grid_for((uint64_t)warps * 32, TB, 148u * 64u), TB, 0, st>>>(p, list, lbeg, ldeg, cnt);
    } else if (k == 2) {
        k_decide_small<32, REFINE, MULTI><<<grid_for((uint64_t)cnt * 32, TB, 148u * 64u), TB, 0, st>>>(p, list, lbeg, ldeg, cnt);
    } else if (k == 3) {
        const uint64_t warps = cnt;
        k_decide_warp<REFINE, MULTI><<<grid_for(warps * 32, 32 * WARPS_PER_BLOCK, 148u * 64u), 32 * WARPS_PER_BLOCK, 0,
                                st>>>(p, list, lbeg, ldeg, cnt);
    } else if (k == 4) {
        size_t sm = HCAP_SMEM * (sizeof(long long) + sizeof(uint32_t));
        unsigned grid = std::min<unsigned>(cnt, (unsigned)c.sm_count * 4);
        k_decide_block<REFINE, false, MULTI><<<grid, TB, sm, st>>>(p, list, lbeg, ldeg, cnt, nullptr, nullptr, 0);
    } else {
        if (ws.nblk_large < 1 || ws.gcap == 0) fail(SC_E_INTERNAL, "hub scratch missing");
        unsigned grid = std::min<unsigned>(cnt, (unsigned)ws.nblk_large);
        k_decide_block<REFINE, true, MULTI><<<grid, TB, 0, st>>>(p, list, lbeg, ldeg, cnt, ws.gkeys.get(),
                                                               ws.gvals.get(), ws.gcap);
    }
    SC_LAUNCH_CHECK();
    c.launches++;
}

// The decide launches of batch b (list slices offs[b*NBUCKET + k] ..). A small
// batch sends its nodes of degree <= WARP_DEGREE (buckets 0-3, contiguous in
// the list) to the warp-per-node kernel in one launch: it computes the same
// decision for them as the lane-group kernels (fixed-point sums are exact in
// any order, ties go to the lower id), and the launches saved are the cost
// that dominates a batch of a few thousand nodes.
Route route_of(const Ctx& c) { return Route{c.tuning.lanes8_max_degree, c.tuning.lanes16_max_degree,
                                             c.tuning.lanes32_max_degree}; }

template <bool REFINE, bool MULTI>
void launch_batch_decide(Ctx& c, Params& p, Workspace& ws, const uint32_t* offs, int b) {
    const uint32_t* o = offs + b * NBUCKET;
    if (o[4] - o[0] <= c.tuning.small_batch) {
        launch_decide<REFINE, MULTI>(c, p, ws, 3, o[0], o[4] - o[0]);
        for (int k = 4; k < NBUCKET; ++k) launch_decide<REFINE, MULTI>(c, p, ws, k, o[k], o[k + 1] - o[k]);
        return;
    }
    // Buckets of one batch read the same snapshot and write disjoint nodes: the
    // non-empty ones run concurrently on the context's side streams (fork and
    // join by events), so one kernel's ramp and last partial wave overlap another.
    int nonempty = 0;
    for (int k = 0; k < NBUCKET; ++k) nonempty += o[k + 1] > o[k];
    if (nonempty < 2 || !c.side[0]) {
        for (int k = 0; k < NBUCKET; ++k) launch_decide<REFINE, MULTI>(c, p, ws, k, o[k], o[k + 1] - o[k]);
        return;
    }
    SC_CUDA(cudaEventRecord(c.ev_fork, c.stream));
    int used = 0;
    bool first = true;
    for (int k = 0; k < NBUCKET; ++k) {
        if (o[k + 1] == o[k]) continue;
        if (first) {  // the first non-empty bucket runs on the main stream
            launch_decide<REFINE, MULTI>(c, p, ws, k, o[k], o[k + 1] - o[k]);
            first = false;
            continue;
        }
        cudaStream_t st = c.side[used % SIDE_STREAMS];
        if (used < SIDE_STREAMS) SC_CUDA(cudaStreamWaitEvent(st, c.ev_fork, 0));
        launch_decide<REFINE, MULTI>(c, p, ws, k, o[k], o[k + 1] - o[k], st);
        ++used;
    }
    for (int t = 0; t < used && t < SIDE_STREAMS; ++t) {
        SC_CUDA(cudaEventRecord(c.ev_join[t], c.side[t]));
        SC_CUDA(cudaStreamWaitEvent(c.stream, c.ev_join[t], 0));
    }
}

struct MoveResult {
    double improvement = 0.0;
    uint64_t sweeps = 0, moves = 0;
    double alg_bytes = 0.0;
};

// Parallel local moving over communities `memb` (ids < S0), extra ids
// [S0, S0+n) are the fresh empty communities.
// A level of a batched run: each node's instance, the instances' settings on
// the device (InstCfg, one per instance) and their gain accumulators.
struct MultiLevel {
    const uint32_t* inst = nullptr;
    const InstCfg* icfg = nullptr;
    long long* gain_inst = nullptr;
};

template <bool REFINE>
void batch_decide(Ctx& c, Params& p, Workspace& ws, const uint32_t* offs, int b) {
    if (p.inst) launch_batch_decide<REFINE, true>(c, p, ws, offs, b);
    else launch_batch_decide<REFINE, false>(c, p, ws, offs, b);
}

void launch_bucket_count(Ctx& c, const Params& p, const DevGraph& g, const uint32_t* alist, const uint32_t* acount,
                         uint64_t seed, uint32_t sweep, int B, uint32_t* counts) {
    const uint64_t n = g.n;
    if (p.inst)
        k_bucket_count<true><<<grid_for(n, TB), TB, 0, c.stream>>>(g.ptr, alist, acount, n, seed, sweep, B,
                                                                   route_of(c), counts, p.inst, p.icfg);
    else
        k_bucket_count<false><<<grid_for(n, TB), TB, 0, c.stream>>>(g.ptr, alist, acount, n, seed, sweep, B,
                                                                    route_of(c), counts, nullptr, nullptr);
    SC_LAUNCH_CHECK();
    c.launches++;
}

void launch_bucket_scatter(Ctx& c, const Params& p, const DevGraph& g, const uint32_t* alist,
                           const uint32_t* acount, uint64_t work, uint64_t seed, uint32_t sweep, int B,
                           Workspace& ws) {
    const uint64_t n = g.n;
    if (p.inst)
        k_bucket_scatter<true><<<grid_for(work, TB), TB, 0, c.stream>>>(g.ptr, alist, acount, n, seed, sweep, B,
                                                                        route_of(c), ws.cursor.get(), ws.list.get(),
                                                                        ws.lbeg.get(), ws.ldeg.get(), p.inst, p.icfg);
    else
        k_bucket_scatter<false><<<grid_for(work, TB), TB, 0, c.stream>>>(g.ptr, alist, acount, n, seed, sweep, B,
                                                                         route_of(c), ws.cursor.get(), ws.list.get(),
                                                                         ws.lbeg.get(), ws.ldeg.get(), nullptr, nullptr);
    SC_LAUNCH_CHECK();
    c.launches++;
}

template <bool REFINE>
void launch_claim_apply(Ctx& c, Params& p, const uint32_t* list, uint32_t cnt, bool claim_only) {
    const unsigned grid = grid_for(cnt, TB);
    if (claim_only) {
        if (p.inst) k_claim<true><<<grid, TB, 0, c.stream>>>(p, list, cnt);
        else k_claim<false><<<grid, TB, 0, c.stream>>>(p, list, cnt);
    } else {
        if (p.inst) k_apply<REFINE, true><<<grid, TB, 0, c.stream>>>(p, list, cnt);
        else k_apply<REFINE, false><<<grid, TB, 0, c.stream>>>(p, list, cnt);
    }
    SC_LAUNCH_CHECK();
    c.launches++;
}

MoveResult local_move(Ctx& c, const DevGraph& g, Workspace& ws, uint32_t* memb, uint64_t S0,
                      const sc_leiden_config& cfg, uint64_t seed, const Scales& sc, double gamma,
                      const MultiLevel* ml = nullptr) {
    MoveResult r;
    const uint64_t n = g.n;
    if (n == 0) return r;
    const uint64_t S = S0 + n;
    const bool need_nc = cfg.objective == SC_OBJECTIVE_CPM || cfg.has_max_community_weight;
    DBuf<long long> Kf(c, S), Wf(c, need_nc ? S : 0);  // Wf only where CPM or the cap reads it
    DBuf<uint32_t> csize(c, S);
    DBuf<unsigned long long> claim(c, cfg.has_max_community_weight ? S : 0);
    zero(c, claim.get(), claim.n);
    zero(c, Kf.get(), S);
    zero(c, Wf.get(), Wf.n);
    zero(c, csize.get(), S);
    k_init_comm<<<grid_for(n, TB), TB, 0, c.stream>>>(memb, n, g.strength, g.node_w, sc.inv, sc.ninv,
                                                      Kf.get(), Wf.get(), csize.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    Params p{};
    p.ptr = g.ptr;
    p.nbr = g.nbr;
    p.w = g.w;
    p.strength = g.strength;
    p.node_w = g.node_w;
    p.self_loop = g.self_loop;
    p.memb = memb;
    p.Kf = Kf.get();
    p.Wf = Wf.get();
    p.csize = csize.get();
    p.constraint = nullptr;
    p.tgt = ws.tgt.get();
    p.hint = ws.hint.get();
    p.from = ws.from.get();
    p.dgain = ws.dgain.get();
    p.epoch = ws.epoch.get();
    p.S0 = S0;
    p.objective = cfg.objective;
    p.gamma = gamma;
    p.four_m = 4.0 * g.total_weight;
    p.thr = 1e-12 * std::max(std::fabs(g.total_weight), 1.0);  // local_move.rs:26-28
    p.scale = sc.scale;
    p.inv_scale = sc.inv;
    p.nscale = sc.nscale;
    p.inv_nscale = sc.ninv;
    p.has_limit = cfg.has_max_community_weight;
    p.limit = cfg.max_community_weight;
    p.need_nc = cfg.objective == SC_OBJECTIVE_CPM || cfg.has_max_community_weight;
    p.theta = 0.0;
    p.seed = seed;
    p.status = c.d_status;
    p.counters = ws.counters.get();
    p.gain_acc = ws.gain_acc.get();
    p.claim = claim.get();
    p.moved = ws.moved.get();
    if (ml) {
        p.inst = ml->inst;
        p.icfg = ml->icfg;
        p.gain_inst = ml->gain_inst;
    }
    zero(c, ws.counters.get(), 4);
    zero(c, ws.gain_acc.get(), 1);
    zero(c, ws.epoch.get(), n);
    zero(c, ws.moved.get(), n);
    zero(c, ws.stamp.get(), n);
    bool all_active = true;  // sweep 0 visits every node
    const int B = LM_BATCHES;
    uint32_t epoch = 0;
    uint64_t moves_before = 0;
    const uint64_t budget = n * 100;  // MAX_MOVES_PER_NODE, local_move.rs:32
    static const int trace = std::getenv("SC_TRACE") ? std::atoi(std::getenv("SC_TRACE")) : 0;
    unsigned long long last_ctr[4] = {0, 0, 0, 0};
    long long last_gacc = 0;
    bool read_fresh = false;  // last_ctr / last_gacc hold the counters' current values
    for (uint32_t sweep = 0; sweep < (uint32_t)MAX_SWEEPS; ++sweep) {
        zero(c, ws.counts.get(), B * NBUCKET);
        zero(c, ws.ncount.get(), 1);
        const uint32_t* alist = all_active ? nullptr : ws.alist.get();
        launch_bucket_count(c, p, g, alist, ws.acount.get(), seed, sweep, B, ws.counts.get());
        uint32_t counts[64];
        unsigned long long ctr[4];
        {
            Mailbox mb(c);
            const uint32_t* hc = mb.get(ws.counts.get(), B * NBUCKET);
            const unsigned long long* hk = mb.get(ws.counters.get(), 4);
            const long long* hg = mb.get(ws.gain_acc.get(), 1);
            mb.wait();
            std::memcpy(counts, hc, sizeof(uint32_t) * B * NBUCKET);
            std::memcpy(ctr, hk, sizeof ctr);
            std::memcpy(last_ctr, hk, sizeof ctr);
            last_gacc = *hg;
            read_fresh = true;  // nothing that changes the counters runs before the next launch below
        }
        uint32_t offs[65];
        offs[0] = 0;
        for (int t = 0; t < B * NBUCKET; ++t) offs[t + 1] = offs[t] + counts[t];
        if (trace >= 2 && sweep > 0)
            std::fprintf(stderr, "[sc]   sweep %u moves=%llu next_active=%u\n", sweep - 1,
                         (unsigned long long)(ctr[0] - moves_before), offs[B * NBUCKET]);
        if (sweep > 0 && ctr[0] == moves_before) break;  // last sweep moved nothing
        if (ctr[0] >= budget) break;
        moves_before = ctr[0];
        if (offs[B * NBUCKET] == 0) break;
        read_fresh = false;
        h2d(c, ws.cursor.get(), offs, B * NBUCKET);
        launch_bucket_scatter(c, p, g, alist, ws.acount.get(), all_active ? n : offs[B * NBUCKET], seed, sweep, B,
                              ws);
        // A batch's re-queue reads memberships and writes only the next sweep's
        // list, so with an auxiliary stream it runs while the next batch decides;
        // it must end before the next batch commits (which changes memberships).
        // (a sweep of a few thousand nodes gains nothing from the overlap and
        // would pay three extra stream operations per batch)
        const bool overlap = c.aux != nullptr && offs[B * NBUCKET] > c.tuning.small_batch;
        bool act_pending = false;
        for (int b = 0; b < B; ++b) {
            ++epoch;
            p.cur = epoch;
            p.seed = seed;
            uint32_t lo = offs[b * NBUCKET], hi = offs[(b + 1) * NBUCKET];
            if (lo == hi) continue;
            batch_decide<false>(c, p, ws, offs, b);
            if (p.has_limit) launch_claim_apply<false>(c, p, ws.list.get() + lo, hi - lo, true);
            if (act_pending) {
                SC_CUDA(cudaStreamWaitEvent(c.stream, c.ev_aux_done, 0));
                act_pending = false;
            }
            launch_claim_apply<false>(c, p, ws.list.get() + lo, hi - lo, false);
            cudaStream_t as = c.stream;
            if (overlap) {
                SC_CUDA(cudaEventRecord(c.ev_aux_start, c.stream));
                SC_CUDA(cudaStreamWaitEvent(c.aux, c.ev_aux_start, 0));
                as = c.aux;
            }
            k_activate<<<grid_for((uint64_t)(hi - lo) * 16, TB, 148u * 64u), TB, 0, as>>>(
                p, ws.list.get() + lo, hi - lo, ws.stamp.get(), sweep + 2, ws.nlist.get(), ws.ncount.get());
            if (overlap) {
                SC_CUDA(cudaEventRecord(c.ev_aux_done, c.aux));
                act_pending = true;
            }
            SC_LAUNCH_CHECK();
            c.launches++;
        }
        if (act_pending) SC_CUDA(cudaStreamWaitEvent(c.stream, c.ev_aux_done, 0));
        std::swap(ws.alist, ws.nlist);
        std::swap(ws.acount, ws.ncount);
        all_active = false;
        r.sweeps++;
    }
    if (!read_fresh) {  // the sweep limit ended the loop after launching a sweep
        Mailbox mb(c);
        const unsigned long long* hk = mb.get(ws.counters.get(), 4);
        const long long* hg = mb.get(ws.gain_acc.get(), 1);
        mb.wait();
        std::memcpy(last_ctr, hk, sizeof last_ctr);
        last_gacc = *hg;
    }
    const unsigned long long* ctr = last_ctr;
    const long long gacc = last_gacc;
    r.moves = ctr[0];
    r.improvement = (double)gacc * sc.scale;
    // algorithmic bytes: 16 per node visit + 12 per scanned entry + 8 per candidate
    r.alg_bytes = 16.0 * (double)ctr[3] + 12.0 * (double)ctr[1] + 8.0 * (double)ctr[2];
    return r;
}

// refine (refine.rs:29-103): refined ids < n; constraint = working membership.
// Adds a refinement's node, entry and candidate counters to the run's totals.
__global__ void k_add_refine_counters(const unsigned long long* __restrict__ ctr, unsigned long long* run) {
    if (threadIdx.x == 0) {
        run[0] += ctr[3];
        run[1] += ctr[1];
        run[2] += ctr[2];
    }
}

// Algorithmic bytes of the refinements of a run, from the counters summed on the device.
double refine_alg_bytes(const unsigned long long* run) {
    return 16.0 * (double)run[0] + 16.0 * (double)run[1] + 8.0 * (double)run[2];
}

void refine(Ctx& c, const DevGraph& g, Workspace& ws, const uint32_t* constraint, uint32_t* refined,
            const sc_leiden_config& cfg, uint64_t seed, const Scales& sc, double gamma,
            const MultiLevel* ml = nullptr) {
    const uint64_t n = g.n;
    if (n == 0) return;
    const bool need_nc = cfg.objective == SC_OBJECTIVE_CPM || cfg.has_max_community_weight;
    DBuf<long long> Kf(c, n), Wf(c, need_nc ? n : 0);  // Wf only where CPM or the cap reads it
    DBuf<uint32_t> csize(c, n);
    DBuf<unsigned long long> claim(c, cfg.has_max_community_weight ? n : 0);
    zero(c, claim.get(), claim.n);
    zero(c, Kf.get(), n);
    zero(c, Wf.get(), Wf.n);
    zero(c, csize.get(), n);
    k_identity<<<grid_for(n, TB), TB, 0, c.stream>>>(refined, n);
    k_init_comm<<<grid_for(n, TB), TB, 0, c.stream>>>(refined, n, g.strength, g.node_w, sc.inv, sc.ninv,
                                                      Kf.get(), Wf.get(), csize.get());
    SC_LAUNCH_CHECK();
    c.launches += 2;
    Params p{};
    p.ptr = g.ptr;
    p.nbr = g.nbr;
    p.w = g.w;
    p.strength = g.strength;
    p.node_w = g.node_w;
    p.self_loop = g.self_loop;
    p.memb = refined;
    p.Kf = Kf.get();
    p.Wf = Wf.get();
    p.csize = csize.get();
    p.constraint = constraint;
    p.tgt = ws.tgt.get();
    p.hint = ws.hint.get();
    p.from = ws.from.get();
    p.dgain = ws.dgain.get();
    p.epoch = ws.epoch.get();
    p.S0 = n;
    p.objective = cfg.objective;
    p.gamma = gamma;
    p.four_m = 4.0 * g.total_weight;
    p.thr = 0.0;
    p.scale = sc.scale;
    p.inv_scale = sc.inv;
    p.nscale = sc.nscale;
    p.inv_nscale = sc.ninv;
    p.has_limit = cfg.has_max_community_weight;
    p.limit = cfg.max_community_weight;
    p.need_nc = cfg.objective == SC_OBJECTIVE_CPM || cfg.has_max_community_weight;
    double mean_edge = g.edge_count > 0 ? g.total_weight / (double)g.edge_count : 1.0;
    p.theta = cfg.refine_randomness * mean_edge;  // refine.rs:44-50
    p.seed = seed;
    p.status = c.d_status;
    p.counters = ws.counters.get();
    p.gain_acc = ws.gain_acc.get();
    p.claim = claim.get();
    p.moved = ws.moved.get();
    if (ml) {
        p.inst = ml->inst;
        p.icfg = ml->icfg;
        p.gain_inst = ml->gain_inst;
    }
    zero(c, ws.counters.get(), 4);
    zero(c, ws.epoch.get(), n);
    const int B = RF_BATCHES;
    zero(c, ws.counts.get(), B * NBUCKET);
    launch_bucket_count(c, p, g, nullptr, nullptr, seed, 0xFFFFFFFFu, B, ws.counts.get());
    uint32_t counts[64];
    {
        Mailbox mb(c);
        const uint32_t* hc = mb.get(ws.counts.get(), B * NBUCKET);
        mb.wait();
        std::memcpy(counts, hc, sizeof(uint32_t) * B * NBUCKET);
    }
    uint32_t offs[65];
    offs[0] = 0;
    for (int t = 0; t < B * NBUCKET; ++t) offs[t + 1] = offs[t] + counts[t];
    h2d(c, ws.cursor.get(), offs, B * NBUCKET);
    launch_bucket_scatter(c, p, g, nullptr, nullptr, n, seed, 0xFFFFFFFFu, B, ws);
    for (int b = 0; b < B; ++b) {
        p.cur = (uint32_t)(b + 1);
        uint32_t lo = offs[b * NBUCKET], hi = offs[(b + 1) * NBUCKET];
        if (lo == hi) continue;
        batch_decide<true>(c, p, ws, offs, b);
        if (p.has_limit) launch_claim_apply<true>(c, p, ws.list.get() + lo, hi - lo, true);
        launch_claim_apply<true>(c, p, ws.list.get() + lo, hi - lo, false);
    }
    // counters go to the run's totals on the device (read once, at the end of the run)
    k_add_refine_counters<<<1, 32, 0, c.stream>>>(ws.counters.get(), c.d_refine_ctr);
    SC_LAUNCH_CHECK();
    c.launches++;
}

struct PassOut {
    DBuf<uint32_t> labels;  // compact, n
    uint64_t n_clusters = 0;
    double improvement = 0.0;
};

// run_once (mod.rs:214-289) from compact initial ids `init` (< C0).
void run_pass(Ctx& c, const DevGraph& g0, const uint32_t* init, uint64_t C0, const sc_leiden_config& cfg,
              uint64_t pass_seed, PassOut& out, sc_run_stats& st, PhaseClock& clock, Workspace& ws) {
    const uint64_t n0 = g0.n;
    const double gamma = cfg.resolution;
    std::unique_ptr<DevGraph> owned;
    const DevGraph* gl = &g0;
    DBuf<uint32_t> memb(c, n0), node_at(c, n0);
    d2d(c, memb.get(), init, n0);
    k_identity<<<grid_for(n0, TB), TB, 0, c.stream>>>(node_at.get(), n0);
    c.launches++;
    uint64_t C = C0;
    double improvement = 0.0;
    static const bool trace = std::getenv("SC_TRACE") != nullptr;
    for (uint64_t level = 0; level < cfg.max_levels; ++level) {
        const uint64_t nl = gl->n, level_E = gl->E;
        const sc_run_stats before = st;
        const uint64_t lvl_seed = hash3(pass_seed, level, 0x1eafull);
        Scales sc = scales_for(*gl);
        prepare_workspace(c, ws, *gl);
        // ids of memb are < C; fresh ids live in [C, C + nl)
        {
            const size_t t = clock.start();
            MoveResult mr = local_move(c, *gl, ws, memb.get(), C, cfg, lvl_seed, sc, gamma);
            clock.stop(t, &st.ms_local_move);
            improvement += mr.improvement;
            st.local_move_sweeps += mr.sweeps;
            st.moves += mr.moves;
            st.alg_bytes_local_move += mr.alg_bytes;
        }
        DBuf<uint32_t> collapse(c, nl);
        uint64_t id_space;
        if (cfg.refine) {
            const size_t t = clock.start();
            refine(c, *gl, ws, memb.get(), collapse.get(), cfg, hash3(lvl_seed, 0x7e71eull, 1), sc, gamma);
            clock.stop(t, &st.ms_refine);
            id_space = nl;
        } else {
            d2d(c, collapse.get(), memb.get(), nl);
            id_space = C + nl;
        }
        const size_t t_agg = clock.start();
        DBuf<uint32_t> grp(c, nl);
        uint32_t G = renumber_ids(c, collapse.get(), nl, id_space, grp.get());
        st.levels++;
        auto trace_level = [&](uint64_t ng) {
            if (!trace) return;
            clock.collect();
            std::fprintf(stderr,
                         "[sc] level %llu n=%llu E=%llu exact=%d/%d groups=%llu sweeps=%llu moves=%llu "
                         "lm=%.3fms ref=%.3fms agg=%.3fms\n",
                         (unsigned long long)level, (unsigned long long)nl, (unsigned long long)level_E,
                         (int)gl->exact_w, (int)gl->exact_nw,
                         (unsigned long long)ng,
                         (unsigned long long)(st.local_move_sweeps - before.local_move_sweeps),
                         (unsigned long long)(st.moves - before.moves), st.ms_local_move - before.ms_local_move,
                         st.ms_refine - before.ms_refine, st.ms_aggregate - before.ms_aggregate);
        };
        if (G >= nl) {
            clock.stop(t_agg, &st.ms_aggregate);
            trace_level(G);
            break;
        }
        std::unique_ptr<DevGraph> coarse(graph_aggregate(c, *gl, grp.get(), G));
        coarse->stream = c.stream;
        st.alg_bytes_aggregate += 12.0 * (double)gl->E + 12.0 * (double)nl + 8.0 * (double)coarse->E +
                                  24.0 * (double)coarse->n;
        // coarse membership from the working partition (mod.rs:269-272), compacted
        DBuf<uint32_t> cm(c, G), cm2(c, G);
        k_scatter_coarse<<<grid_for(nl, TB), TB, 0, c.stream>>>(grp.get(), memb.get(), nl, cm.get());
        k_gather<<<grid_for(n0, TB), TB, 0, c.stream>>>(grp.get(), node_at.get(), n0);
        SC_LAUNCH_CHECK();
        c.launches += 2;
        C = renumber_ids(c, cm.get(), G, C + nl, cm2.get());
        memb = std::move(cm2);
        owned = std::move(coarse);
        gl = owned.get();
        clock.stop(t_agg, &st.ms_aggregate);
        trace_level(G);
    }
    // final ascending renumber (mod.rs:282-286)
    const uint64_t nl = gl->n;
    DBuf<uint32_t> fin(c, nl);
    uint32_t K = renumber_ids(c, memb.get(), nl, C + nl, fin.get());
    out.labels.alloc(c, n0);
    d2d(c, out.labels.get(), node_at.get(), n0);
    k_gather<<<grid_for(n0, TB), TB, 0, c.stream>>>(fin.get(), out.labels.get(), n0);
    SC_LAUNCH_CHECK();
    c.launches++;
    out.n_clusters = K;
    out.improvement = improvement;
}

// ------------------------------------------------------------ batched runs over a disjoint union
// Many leiden() runs at once: the instances' graphs form one disjoint union
// (instance I's nodes are [bounds[I], bounds[I+1]) at every level) and every
// kernel launch covers the nodes of all instances. Each node reads its
// instance's settings (InstCfg) and hashes instance-local ids, community ids
// keep their order inside an instance, and an instance freezes exactly where
// its own run would stop (its graph stopped shrinking, max_levels, or its
// passes are done), so every instance takes the decisions of its own run.

__global__ void k_inst_of_nodes(const uint64_t* __restrict__ bounds, uint32_t* inst) {
    const uint32_t I = blockIdx.y;
    const uint64_t b = bounds[I], e = bounds[I + 1];
    for (uint64_t v = b + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < e; v += (uint64_t)gridDim.x * blockDim.x)
        inst[v] = I;
}

// Per instance (one block each): 2m = the Σ of its nodes' strengths (one warp;
// any order inside the exact regime, the node order outside it) and its
// edge_count, the entries with row <= neighbour.
__global__ void k_inst_stats(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                             const uint32_t* __restrict__ erow, const double* __restrict__ strength,
                             const uint64_t* __restrict__ bounds, int exact, double* two_m,
                             unsigned long long* ecount) {
    __shared__ unsigned long long s_cnt;
    const uint32_t I = blockIdx.x;
    const uint64_t b = bounds[I], e = bounds[I + 1];
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    if (threadIdx.x < 32) {
        const double t = warp_fold(b, e, 0.0, exact != 0, [&](uint64_t v) { return strength[v]; });
        if (threadIdx.x == 0) two_m[I] = t;
    }
    unsigned long long cnt = 0;
    const uint64_t eb = ptr[b], ee = ptr[e];
    for (uint64_t j = eb + threadIdx.x; j < ee; j += blockDim.x) cnt += nbr[j] >= erow[j];
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_cnt, cnt);
    __syncthreads();
    if (threadIdx.x == 0) ecount[I] = s_cnt;
}

__global__ void k_mark_ids(const uint32_t* __restrict__ ids, uint64_t n, uint32_t* used) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        used[ids[i]] = 1;
}

__global__ void k_rank_ids(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ rank, uint64_t n,
                           uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = rank[ids[i]];
}

__global__ void k_gather_at(const uint32_t* __restrict__ rank, const uint64_t* __restrict__ at, uint32_t count,
                            uint32_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= count; i += gridDim.x * blockDim.x) out[i] = rank[at[i]];
}

__global__ void k_inst_keys(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ inst, uint64_t n,
                            uint64_t* keys, uint32_t* idx) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        keys[i] = ((uint64_t)inst[i] << 32) | ids[i];
        idx[i] = (uint32_t)i;
    }
}

__global__ void k_key_heads(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* head, uint32_t* per_inst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t h = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
        head[i] = h;
        if (h) atomicAdd(per_inst + (uint32_t)(keys[i] >> 32), 1u);
    }
}

__global__ void k_scatter_key_rank(const uint32_t* __restrict__ order, const uint32_t* __restrict__ incl, uint64_t n,
                                   uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[order[i]] = incl[i] - 1;
}

__global__ void k_scatter_inst(const uint32_t* __restrict__ grp, const uint32_t* __restrict__ inst, uint64_t n,
                               uint32_t* inst_c) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        inst_c[grp[v]] = inst[v];
}

__global__ void k_sub_base(uint32_t* x, const uint32_t* __restrict__ inst, const uint32_t* __restrict__ base,
                           uint64_t n) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        x[v] -= base[inst[v]];
}

// Ascending ranks of ids in [0, id_space) whose instance ranges are disjoint
// and ordered (instance I's ids inside [bounds[I], bounds[I+1])): the ranks
// keep each instance contiguous; counts[I] = its distinct ids.
void renumber_ranged(Ctx& c, const uint32_t* ids, uint64_t n, uint64_t id_space, const uint64_t* d_bounds,
                     uint32_t count, uint32_t* out, std::vector<uint32_t>& counts) {
    DBuf<uint32_t> used(c, id_space + 1), rank(c, id_space + 1), at(c, count + 1);
    zero(c, used.get(), id_space + 1);
    k_mark_ids<<<grid_for(n, TB), TB, 0, c.stream>>>(ids, n, used.get());
    exclusive_sum(c, used.get(), rank.get(), id_space + 1);
    k_rank_ids<<<grid_for(n, TB), TB, 0, c.stream>>>(ids, rank.get(), n, out);
    k_gather_at<<<grid_for(count + 1, TB), TB, 0, c.stream>>>(rank.get(), d_bounds, count, at.get());
    SC_LAUNCH_CHECK();
    c.launches += 3;
    std::vector<uint32_t> r(count + 1);
    d2h(c, r.data(), at.get(), count + 1);
    sync(c);
    counts.resize(count);
    for (uint32_t i = 0; i < count; ++i) counts[i] = r[i + 1] - r[i];
}

// Ascending ranks of (instance, id): each instance's ids keep their order and
// take a contiguous range of ranks; counts[I] = instance I's distinct ids.
void renumber_by_instance(Ctx& c, const uint32_t* ids, const uint32_t* inst, uint64_t n, uint32_t count,
                          uint32_t* out, std::vector<uint32_t>& counts) {
    counts.assign(count, 0);
    if (n == 0) return;
    DBuf<uint64_t> keys(c, n), keys_s(c, n);
    DBuf<uint32_t> idx(c, n), order(c, n), head(c, n), incl(c, n), per(c, count);
    zero(c, per.get(), count);
    k_inst_keys<<<grid_for(n, TB), TB, 0, c.stream>>>(ids, inst, n, keys.get(), idx.get());
    SC_LAUNCH_CHECK();
    sort_pairs(c, keys.get(), keys_s.get(), idx.get(), order.get(), n, 32 + bits_for(count));
    k_key_heads<<<grid_for(n, TB), TB, 0, c.stream>>>(keys_s.get(), n, head.get(), per.get());
    inclusive_sum(c, head.get(), incl.get(), n);
    k_scatter_key_rank<<<grid_for(n, TB), TB, 0, c.stream>>>(order.get(), incl.get(), n, out);
    SC_LAUNCH_CHECK();
    c.launches += 3;
    d2h(c, counts.data(), per.get(), count);
    sync(c);
}

// Per-pass state of a batched run.
struct MultiPass {
    uint32_t count = 0;
    const sc_leiden_config* cfgs = nullptr;
    std::vector<uint64_t> pass_seed;   // per instance
    std::vector<uint8_t> active;       // the instance runs this pass
    std::vector<uint64_t> n0;          // nodes per instance at level 0
    std::vector<double> improvement;   // out: per instance
    std::vector<uint32_t> n_clusters;  // out: per instance
    std::vector<double> total_weight0; // out: per instance, level 0
};

// run_once (mod.rs:214-289) for every active instance of the union g0 at once,
// from the compact union ids `init` (< C0; each instance's ids a contiguous,
// ordered range). Output labels are union ids, instance I's in a contiguous
// range of n_clusters[I] starting after instance I-1's.
void run_pass_multi(Ctx& c, const DevGraph& g0, const uint32_t* init, uint64_t C0, MultiPass& mp, PassOut& out,
                    sc_run_stats& st, PhaseClock& clock, Workspace& ws) {
    const uint32_t K = mp.count;
    const uint64_t n0 = g0.n;
    const sc_leiden_config& base_cfg = mp.cfgs[0];
    std::unique_ptr<DevGraph> owned;
    const DevGraph* gl = &g0;
    DBuf<uint32_t> memb(c, n0), node_at(c, n0), inst(c, n0);
    d2d(c, memb.get(), init, n0);
    k_identity<<<grid_for(n0, TB), TB, 0, c.stream>>>(node_at.get(), n0);
    c.launches++;
    std::vector<uint64_t> nI = mp.n0;
    std::vector<uint64_t> bounds(K + 1, 0);
    auto set_bounds = [&]() {
        bounds[0] = 0;
        for (uint32_t i = 0; i < K; ++i) bounds[i + 1] = bounds[i] + nI[i];
    };
    set_bounds();
    DBuf<uint64_t> d_bounds(c, K + 1);
    h2d(c, d_bounds.get(), bounds.data(), K + 1);
    if (n0) {
        k_inst_of_nodes<<<dim3(grid_for(*std::max_element(nI.begin(), nI.end()), TB, 148u * 4u), K), TB, 0, c.stream>>>(
            d_bounds.get(), inst.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    std::vector<uint8_t> frozen(K);
    for (uint32_t i = 0; i < K; ++i) frozen[i] = mp.active[i] ? 0 : 1;
    mp.improvement.assign(K, 0.0);
    mp.total_weight0.assign(K, 0.0);
    DBuf<InstCfg> icfg_lm(c, K), icfg_rf(c, K);
    DBuf<long long> gain_inst(c, K);
    DBuf<double> d_two_m(c, K);
    DBuf<unsigned long long> d_ecount(c, K);
    std::vector<InstCfg> h_lm(K), h_rf(K);
    std::vector<double> two_m(K);
    std::vector<unsigned long long> ecount(K);
    std::vector<long long> gains(K);
    std::vector<uint32_t> G(K);
    uint64_t C = C0;
    static const bool trace = std::getenv("SC_TRACE") != nullptr;
    for (uint64_t level = 0;; ++level) {
        const sc_run_stats before = st;
        for (uint32_t i = 0; i < K; ++i)
            if (!frozen[i] && level >= mp.cfgs[i].max_levels) frozen[i] = 1;
        if (std::all_of(frozen.begin(), frozen.end(), [](uint8_t f) { return f != 0; })) break;
        const uint64_t nl = gl->n;
        Scales sc = scales_for(*gl);
        prepare_workspace(c, ws, *gl);
        // the instances' level statistics
        k_inst_stats<<<K, TB, 0, c.stream>>>(gl->ptr, gl->nbr, gl->erow, gl->strength, d_bounds.get(),
                                            (int)gl->exact_w, d_two_m.get(), d_ecount.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        d2h(c, two_m.data(), d_two_m.get(), K);
        d2h(c, ecount.data(), d_ecount.get(), K);
        sync(c);
        for (uint32_t i = 0; i < K; ++i) {
            const sc_leiden_config& cf = mp.cfgs[i];
            const double m = 0.5 * two_m[i];
            if (level == 0) mp.total_weight0[i] = m;
            const uint64_t lvl_seed = hash3(mp.pass_seed[i], level, 0x1eafull);
            InstCfg a{};
            a.gamma = cf.resolution;
            a.four_m = 4.0 * m;
            a.thr = 1e-12 * std::max(std::fabs(m), 1.0);  // local_move.rs:26-28
            a.theta = 0.0;
            a.seed = lvl_seed;
            a.base = (uint32_t)bounds[i];
            a.frozen = frozen[i];
            h_lm[i] = a;
            InstCfg r = a;
            r.thr = 0.0;
            r.theta = cf.refine_randomness * (ecount[i] > 0 ? m / (double)ecount[i] : 1.0);  // refine.rs:44-50
            r.seed = hash3(lvl_seed, 0x7e71eull, 1);
            h_rf[i] = r;
        }
        h2d(c, icfg_lm.get(), h_lm.data(), K);
        h2d(c, icfg_rf.get(), h_rf.data(), K);
        zero(c, gain_inst.get(), K);
        MultiLevel ml_lm{inst.get(), icfg_lm.get(), gain_inst.get()};
        MultiLevel ml_rf{inst.get(), icfg_rf.get(), gain_inst.get()};
        {
            const size_t t = clock.start();
            MoveResult mr = local_move(c, *gl, ws, memb.get(), C, base_cfg, 0, sc, base_cfg.resolution, &ml_lm);
            clock.stop(t, &st.ms_local_move);
            st.local_move_sweeps += mr.sweeps;
            st.moves += mr.moves;
            st.alg_bytes_local_move += mr.alg_bytes;
        }
        d2h(c, gains.data(), gain_inst.get(), K);
        DBuf<uint32_t> collapse(c, nl);
        if (base_cfg.refine) {
            const size_t t = clock.start();
            refine(c, *gl, ws, memb.get(), collapse.get(), base_cfg, 0, sc, base_cfg.resolution, &ml_rf);
            clock.stop(t, &st.ms_refine);
        } else {
            d2d(c, collapse.get(), memb.get(), nl);
        }
        sync(c);  // gains
        for (uint32_t i = 0; i < K; ++i)
            if (!frozen[i]) mp.improvement[i] += (double)gains[i] * sc.scale;
        const size_t t_agg = clock.start();
        DBuf<uint32_t> grp(c, nl);
        if (base_cfg.refine) renumber_ranged(c, collapse.get(), nl, nl, d_bounds.get(), K, grp.get(), G);
        else renumber_by_instance(c, collapse.get(), inst.get(), nl, K, grp.get(), G);
        st.levels++;
        uint64_t Gtot = 0;
        bool any_shrinks = false;
        uint32_t running = 0;
        for (uint32_t i = 0; i < K; ++i) {
            Gtot += G[i];
            running += !frozen[i];
            if (!frozen[i] && G[i] >= nI[i]) frozen[i] = 1;  // the graph no longer shrinks (mod.rs:263-265)
            if (!frozen[i]) any_shrinks = true;
        }
        auto trace_level = [&]() {
            if (!trace) return;
            clock.collect();
            std::fprintf(stderr,
                         "[sc] union level %llu instances=%u running=%u n=%llu E=%llu exact=%d groups=%llu sweeps=%llu "
                         "moves=%llu lm=%.3fms ref=%.3fms agg=%.3fms\n",
                         (unsigned long long)level, K, running, (unsigned long long)nl, (unsigned long long)gl->E,
                         (int)gl->exact_w, (unsigned long long)Gtot,
                         (unsigned long long)(st.local_move_sweeps - before.local_move_sweeps),
                         (unsigned long long)(st.moves - before.moves), st.ms_local_move - before.ms_local_move,
                         st.ms_refine - before.ms_refine, st.ms_aggregate - before.ms_aggregate);
        };
        if (!any_shrinks) {
            clock.stop(t_agg, &st.ms_aggregate);
            trace_level();
            break;
        }
        std::unique_ptr<DevGraph> coarse(graph_aggregate(c, *gl, grp.get(), (uint32_t)Gtot));
        coarse->stream = c.stream;
        st.alg_bytes_aggregate += 12.0 * (double)gl->E + 12.0 * (double)nl + 8.0 * (double)coarse->E +
                                  24.0 * (double)coarse->n;
        DBuf<uint32_t> cm(c, Gtot), cm2(c, Gtot), inst_c(c, Gtot);
        k_scatter_coarse<<<grid_for(nl, TB), TB, 0, c.stream>>>(grp.get(), memb.get(), nl, cm.get());
        k_scatter_inst<<<grid_for(nl, TB), TB, 0, c.stream>>>(grp.get(), inst.get(), nl, inst_c.get());
        k_gather<<<grid_for(n0, TB), TB, 0, c.stream>>>(grp.get(), node_at.get(), n0);
        SC_LAUNCH_CHECK();
        c.launches += 3;
        C = renumber_ids(c, cm.get(), Gtot, C + nl, cm2.get());
        memb = std::move(cm2);
        inst = std::move(inst_c);
        owned = std::move(coarse);
        gl = owned.get();
        for (uint32_t i = 0; i < K; ++i) nI[i] = G[i];
        set_bounds();
        h2d(c, d_bounds.get(), bounds.data(), K + 1);
        clock.stop(t_agg, &st.ms_aggregate);
        trace_level();
    }
    // final ascending renumber per instance (mod.rs:282-286)
    const uint64_t nl = gl->n;
    DBuf<uint32_t> fin(c, nl);
    std::vector<uint32_t> Kc;
    renumber_by_instance(c, memb.get(), inst.get(), nl, K, fin.get(), Kc);
    out.labels.alloc(c, n0);
    d2d(c, out.labels.get(), node_at.get(), n0);
    k_gather<<<grid_for(n0, TB), TB, 0, c.stream>>>(fin.get(), out.labels.get(), n0);
    SC_LAUNCH_CHECK();
    c.launches++;
    mp.n_clusters = Kc;
    uint64_t tot = 0;
    for (uint32_t k : Kc) tot += k;
    out.n_clusters = tot;
}

// LeidenConfig::validate (mod.rs:117-153)
void validate_config(const sc_leiden_config& cfg) {
    double r = cfg.resolution;
    if (cfg.objective != SC_OBJECTIVE_RB && cfg.objective != SC_OBJECTIVE_CPM)
        fail(SC_E_INVALID_CONFIG, "invalid configuration: unknown objective %d", cfg.objective);
    if (!std::isfinite(r) || r < 0.0)
        fail(SC_E_INVALID_CONFIG, "invalid configuration: resolution must be finite and non-negative, got %s",
             fmt_f64(r).c_str());
    if (cfg.n_iterations == 0) fail(SC_E_INVALID_CONFIG, "invalid configuration: n_iterations must be at least 1");
    if (cfg.max_levels == 0) fail(SC_E_INVALID_CONFIG, "invalid configuration: max_levels must be at least 1");
    if (cfg.patience == 0) fail(SC_E_INVALID_CONFIG, "invalid configuration: patience must be at least 1");
    if (!std::isfinite(cfg.refine_randomness) || cfg.refine_randomness < 0.0)
        fail(SC_E_INVALID_CONFIG,
             "invalid configuration: refine_randomness must be finite and non-negative, got %s",
             fmt_f64(cfg.refine_randomness).c_str());
    if (cfg.has_max_community_weight &&
        (!std::isfinite(cfg.max_community_weight) || cfg.max_community_weight <= 0.0))
        fail(SC_E_INVALID_CONFIG,
             "invalid configuration: max_community_weight must be finite and positive, got %s",
             fmt_f64(cfg.max_community_weight).c_str());
}

}  // namespace

// leiden (mod.rs:168-204). initial_host: optional warm-start labels (n entries).
void leiden(Ctx& c, const DevGraph& g, const sc_leiden_config& cfg, const uint64_t* initial_host,
            uint32_t* d_labels_out, uint64_t* n_clusters) {
    validate_config(cfg);
    std::memset(&c.stats, 0, sizeof c.stats);
    PhaseClock clock(c);
    const size_t t_total = clock.start();
    zero(c, c.d_refine_ctr, 3);
    const uint64_t n = g.n;
    if (n == 0) {
        *n_clusters = 0;
        return;
    }
    uint64_t seed = cfg.has_seed ? cfg.seed : (uint64_t)std::random_device{}() << 32 ^ std::random_device{}();
    DBuf<uint32_t> labels(c, n);
    uint64_t C;
    if (initial_host) {
        DBuf<uint64_t> ini(c, n);
        h2d(c, ini.get(), initial_host, n);
        C = renumber_u64_labels(c, ini.get(), n, labels.get(), nullptr);
    } else {
        k_identity<<<grid_for(n, TB), TB, 0, c.stream>>>(labels.get(), n);
        c.launches++;
        C = n;
    }
    uint64_t clusters = C;
    uint64_t stagnant = 0;
    Workspace ws;  // shared by every level of every pass
    for (uint64_t it = 0; it < cfg.n_iterations; ++it) {
        PassOut po;
        run_pass(c, g, labels.get(), C, cfg, hash3(seed, it, 0x9a55ull), po, c.stats, clock, ws);
        labels = std::move(po.labels);
        C = po.n_clusters;
        clusters = C;
        c.stats.passes++;
        double scale = std::max(std::fabs(g.total_weight), 1.0);
        if (po.improvement <= cfg.tolerance * scale) {
            stagnant++;
            if (stagnant >= cfg.patience) break;
        } else {
            stagnant = 0;
        }
    }
    d2d(c, d_labels_out, labels.get(), n);
    clock.stop(t_total, &c.stats.ms_total);
    {
        Mailbox mb(c);
        const uint32_t* hs = mb.get(c.d_status, 1);
        const unsigned long long* hr = mb.get(c.d_refine_ctr, 3);
        mb.wait();
        const uint32_t status = *hs;
        c.stats.alg_bytes_refine = refine_alg_bytes(hr);
        raise_device_status(c, status);
    }
    clock.collect();
    c.stats.ms_other = c.stats.ms_total - c.stats.ms_local_move - c.stats.ms_refine - c.stats.ms_aggregate;
    c.stats.kernel_launches = c.launches;
    *n_clusters = clusters;
}

// Every instance's leiden() (mod.rs:168-204) over the disjoint union g of
// their graphs (instance I owns nodes [offset_I, offset_I + n[I]), in order),
// with instance I starting from initial[I] (host labels, nullable). Writes
// each instance's labels (consecutive from 0 within the instance) to
// d_labels_out in union node order and its cluster count to n_clusters.
void leiden_union(Ctx& c, const DevGraph& g, uint32_t K, const uint64_t* n, const sc_leiden_config* cfgs,
                  const uint64_t* const* initial, uint32_t* d_labels_out, uint64_t* n_clusters) {
    if (K == 0) return;
    for (uint32_t i = 0; i < K; ++i) validate_config(cfgs[i]);
    for (uint32_t i = 1; i < K; ++i) {
        if (cfgs[i].objective != cfgs[0].objective || (cfgs[i].refine != 0) != (cfgs[0].refine != 0) ||
            cfgs[i].has_max_community_weight != cfgs[0].has_max_community_weight ||
            (cfgs[i].has_max_community_weight && cfgs[i].max_community_weight != cfgs[0].max_community_weight))
            fail(SC_E_INVALID_CONFIG,
                 "invalid configuration: a batched run needs one objective kind, refine setting and "
                 "max_community_weight for all instances");
    }
    uint64_t total = 0;
    for (uint32_t i = 0; i < K; ++i) total += n[i];
    if (total != g.n) fail(SC_E_INTERNAL, "instance sizes do not add up to the union");
    std::memset(&c.stats, 0, sizeof c.stats);
    PhaseClock clock(c);
    const size_t t_total = clock.start();
    zero(c, c.d_refine_ctr, 3);
    MultiPass mp;
    mp.count = K;
    mp.cfgs = cfgs;
    mp.n0.assign(n, n + K);
    std::vector<uint64_t> seed(K);
    for (uint32_t i = 0; i < K; ++i)
        seed[i] = cfgs[i].has_seed ? cfgs[i].seed : ((uint64_t)std::random_device{}() << 32 ^ std::random_device{}());
    // initial union ids: each instance's compact ranks, offset past the instances before it
    DBuf<uint32_t> labels(c, std::max<uint64_t>(total, 1));
    std::vector<uint32_t> Ci(K);
    {
        uint64_t off = 0, cb = 0;
        for (uint32_t i = 0; i < K; ++i) {
            if (n[i] == 0) {
                Ci[i] = 0;
                continue;
            }
            if (initial && initial[i]) {
                DBuf<uint64_t> ini(c, n[i]);
                h2d(c, ini.get(), initial[i], n[i]);
                Ci[i] = renumber_u64_labels(c, ini.get(), n[i], labels.get() + off, nullptr);
            } else {
                k_identity<<<grid_for(n[i], TB), TB, 0, c.stream>>>(labels.get() + off, n[i]);
                c.launches++;
                Ci[i] = (uint32_t)n[i];
            }
            off += n[i];
        }
        // shift instance I's ids by the ids of the instances before it
        std::vector<uint32_t> shift(K);
        DBuf<uint32_t> d_shift(c, K), inst0(c, std::max<uint64_t>(total, 1));
        std::vector<uint64_t> b(K + 1, 0);
        for (uint32_t i = 0; i < K; ++i) {
            shift[i] = (uint32_t)(0u - (uint32_t)cb);  // k_sub_base subtracts: x - (-cb) = x + cb
            cb += Ci[i];
            b[i + 1] = b[i] + n[i];
        }
        DBuf<uint64_t> d_b(c, K + 1);
        h2d(c, d_b.get(), b.data(), K + 1);
        h2d(c, d_shift.get(), shift.data(), K);
        if (total) {
            k_inst_of_nodes<<<dim3(grid_for(*std::max_element(n, n + K), TB, 148u * 4u), K), TB, 0, c.stream>>>(
                d_b.get(), inst0.get());
            k_sub_base<<<grid_for(total, TB), TB, 0, c.stream>>>(labels.get(), inst0.get(), d_shift.get(), total);
            SC_LAUNCH_CHECK();
            c.launches += 2;
        }
    }
    uint64_t C = 0;
    for (uint32_t k : Ci) C += k;
    std::vector<uint64_t> stagnant(K, 0);
    std::vector<uint8_t> stopped(K, 0);
    std::vector<uint32_t> clusters(Ci.begin(), Ci.end());
    Workspace ws;
    uint64_t max_it = 0;
    for (uint32_t i = 0; i < K; ++i) max_it = std::max<uint64_t>(max_it, cfgs[i].n_iterations);
    for (uint64_t it = 0; it < max_it; ++it) {
        mp.active.assign(K, 0);
        mp.pass_seed.resize(K);
        bool any = false;
        for (uint32_t i = 0; i < K; ++i) {
            mp.active[i] = !stopped[i] && it < cfgs[i].n_iterations && n[i] > 0;
            any = any || mp.active[i];
            mp.pass_seed[i] = hash3(seed[i], it, 0x9a55ull);
        }
        if (!any) break;
        PassOut po;
        run_pass_multi(c, g, labels.get(), C, mp, po, c.stats, clock, ws);
        labels = std::move(po.labels);
        C = po.n_clusters;
        for (uint32_t i = 0; i < K; ++i) {
            clusters[i] = mp.n_clusters[i];
            if (!mp.active[i]) continue;
            const double scale = std::max(std::fabs(mp.total_weight0[i]), 1.0);
            if (mp.improvement[i] <= cfgs[i].tolerance * scale) {
                if (++stagnant[i] >= cfgs[i].patience) stopped[i] = 1;
            } else {
                stagnant[i] = 0;
            }
        }
        c.stats.passes++;
    }
    // union ids -> instance-local labels
    {
        std::vector<uint32_t> base(K);
        uint64_t cb = 0;
        for (uint32_t i = 0; i < K; ++i) {
            base[i] = (uint32_t)cb;
            cb += clusters[i];
        }
        DBuf<uint32_t> d_base(c, K), inst0(c, std::max<uint64_t>(total, 1));
        std::vector<uint64_t> b(K + 1, 0);
        for (uint32_t i = 0; i < K; ++i) b[i + 1] = b[i] + n[i];
        DBuf<uint64_t> d_b(c, K + 1);
        h2d(c, d_b.get(), b.data(), K + 1);
        h2d(c, d_base.get(), base.data(), K);
        if (total) {
            k_inst_of_nodes<<<dim3(grid_for(*std::max_element(n, n + K), TB, 148u * 4u), K), TB, 0, c.stream>>>(
                d_b.get(), inst0.get());
            k_sub_base<<<grid_for(total, TB), TB, 0, c.stream>>>(labels.get(), inst0.get(), d_base.get(), total);
            SC_LAUNCH_CHECK();
            c.launches += 2;
            d2d(c, d_labels_out, labels.get(), total);
        }
    }
    clock.stop(t_total, &c.stats.ms_total);
    {
        Mailbox mb(c);
        const uint32_t* hs = mb.get(c.d_status, 1);
        const unsigned long long* hr = mb.get(c.d_refine_ctr, 3);
        mb.wait();
        const uint32_t status = *hs;
        c.stats.alg_bytes_refine = refine_alg_bytes(hr);
        raise_device_status(c, status);
    }
    clock.collect();
    c.stats.ms_other = c.stats.ms_total - c.stats.ms_local_move - c.stats.ms_refine - c.stats.ms_aggregate;
    c.stats.kernel_launches = c.launches;
    for (uint32_t i = 0; i < K; ++i) n_clusters[i] = clusters[i];
}

bool tuning_valid(const sc_tuning& t) {
    return t.lanes8_max_degree <= 8 && t.lanes8_max_degree <= t.lanes16_max_degree && t.lanes16_max_degree <= 16 &&
           t.lanes16_max_degree <= t.lanes32_max_degree && t.lanes32_max_degree <= 32;
}

uint32_t autotune(Ctx& c, const DevGraph& g, const sc_leiden_config& cfg, sc_tuning* chosen, double* ms_chosen,
                  double* ms_default) {
    validate_config(cfg);
    static const sc_tuning candidates[] = {
        {8, 16, 32, 4096},   // default
        {0, 16, 32, 4096},   // no 8-lane groups
        {8, 8, 32, 4096},    // no 16-lane groups
        {8, 16, 16, 4096},   // degree 17-32 on the warp kernel
        {0, 0, 32, 4096},    // 32-lane groups only
        {8, 16, 32, 0},      // never fuse a small batch
        {8, 16, 32, 1024},
        {8, 16, 32, 16384},
    };
    sc_leiden_config one = cfg;
    one.n_iterations = 1;
    one.max_levels = 1;
    const sc_tuning saved = c.tuning;
    DBuf<uint32_t> lab(c, g.n);
    uint64_t ncl = 0;
    double best = INFINITY, def = 0.0;
    sc_tuning pick = candidates[0];
    try {
        c.tuning = candidates[0];
        leiden(c, g, one, nullptr, lab.get(), &ncl);  // warm-up: pools, caches, first-call costs
        uint32_t k = 0;
        for (const sc_tuning& t : candidates) {
            c.tuning = t;
            leiden(c, g, one, nullptr, lab.get(), &ncl);
            const double ms = c.stats.ms_total;
            if (k == 0) def = ms;
            if (ms < best) {
                best = ms;
                pick = t;
            }
            ++k;
        }
    } catch (...) {
        c.tuning = saved;
        throw;
    }
    c.tuning = pick;
    if (chosen) *chosen = pick;
    if (ms_chosen) *ms_chosen = best;
    if (ms_default) *ms_default = def;
    return (uint32_t)(sizeof candidates / sizeof candidates[0]);
}

}  // namespace sc
