// sc_mlp.cu — learned warm start for Leiden: an edge MLP proposes an initial
// membership that leiden_from then refines.
//
// Community ids are arbitrary (any permutation of a partition is the same
// partition), so the network does not classify nodes into ids: it scores each
// undirected edge (i, j) from the features of its two endpoints, their shared
// neighbourhood, the partitions found at neighbouring resolutions and the kNN
// embedding the graph came from, F = 15:
//   w, log1p(k_i) + log1p(k_j), |log1p(k_i) - log1p(k_j)|, log(d_i) + log(d_j),
//   |log d_i - log d_j|, w/k_i + w/k_j, log(gamma), gamma k_i k_j / (2 m w),
//   sum_c min(w_ic, w_jc) / min(k_i, k_j), |N(i) & N(j)| / min(d_i, d_j),
//   [i, j together at the coarser neighbour], [i, j together at the finer one],
//   (a_i(C(j)) + a_j(C(i))) / 2 at the coarser neighbour C, the same at the
//   finer one, |y_i - y_j|^2 / ((s_i + s_j) / 2)
// (w edge weight, k strength, d degree, gamma the RB resolution; the 8th is the
// configuration-model null term relative to the edge, the quantity local moving
// weighs; the 9th and 10th compare the endpoints' neighbour histograms, c over
// the common neighbours other than i and j; a_i(L) is the share of k_i on the
// neighbours x != i with label L, the node's neighbour-label histogram read at
// the other endpoint's community; y_i is the node's embedding projected to
// EMB_R components by a fixed sign matrix and s_i the mean of |y_i - y_x|^2 over
// its neighbours, so the last is the edge's length in the embedding relative
// to the local scale; features 10-13 are 0 without a context, 14 without an
// embedding) and outputs the logit that i and j share a community:
//   h = relu(x W1 + b1) (hidden H), z = h . w2 + b2.
// Weights are BF16 in the forward pass with FP32 accumulation; an FP32 master
// copy is updated by Adam. Training labels are partitions plain Leiden found;
// the proposal is the connected components of the confident edges (p >
// threshold) between core nodes, a core node being one whose share of
// confident edges is at least core_fraction. Edges at a community boundary
// look like interior edges to local features, so components of all confident
// edges chain neighbouring communities together; a boundary node has some
// unconfident edge, stays a singleton, and is placed by local moving.
//
// Kernels: the contraction runs on the tensor cores (mma.sync BF16 with FP32
// accumulation, 16 edges per warp step, features and hidden gradients split
// into two BF16 parts so the sums keep FP32-level accuracy); gradients
// accumulate in registers, then per block in shared memory, then in a
// fixed-order reduction over blocks (deterministic). The features that depend
// on neither gamma nor a context (EDGE_SF values per edge) are computed once
// per graph, a warp per row (a block per hub row), and kept with the graph;
// each call assembles them with log(gamma), the null term and the context
// features (label shares from per-chunk label groups).
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <vector>

#include "sc_prims.cuh"

namespace sc {

constexpr int MLP_F = 15;  // plus a constant 1 as the 16th MMA column
constexpr int MLP_H = 128;
constexpr int MLP_NPARAM = MLP_F * MLP_H + MLP_H + MLP_H + 1;  // W1, b1, w2, b2

struct Mlp {
    int device = 0;
    float* master = nullptr;  // MLP_NPARAM, FP32
    float* m = nullptr;       // Adam first moment
    float* v = nullptr;       // Adam second moment
    float* norm = nullptr;    // 2 MLP_F: feature means, then inverse standard deviations
    bool has_norm = false;
    uint64_t step = 0;
};

namespace {

constexpr unsigned TB = 256;
constexpr int MLP_BLOCKS = 148 * 4;

// For every stored entry e = (i, j): Σ w_ix over the neighbours x != i of i
// with label(x) = label(j), over k_i — the entry of i's neighbour-label
// histogram at j's community, as a share of i's strength. A warp takes a run
// of the row's 32-entry chunks (the e-chunks) and walks all its chunks (the
// x-chunks): in each x-chunk the lanes of one label find each other with
// __match_any_sync, the lowest of them sums the group's weights in lane order,
// and the warp broadcasts (label, sum) once per distinct label; a lane adds
// the sums of its entry's label. Per entry the order is fixed (chunks
// ascending, lanes ascending inside a chunk), so the result is the same on
// every run.
__device__ void label_share_chunks(const uint32_t* __restrict__ nbr,
                                   const float* __restrict__ w, const uint32_t* __restrict__ label, uint32_t i,
                                   uint64_t a, uint64_t b, uint64_t ce_begin, uint64_t ce_step, double ki,
                                   float* __restrict__ share) {
    const int lane = threadIdx.x & 31;
    for (uint64_t e0 = a + ce_begin * 32; e0 < b; e0 += ce_step * 32) {
        const uint64_t e = e0 + lane;
        const uint32_t L = e < b ? label[nbr[e]] : 0u;
        double acc = 0.0;
        for (uint64_t x0 = a; x0 < b; x0 += 32) {
            const uint64_t x = x0 + lane;
            bool valid = false;
            uint32_t lx = 0u;
            float wx = 0.0f;
            if (x < b) {
                const uint32_t v = nbr[x];
                valid = v != i;
                lx = label[v];
                wx = w[x];
            }
            const unsigned long long key = valid ? (unsigned long long)lx : ((1ull << 32) | (unsigned)lane);
            const unsigned peers = __match_any_sync(0xFFFFFFFFu, key);
            double sum = 0.0;
            for (int t = 0; t < 32; ++t) {
                const float wt = __shfl_sync(0xFFFFFFFFu, wx, t);
                if ((peers >> t) & 1u) sum += (double)wt;
            }
            unsigned leaders = __ballot_sync(0xFFFFFFFFu, valid && (__ffs(peers) - 1) == lane);
            while (leaders) {
                const int l = __ffs(leaders) - 1;
                leaders &= leaders - 1;
                const uint32_t Ll = __shfl_sync(0xFFFFFFFFu, lx, l);
                const double Sl = __shfl_sync(0xFFFFFFFFu, sum, l);
                if (Ll == L) acc += Sl;
            }
        }
        if (e < b) share[e] = (float)(acc / ki);
    }
}

// Rows of at most 32 chunks: a warp per row. Longer rows are left to
// k_label_share_big.
__global__ void k_label_share(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                              const float* __restrict__ w, const uint32_t* __restrict__ label,
                              const double* __restrict__ strength, uint64_t n, float* __restrict__ share) {
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < n; i += nwarps) {
        const uint64_t a = ptr[i], b = ptr[i + 1];
        if (b - a > 32 * 32) continue;
        label_share_chunks(nbr, w, label, (uint32_t)i, a, b, 0, 1, fmax(strength[i], 1e-300), share);
    }
}

// Rows of more than 32 chunks (listed in big[0, nbig)): a block per row, its
// warps on alternate e-chunks.
__global__ void k_label_share_big(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                                  const float* __restrict__ w, const uint32_t* __restrict__ label,
                                  const double* __restrict__ strength, const uint32_t* __restrict__ big,
                                  uint32_t nbig, float* __restrict__ share) {
    const uint64_t wib = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t k = blockIdx.x; k < nbig; k += gridDim.x) {
        const uint32_t i = big[k];
        label_share_chunks(nbr, w, label, i, ptr[i], ptr[i + 1], wib, nw, fmax(strength[i], 1e-300), share);
    }
}

// The stored entry (j, i): rows are strictly increasing, the graph symmetric.
__device__ __forceinline__ uint64_t entry_of(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr,
                                             uint32_t j, uint32_t i) {
    uint64_t lo = ptr[j], hi = ptr[j + 1];
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (nbr[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// s_i: mean of |y_i - y_x|^2 over the neighbours x != i (0 for none).
__global__ void k_emb_scale(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr, uint64_t n,
                            const float* __restrict__ emb, float* scale) {
    static_assert(EMB_R == 16, "four float4 loads per projected point");
    const float4* e4 = reinterpret_cast<const float4*>(emb);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float4 yi[4];
        for (int q = 0; q < 4; ++q) yi[q] = e4[i * 4 + q];
        double s = 0.0;
        uint64_t cnt = 0;
        for (uint64_t x = ptr[i]; x < ptr[i + 1]; ++x) {
            const uint32_t v = nbr[x];
            if (v == (uint32_t)i) continue;
            float t = 0.0f;
            for (int q = 0; q < 4; ++q) {
                const float4 yv = e4[(uint64_t)v * 4 + q];
                const float d0 = yi[q].x - yv.x, d1 = yi[q].y - yv.y, d2 = yi[q].z - yv.z, d3 = yi[q].w - yv.w;
                t = __fmaf_rn(d0, d0, t);
                t = __fmaf_rn(d1, d1, t);
                t = __fmaf_rn(d2, d2, t);
                t = __fmaf_rn(d3, d3, t);
            }
            s += (double)t;
            ++cnt;
        }
        scale[i] = cnt ? (float)(s / (double)cnt) : 0.0f;
    }
}

__global__ void k_node_logs(const uint64_t* __restrict__ ptr, const double* __restrict__ strength, uint64_t n,
                            float2* nlog) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        nlog[i] = make_float2((float)log1p(strength[i]), (float)log((double)(ptr[i + 1] - ptr[i])));
}

// Upper entries (neighbour > row) per row: the undirected edges i < j that
// row i owns. cnt[n] = 0, so the exclusive sum ends with the edge count.
__global__ void k_upper_counts(const uint64_t* __restrict__ ptr, const uint32_t* __restrict__ nbr, uint64_t n,
                               uint64_t* cnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x)
        cnt[i] = i < n ? ptr[i + 1] - entry_of(ptr, nbr, (uint32_t)i, (uint32_t)i + 1u) : 0;
}

constexpr int ROW_STAGE = 256;   // row entries a warp keeps in shared memory (rows up to this size)
constexpr int BIG_STAGE = 8192;  // row entries a block keeps in shared memory for a larger row
constexpr int EDGE_LANES = 8;    // lanes per edge: a warp works on 4 edges of a row at once

// The structural features of an edge, stored with the graph (EDGE_SF per
// edge): features 0-5 of the MLP, k_i k_j / (2 m w) (feature 7 over gamma),
// features 8 and 9, and feature 14.
constexpr int EDGE_SF = 10;

struct FeatArgs {
    const uint64_t* ptr;
    const uint32_t* nbr;
    const float* w;
    const double* strength;
    const float2* nlog;  // per node: log1p(strength), log(degree)
    double two_m;
    const float* emb;
    const float* emb_scale;
    const uint64_t* base;
    float* sf;
    uint32_t* ei;
    uint32_t* ej;
    uint64_t* ee;
};

// Row i's entries [a, b), staged (ids and weights at x - a in shared memory)
// or not (read from the graph).
struct RowView {
    uint32_t i;
    uint64_t a, b, us;  // us: first entry with neighbour > i
    const uint32_t* sid;
    const float* sw;
    bool staged;
};

// The structural features of edge (i, nbr[e]) by the 8 lanes of a group (gl = lane in
// the group). Called by all 32 lanes of the warp together (the reductions
// shuffle across the full warp, each group within itself); inactive groups
// take part with nothing to do. The 8 lanes walk one endpoint's row (lane l
// takes entries l, l + 8, ...) and look each entry up in the other row by
// binary search: row i from shared memory when staged, unless row j is much
// the shorter one. Sums are reductions over the 8 lanes in a fixed tree; lane
// l writes features l and l + 8. Edge (i, j) lands at base[i] + its rank among
// i's upper entries, i.e. in ascending (i, j) order, with its endpoints and
// its entries (i, j) and (j, i).
__device__ __forceinline__ void edge_group(const FeatArgs& A, const RowView& R, uint64_t e, bool active, int gl) {
    const uint64_t* __restrict__ ptr = A.ptr;
    const uint32_t* __restrict__ nbr = A.nbr;
    const float* __restrict__ w = A.w;
    const uint32_t i = R.i;
    const uint64_t di_n = R.b - R.a;
    const uint32_t j = active ? (R.staged ? R.sid[e - R.a] : nbr[e]) : i;
    const uint64_t ja = ptr[j], jb = ptr[j + 1];
    const uint64_t dj_n = jb - ja;
    // common neighbours c != i, j: walk one row, search the other
    const bool walk_j = R.staged ? dj_n <= 8 * di_n : dj_n <= di_n;
    double cw = 0.0;
    uint32_t cn = 0;
    unsigned long long rev = ~0ull;  // the entry (j, i), found while walking row j
    const uint64_t wa = active ? (walk_j ? ja : R.a) : 0, wb = active ? (walk_j ? jb : R.b) : 0;
    for (uint64_t x = wa + gl; x < wb; x += EDGE_LANES) {
        const bool from_smem = !walk_j && R.staged;
        const uint32_t cc = from_smem ? R.sid[x - R.a] : nbr[x];
        const float wc = from_smem ? R.sw[x - R.a] : w[x];
        if (walk_j && cc == i) rev = x;
        if (cc == i || cc == j) continue;
        float wo = 0.0f;
        bool found = false;
        if (walk_j && R.staged) {
            uint32_t lo = 0, hi = (uint32_t)di_n;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (R.sid[mid] < cc) lo = mid + 1;
                else hi = mid;
            }
            if (lo < di_n && R.sid[lo] == cc) {
                found = true;
                wo = R.sw[lo];
            }
        } else {
            const uint64_t oa = walk_j ? R.a : ja, ob = walk_j ? R.b : jb;
            uint64_t lo = oa, hi = ob;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (nbr[mid] < cc) lo = mid + 1;
                else hi = mid;
            }
            if (lo < ob && nbr[lo] == cc) {
                found = true;
                wo = w[lo];
            }
        }
        if (found) {
            cw += (double)fminf(wc, wo);
            ++cn;
        }
    }
    for (int o = EDGE_LANES / 2; o; o >>= 1) {
        cw += __shfl_xor_sync(0xFFFFFFFFu, cw, o);
        cn += __shfl_xor_sync(0xFFFFFFFFu, cn, o);
        rev = min(rev, (unsigned long long)__shfl_xor_sync(0xFFFFFFFFu, rev, o));
    }
    if (active && rev == ~0ull) rev = entry_of(ptr, nbr, j, i);
    float ed2 = 0.0f;
    if (A.emb) {
        float t = 0.0f;
        if (active)
            for (int r = gl; r < EMB_R; r += EDGE_LANES) {
                const float dd = A.emb[(uint64_t)i * EMB_R + r] - A.emb[(uint64_t)j * EMB_R + r];
                t = __fmaf_rn(dd, dd, t);
            }
        for (int o = EDGE_LANES / 2; o; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
        ed2 = t;
    }
    if (!active) return;
    const uint64_t pos = A.base[i] + (e - R.us);
    // every lane of the group forms all EDGE_SF values (same addresses: one
    // transaction per load), then writes values gl and gl + 8
    const float wij = R.staged ? R.sw[e - R.a] : w[e];
    const double kid = A.strength[i], kjd = A.strength[j];
    const float ki = (float)kid, kj = (float)kjd, di = (float)di_n, dj = (float)dj_n;
    const float2 li = A.nlog[i], lj = A.nlog[j];
    static_assert(EDGE_SF == 10 && EDGE_LANES == 8, "lane gl writes values gl and gl + 8");
    const float v0 = wij, v1 = li.x + lj.x, v2 = fabsf(li.x - lj.x), v3 = li.y + lj.y, v4 = fabsf(li.y - lj.y);
    const float v5 = wij / fmaxf(ki, 1e-30f) + wij / fmaxf(kj, 1e-30f);
    const float v6 = A.two_m > 0.0 ? (float)(kid * kjd / (A.two_m * fmax((double)wij, 1e-300))) : 0.0f;
    const float v7 = (float)(cw / fmax(fmin(kid, kjd), 1e-300));
    const float v8 = (float)cn / fmaxf(fminf(di, dj), 1.0f);
    const float v9 = A.emb ? ed2 / fmaxf(0.5f * (A.emb_scale[i] + A.emb_scale[j]), 1e-30f) : 0.0f;
    const float o0 = gl == 0 ? v0 : gl == 1 ? v1 : gl == 2 ? v2 : gl == 3 ? v3 : gl == 4 ? v4 : gl == 5 ? v5
                   : gl == 6 ? v6 : v7;
    const float o1 = gl == 0 ? v8 : v9;
    A.sf[pos * EDGE_SF + gl] = o0;
    if (gl < EDGE_SF - 8) A.sf[pos * EDGE_SF + gl + 8] = o1;
    if (gl == 0) {
        A.ei[pos] = i;
        A.ej[pos] = j;
        A.ee[2 * pos] = e;
        A.ee[2 * pos + 1] = rev;
    }
}

// The MLP's input of every edge: the structural values, log(gamma), gamma
// times the null-term ratio, and the context features (co-membership at the
// coarser and finer partitions, the two endpoints' label shares).
__global__ void k_assemble(uint64_t M, const float* __restrict__ sf, const uint32_t* __restrict__ ei,
                           const uint32_t* __restrict__ ej, const uint64_t* __restrict__ ee, float lgam,
                           double gamma, const uint32_t* __restrict__ coarse, const uint32_t* __restrict__ fine,
                           const float* __restrict__ share_c, const float* __restrict__ share_f,
                           float* __restrict__ feat) {
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < M; m += (uint64_t)gridDim.x * blockDim.x) {
        const float* s = sf + m * EDGE_SF;
        float* f = feat + m * MLP_F;
        for (int k = 0; k < 6; ++k) f[k] = s[k];
        f[6] = lgam;
        f[7] = (float)(gamma * (double)s[6]);
        f[8] = s[7];
        f[9] = s[8];
        const uint32_t i = ei[m], j = ej[m];
        const uint64_t e = ee[2 * m], rev = ee[2 * m + 1];
        f[10] = coarse ? (coarse[i] == coarse[j] ? 1.0f : 0.0f) : 0.0f;
        f[11] = fine ? (fine[i] == fine[j] ? 1.0f : 0.0f) : 0.0f;
        f[12] = coarse ? 0.5f * (share_c[e] + share_c[rev]) : 0.0f;
        f[13] = fine ? 0.5f * (share_f[e] + share_f[rev]) : 0.0f;
        f[14] = s[9];
    }
}

// Rows of at most ROW_STAGE entries: a warp per row, 4 edges at a time.
// Larger rows are left to k_edge_big_rows.
__global__ void __launch_bounds__(TB, 4) k_edge_rows(FeatArgs A, uint64_t n) {
    __shared__ uint32_t s_id[TB / 32][ROW_STAGE];
    __shared__ float s_w[TB / 32][ROW_STAGE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int grp = lane / EDGE_LANES, gl = lane % EDGE_LANES;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t iw = warp; iw < n; iw += nwarps) {
        RowView R;
        R.i = (uint32_t)iw;
        R.a = A.ptr[R.i];
        R.b = A.ptr[R.i + 1];
        if (R.b - R.a > (uint64_t)ROW_STAGE) continue;
        R.sid = s_id[wib];
        R.sw = s_w[wib];
        R.staged = true;
        __syncwarp();
        uint32_t below = 0;  // entries with neighbour <= i
        for (uint64_t x = lane; x < R.b - R.a; x += 32) {
            const uint32_t v = A.nbr[R.a + x];
            s_id[wib][x] = v;
            s_w[wib][x] = A.w[R.a + x];
            below += v <= R.i;
        }
        for (int o = 16; o; o >>= 1) below += __shfl_xor_sync(0xFFFFFFFFu, below, o);
        __syncwarp();
        R.us = R.a + below;
        for (uint64_t e0 = R.us; e0 < R.b; e0 += 32 / EDGE_LANES) {
            const uint64_t e = e0 + grp;
            edge_group(A, R, e, e < R.b, gl);
        }
    }
}

// Rows of more than ROW_STAGE entries (hubs of the kNN graph: a point in many
// other points' lists), listed in big[0, nbig): a block per row, its 32 lane
// groups on 32 edges at a time, the row staged in shared memory up to
// BIG_STAGE entries (beyond that the searches read the graph).
__global__ void __launch_bounds__(TB) k_edge_big_rows(FeatArgs A, const uint32_t* __restrict__ big, uint32_t nbig) {
    extern __shared__ __align__(16) unsigned char big_smem[];
    uint32_t* sid = reinterpret_cast<uint32_t*>(big_smem);
    float* sw = reinterpret_cast<float*>(big_smem + BIG_STAGE * sizeof(uint32_t));
    __shared__ uint32_t s_below;
    const int lane = threadIdx.x & 31;
    const int grp = threadIdx.x / EDGE_LANES, gl = lane % EDGE_LANES;
    constexpr int GROUPS = TB / EDGE_LANES;
    for (uint32_t k = blockIdx.x; k < nbig; k += gridDim.x) {
        RowView R;
        R.i = big[k];
        R.a = A.ptr[R.i];
        R.b = A.ptr[R.i + 1];
        R.staged = R.b - R.a <= (uint64_t)BIG_STAGE;
        R.sid = sid;
        R.sw = sw;
        __syncthreads();
        if (threadIdx.x == 0) s_below = 0;
        __syncthreads();
        uint32_t below = 0;
        for (uint64_t x = threadIdx.x; x < R.b - R.a; x += blockDim.x) {
            const uint32_t v = A.nbr[R.a + x];
            if (R.staged) {
                sid[x] = v;
                sw[x] = A.w[R.a + x];
            }
            below += v <= R.i;
        }
        for (int o = 16; o; o >>= 1) below += __shfl_xor_sync(0xFFFFFFFFu, below, o);
        if (lane == 0) atomicAdd(&s_below, below);
        __syncthreads();
        R.us = R.a + s_below;
        for (uint64_t e0 = R.us; e0 < R.b; e0 += GROUPS) {
            const uint64_t e = e0 + grp;
            edge_group(A, R, e, e < R.b, gl);
        }
    }
}

// Rows of more than `limit` entries (in no particular order: each row's
// results have fixed places).
__global__ void k_big_rows(const uint64_t* __restrict__ ptr, uint64_t n, uint64_t limit, uint32_t* big,
                           unsigned* nbig) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (ptr[i + 1] - ptr[i] > limit) big[atomicAdd(nbig, 1u)] = (uint32_t)i;
}

// Per-feature mean / inverse std over the edges (fixed-order block partials).
// The scaler is fitted once, on the first graph a model trains on, and is part
// of the model from then on: a feature that is constant within one graph (the
// resolution) keeps its value across graphs instead of standardising to zero.
constexpr int MLP_GAMMA_FEATURE = 6;

__global__ void k_feat_partials(const float* __restrict__ feat, uint64_t M, double* partial) {
    __shared__ double s[2 * MLP_F][TB / 32];
    double acc[2 * MLP_F] = {};
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < M;
         e += (uint64_t)gridDim.x * blockDim.x)
        for (int f = 0; f < MLP_F; ++f) {
            const double x = feat[e * MLP_F + f];
            acc[f] += x;
            acc[MLP_F + f] += x * x;
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int f = 0; f < 2 * MLP_F; ++f) {
        double x = acc[f];
        for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xFFFFFFFFu, x, o);
        if (lane == 0) s[f][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < 2 * MLP_F) {
        double x = 0.0;
        for (int k = 0; k < (int)(blockDim.x / 32); ++k) x += s[threadIdx.x][k];
        partial[blockIdx.x * 2 * MLP_F + threadIdx.x] = x;
    }
}

__global__ void k_feat_finalize(const double* __restrict__ partial, int nblocks, uint64_t M, float* norm) {
    if (threadIdx.x >= MLP_F) return;
    double s = 0.0, s2 = 0.0;
    for (int b = 0; b < nblocks; ++b) {
        s += partial[b * 2 * MLP_F + threadIdx.x];
        s2 += partial[b * 2 * MLP_F + MLP_F + threadIdx.x];
    }
    const double mean = M ? s / (double)M : 0.0;
    const double var = M ? fmax(s2 / (double)M - mean * mean, 0.0) : 0.0;
    if (threadIdx.x == MLP_GAMMA_FEATURE) {  // log(gamma): passed through unscaled
        norm[threadIdx.x] = 0.0f;
        norm[MLP_F + threadIdx.x] = 1.0f;
        return;
    }
    norm[threadIdx.x] = (float)mean;
    norm[MLP_F + threadIdx.x] = (float)(var > 1e-12 ? 1.0 / sqrt(var) : 1.0);
}

__global__ void k_normalize(float* feat, uint64_t M, const float* __restrict__ norm) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < M * MLP_F;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const int f = (int)(i % MLP_F);
        feat[i] = (feat[i] - norm[f]) * norm[MLP_F + f];
    }
}


__global__ void k_to_bf16(const float* __restrict__ master, __nv_bfloat16* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x)
        out[i] = __float2bfloat16_rn(master[i]);
}

// ------------------------------------------------------------ tensor-core forward / backward
// Forward (and with GRAD, backward) over the edge stream on the tensor cores
// (mma.sync m16n8k16, BF16 in, FP32 accumulate). Parameter layout:
// W1[f * H + u], b1[u], w2[u], b2. A warp takes 16 edges per step: X (16
// edges x 16 columns: the MLP_F = 15 features, then a 1 in the last column of
// every real edge) as two BF16 parts x = x_hi + x_lo; H = X W1 is 16 MMAs per
// part (W1 is BF16 already, its row 15 zero, so the 1 adds nothing). Thread
// (g, t) of the warp holds H[g][8n + 2t + j] and H[g + 8][...] for the 16
// n-tiles n. Backward: dW1 = X^T dH with dH = relu'(H) dz w2 split in BF16
// parts too (three MMAs per n-tile: hi.hi, hi.lo, lo.hi); row 15 of X^T (the
// ones) gives db1 in the same MMAs. dw2 = H^T dz and db2 fold per lane; the
// block then reduces every warp's parameters in warp order and the grid in
// block order (deterministic).
constexpr int TC_WARPS = 4;
constexpr int TC_THREADS = 32 * TC_WARPS;

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Shared tiles keep rows of XS = 24 BF16 (12 words): the fragment reads of
// lanes (g, t) then fall on banks 12 g + t, all 32 distinct.
constexpr int XS = 24;

struct alignas(16) TcSmem {
    __nv_bfloat16 w1t[MLP_H * XS];  // W1 transposed: [unit][feature], features 12..15 zero
    float b1[MLP_H], w2[MLP_H];
    float b2;
};

// per warp: X and X^T (hi and lo parts) 16 x XS each, dH^T (hi and lo) MLP_H x XS
constexpr int TC_WARP_TILE = 4 * 16 * XS + 2 * MLP_H * XS;

__device__ __forceinline__ uint32_t word_at(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

template <bool GRAD>
__global__ void __launch_bounds__(TC_THREADS) k_mlp_tc(const float* __restrict__ feat, const uint8_t* __restrict__ label,
                                                       uint64_t M, const __nv_bfloat16* __restrict__ wb,
                                                       float* __restrict__ out_p, float* __restrict__ partial_grad,
                                                       double* __restrict__ partial_loss) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(smem_raw);
    __nv_bfloat16* wbase = reinterpret_cast<__nv_bfloat16*>(smem_raw + sizeof(TcSmem));
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    __nv_bfloat16* xh = wbase + (size_t)wid * TC_WARP_TILE;  // [edge][feature]
    __nv_bfloat16* xl = xh + 16 * XS;
    __nv_bfloat16* xth = xl + 16 * XS;  // [feature][edge]
    __nv_bfloat16* xtl = xth + 16 * XS;
    __nv_bfloat16* dhh = xtl + 16 * XS;  // [unit][edge]
    __nv_bfloat16* dhl = dhh + MLP_H * XS;
    for (int i = threadIdx.x; i < MLP_H * 16; i += blockDim.x) {
        const int u = i >> 4, f = i & 15;
        S.w1t[u * XS + f] = f < MLP_F ? wb[f * MLP_H + u] : __float2bfloat16_rn(0.0f);
    }
    for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
        S.b1[i] = __bfloat162float(wb[MLP_F * MLP_H + i]);
        S.w2[i] = __bfloat162float(wb[MLP_F * MLP_H + MLP_H + i]);
    }
    if (threadIdx.x == 0) S.b2 = __bfloat162float(wb[MLP_F * MLP_H + 2 * MLP_H]);
    __syncthreads();
    float gw1[16][4];  // dW1 (rows f = g, g + 8) and, in row 12, db1
    float gw2[16][2];  // dw2 partials of this lane's columns
#pragma unroll
    for (int n = 0; n < 16; ++n) {
        gw1[n][0] = gw1[n][1] = gw1[n][2] = gw1[n][3] = 0.0f;
        gw2[n][0] = gw2[n][1] = 0.0f;
    }
    float gb2 = 0.0f;
    double loss = 0.0;
    const uint64_t warp_g = (uint64_t)blockIdx.x * TC_WARPS + wid;
    const uint64_t nwarps = (uint64_t)gridDim.x * TC_WARPS;
    for (uint64_t base = warp_g * 16; base < M; base += nwarps * 16) {
        // X tile: lane l stages edge l / 2, features 8 (l % 2) .. +7 (a 1 in column 12)
        {
            const int e = lane >> 1, f0 = (lane & 1) * 8;
            const uint64_t ge = base + e;
            const bool valid = ge < M;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int f = f0 + j;
                float x = 0.0f;
                if (valid) x = f < MLP_F ? feat[ge * MLP_F + f] : (f == MLP_F ? 1.0f : 0.0f);
                const __nv_bfloat16 hi = __float2bfloat16_rn(x);
                const __nv_bfloat16 lo = __float2bfloat16_rn(x - __bfloat162float(hi));
                xh[e * XS + f] = hi;
                xl[e * XS + f] = lo;
                xth[f * XS + e] = hi;
                xtl[f * XS + e] = lo;
            }
        }
        __syncwarp();
        const uint32_t ah[4] = {word_at(xh + g * XS + 2 * t), word_at(xh + (g + 8) * XS + 2 * t),
                                word_at(xh + g * XS + 2 * t + 8), word_at(xh + (g + 8) * XS + 2 * t + 8)};
        const uint32_t al[4] = {word_at(xl + g * XS + 2 * t), word_at(xl + (g + 8) * XS + 2 * t),
                                word_at(xl + g * XS + 2 * t + 8), word_at(xl + (g + 8) * XS + 2 * t + 8)};
        float h[16][4];
        float z0 = 0.0f, z1 = 0.0f;
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const __nv_bfloat16* wc = S.w1t + (8 * n + g) * XS;  // this lane's B column
            const uint32_t b0 = word_at(wc + 2 * t), b1 = word_at(wc + 2 * t + 8);
            float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            mma_bf16_16816(c, ah, b0, b1);
            mma_bf16_16816(c, al, b0, b1);
            const int c0 = 8 * n + 2 * t;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                h[n][j] = fmaxf(c[j] + S.b1[c0 + j], 0.0f);
                h[n][2 + j] = fmaxf(c[2 + j] + S.b1[c0 + j], 0.0f);
                z0 = __fmaf_rn(h[n][j], S.w2[c0 + j], z0);
                z1 = __fmaf_rn(h[n][2 + j], S.w2[c0 + j], z1);
            }
        }
        // the four lanes of a quad hold the same rows: fold their columns
        z0 += __shfl_xor_sync(0xFFFFFFFFu, z0, 1);
        z0 += __shfl_xor_sync(0xFFFFFFFFu, z0, 2);
        z1 += __shfl_xor_sync(0xFFFFFFFFu, z1, 1);
        z1 += __shfl_xor_sync(0xFFFFFFFFu, z1, 2);
        z0 += S.b2;
        z1 += S.b2;
        const float p0 = 1.0f / (1.0f + expf(-z0)), p1 = 1.0f / (1.0f + expf(-z1));
        const uint64_t e0 = base + g, e1 = base + g + 8;
        if (!GRAD) {
            if (t == 0) {
                if (e0 < M) out_p[e0] = p0;
                if (e1 < M) out_p[e1] = p1;
            }
            __syncwarp();
            continue;
        }
        const float y0 = (e0 < M && label[e0]) ? 1.0f : 0.0f, y1 = (e1 < M && label[e1]) ? 1.0f : 0.0f;
        const float dz0 = e0 < M ? p0 - y0 : 0.0f, dz1 = e1 < M ? p1 - y1 : 0.0f;
        if (t == 0) {
            // BCE with logits, numerically stable: max(z,0) - z y + log(1 + e^-|z|)
            if (e0 < M) loss += (double)(fmaxf(z0, 0.0f) - z0 * y0 + log1pf(expf(-fabsf(z0))));
            if (e1 < M) loss += (double)(fmaxf(z1, 0.0f) - z1 * y1 + log1pf(expf(-fabsf(z1))));
            gb2 += dz0 + dz1;
        }
        // dH^T (this lane's units; edges g, g + 8) into shared memory as BF16 parts; dw2 partials
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const int c0 = 8 * n + 2 * t;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const float w = S.w2[c0 + j];
                gw2[n][j] = __fmaf_rn(h[n][j], dz0, gw2[n][j]);
                gw2[n][j] = __fmaf_rn(h[n][2 + j], dz1, gw2[n][j]);
                const float d0 = h[n][j] > 0.0f ? dz0 * w : 0.0f;
                const float d1 = h[n][2 + j] > 0.0f ? dz1 * w : 0.0f;
                const __nv_bfloat16 h0 = __float2bfloat16_rn(d0), h1 = __float2bfloat16_rn(d1);
                __nv_bfloat16* rh = dhh + (c0 + j) * XS;
                __nv_bfloat16* rl = dhl + (c0 + j) * XS;
                rh[g] = h0;
                rl[g] = __float2bfloat16_rn(d0 - __bfloat162float(h0));
                rh[g + 8] = h1;
                rl[g + 8] = __float2bfloat16_rn(d1 - __bfloat162float(h1));
            }
        }
        __syncwarp();
        // X^T as the A operand: rows = features (g, g + 8), columns = edges
        const uint32_t th[4] = {word_at(xth + g * XS + 2 * t), word_at(xth + (g + 8) * XS + 2 * t),
                                word_at(xth + g * XS + 2 * t + 8), word_at(xth + (g + 8) * XS + 2 * t + 8)};
        const uint32_t tl[4] = {word_at(xtl + g * XS + 2 * t), word_at(xtl + (g + 8) * XS + 2 * t),
                                word_at(xtl + g * XS + 2 * t + 8), word_at(xtl + (g + 8) * XS + 2 * t + 8)};
#pragma unroll
        for (int n = 0; n < 16; ++n) {
            const __nv_bfloat16* ch = dhh + (8 * n + g) * XS;
            const __nv_bfloat16* cl = dhl + (8 * n + g) * XS;
            const uint32_t bh0 = word_at(ch + 2 * t), bh1 = word_at(ch + 2 * t + 8);
            const uint32_t bl0 = word_at(cl + 2 * t), bl1 = word_at(cl + 2 * t + 8);
            mma_bf16_16816(gw1[n], th, bh0, bh1);
            mma_bf16_16816(gw1[n], th, bl0, bl1);
            mma_bf16_16816(gw1[n], tl, bh0, bh1);
        }
        __syncwarp();
    }
    if (!GRAD) return;
    // dw2 over the lanes that share columns (same t): fixed butterfly over g
#pragma unroll
    for (int n = 0; n < 16; ++n)
#pragma unroll
        for (int j = 0; j < 2; ++j)
            for (int o = 4; o < 32; o <<= 1) gw2[n][j] += __shfl_xor_sync(0xFFFFFFFFu, gw2[n][j], o);
    for (int o = 4; o < 32; o <<= 1) {
        gb2 += __shfl_xor_sync(0xFFFFFFFFu, gb2, o);
        loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
    }
    // block reduction in shared memory, warps in index order (deterministic)
    float* sg = reinterpret_cast<float*>(wbase);  // reuses the tiles: MLP_NPARAM floats
    __shared__ double sl;
    __syncthreads();
    for (int k = 0; k < TC_WARPS; ++k) {
        if (wid == k) {
            const bool first = k == 0;
#pragma unroll
            for (int n = 0; n < 16; ++n)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int col = 8 * n + 2 * t + j;
                    // dW1 rows g and g + 8 (< 12), db1 in row 12
                    const int r0 = g, r1 = g + 8;
                    const float v0 = gw1[n][j], v1 = gw1[n][2 + j];
                    if (r0 < MLP_F) sg[r0 * MLP_H + col] = first ? v0 : sg[r0 * MLP_H + col] + v0;
                    if (r1 < MLP_F) sg[r1 * MLP_H + col] = first ? v1 : sg[r1 * MLP_H + col] + v1;
                    if (r1 == MLP_F) sg[MLP_F * MLP_H + col] = first ? v1 : sg[MLP_F * MLP_H + col] + v1;
                    if (g == 0)
                        sg[MLP_F * MLP_H + MLP_H + col] =
                            first ? gw2[n][j] : sg[MLP_F * MLP_H + MLP_H + col] + gw2[n][j];
                }
            if (lane == 0) {
                sg[MLP_NPARAM - 1] = first ? gb2 : sg[MLP_NPARAM - 1] + gb2;
                sl = first ? loss : sl + loss;
            }
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) partial_grad[(uint64_t)blockIdx.x * MLP_NPARAM + i] = sg[i];
    if (threadIdx.x == 0) partial_loss[blockIdx.x] = sl;
}

size_t tc_smem_bytes() {
    return sizeof(TcSmem) + (size_t)TC_WARPS * TC_WARP_TILE * sizeof(__nv_bfloat16);
}

template <bool GRAD>
void launch_mlp_tc(Ctx& c, const float* feat, const uint8_t* label, uint64_t M, const __nv_bfloat16* wb, float* out_p,
                   float* partial_grad, double* partial_loss) {
    const size_t sm = tc_smem_bytes();
    SC_CUDA(cudaFuncSetAttribute(k_mlp_tc<GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_mlp_tc<GRAD><<<MLP_BLOCKS, TC_THREADS, sm, c.stream>>>(feat, label, M, wb, out_p, partial_grad, partial_loss);
    SC_LAUNCH_CHECK();
    c.launches++;
}

__global__ void k_grad_reduce(const float* __restrict__ partial, const double* __restrict__ partial_loss, int nblocks,
                              uint64_t M, float* grad, double* loss) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < nblocks; ++b) acc += partial[(uint64_t)b * MLP_NPARAM + i];
        grad[i] = M ? (float)(acc / (double)M) : 0.0f;  // mean over edges
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double acc = 0.0;
        for (int b = 0; b < nblocks; ++b) acc += partial_loss[b];
        *loss = M ? acc / (double)M : 0.0;
    }
}

__global__ void k_adam(float* master, float* m, float* v, const float* __restrict__ grad, float lr, float b1, float b2,
                       float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
        const float g = grad[i];
        m[i] = b1 * m[i] + (1.0f - b1) * g;
        v[i] = b2 * v[i] + (1.0f - b2) * g * g;
        master[i] -= lr * (m[i] / bc1) / (sqrtf(v[i] / bc2) + eps);
    }
}

__global__ void k_edge_labels(const uint32_t* __restrict__ ei, const uint32_t* __restrict__ ej, uint64_t M,
                              const uint32_t* __restrict__ memb, uint8_t* label) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < M;
         e += (uint64_t)gridDim.x * blockDim.x)
        label[e] = memb[ei[e]] == memb[ej[e]];
}

// Connected components of the confident edges: min-label hooking + pointer jumping.
// Per node: undirected non-loop edges and confident ones among them.
__global__ void k_conf_degree(const uint32_t* __restrict__ ei, const uint32_t* __restrict__ ej,
                              const float* __restrict__ p, uint64_t M, float thr, uint32_t* deg, uint32_t* conf) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < M;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = ei[e], b = ej[e];
        atomicAdd(deg + a, 1u);
        atomicAdd(deg + b, 1u);
        if (p[e] > thr) {
            atomicAdd(conf + a, 1u);
            atomicAdd(conf + b, 1u);
        }
    }
}

// Edge mask: confident and both endpoints core (conf >= phi * deg).
__global__ void k_core_mask(const uint32_t* __restrict__ ei, const uint32_t* __restrict__ ej,
                            const float* __restrict__ p, uint64_t M, float thr, double phi,
                            const uint32_t* __restrict__ deg, const uint32_t* __restrict__ conf, uint8_t* keep) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < M;
         e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = ei[e], b = ej[e];
        keep[e] = p[e] > thr && (double)conf[a] >= phi * (double)deg[a] && (double)conf[b] >= phi * (double)deg[b];
    }
}

__global__ void k_cc_hook(const uint32_t* __restrict__ ei, const uint32_t* __restrict__ ej,
                          const uint8_t* __restrict__ keep, uint64_t M, uint32_t* lab, int* changed) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < M;
         e += (uint64_t)gridDim.x * blockDim.x) {
        if (!keep[e]) continue;
        const uint32_t a = lab[ei[e]], b = lab[ej[e]];
        if (a == b) continue;
        const uint32_t lo = min(a, b), hi = max(a, b);
        if (atomicMin(lab + hi, lo) > lo) *changed = 1;
    }
}

__global__ void k_cc_jump(uint32_t* lab, uint64_t n, int* changed) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t l = lab[v];
        const uint32_t ll = lab[l];
        if (ll != l) {
            lab[v] = ll;
            *changed = 1;
        }
    }
}

__global__ void k_iota_u32(uint32_t* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (uint32_t)i;
}

__global__ void k_init_params(float* p, uint64_t seed) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
        const double u = (double)(hash3(seed, 0x31415ull, (uint64_t)i) >> 11) * 0x1.0p-53;  // [0, 1)
        float x = 0.0f;
        if (i < MLP_F * MLP_H) x = (float)((2.0 * u - 1.0) * sqrt(6.0 / (MLP_F + MLP_H)));
        else if (i >= MLP_F * MLP_H + MLP_H && i < MLP_F * MLP_H + 2 * MLP_H)
            x = (float)((2.0 * u - 1.0) * sqrt(6.0 / (MLP_H + 1)));
        p[i] = x;
    }
}

struct EdgeSet {
    uint64_t M = 0;
    DBuf<float> feat;
    const uint32_t* ei = nullptr;  // the graph's edge list (kept with the graph)
    const uint32_t* ej = nullptr;
};

template <class T>
T* graph_pool_alloc(Ctx& c, uint64_t count) {
    T* p = nullptr;
    if (!count) return p;
    const cudaError_t e = cudaMallocFromPoolAsync((void**)&p, count * sizeof(T), user_graph_pool(c.device), c.stream);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        fail(SC_E_OUT_OF_MEMORY, "device allocation of %llu bytes failed", (unsigned long long)(count * sizeof(T)));
    }
    if (e != cudaSuccess) throw_cuda(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
    return p;
}

// Frees the graph's cached edge features (caller holds edge_mu).
void drop_edge_cache(const DevGraph& g) {
    if (!g.edge_sf && !g.edge_i && !g.edge_j && !g.edge_e) {
        g.edge_ready = false;
        return;
    }
    SC_CUDA(cudaDeviceSynchronize());  // any context's stream may still read them
    for (void* p : {(void*)g.edge_sf, (void*)g.edge_i, (void*)g.edge_j, (void*)g.edge_e})
        if (p) SC_CUDA(cudaFreeAsync(p, (cudaStream_t)0));
    SC_CUDA(cudaStreamSynchronize((cudaStream_t)0));
    g.edge_sf = nullptr;
    g.edge_i = g.edge_j = nullptr;
    g.edge_e = nullptr;
    g.edge_m = 0;
    g.edge_ready = false;
}

// The graph's structural edge features, computed once per graph (and again
// after a new embedding): they depend on neither the resolution nor a context.
void build_structural(Ctx& c, const DevGraph& g) {
    std::lock_guard<std::mutex> lock(g.edge_mu);
    if (g.edge_ready) return;
    drop_edge_cache(g);  // the leftovers of a build that failed
    static const bool trace = std::getenv("SC_TRACE") != nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    // edge positions: upper entries per row, exclusive sum
    DBuf<uint64_t> cnt(c, g.n + 1), base(c, g.n + 1);
    k_upper_counts<<<grid_for(g.n + 1, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.n, cnt.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    exclusive_sum(c, cnt.get(), base.get(), g.n + 1);
    const uint64_t M = to_host(c, base.get() + g.n);
    g.edge_sf = graph_pool_alloc<float>(c, M * EDGE_SF);
    g.edge_i = graph_pool_alloc<uint32_t>(c, M);
    g.edge_j = graph_pool_alloc<uint32_t>(c, M);
    g.edge_e = graph_pool_alloc<uint64_t>(c, 2 * M);
    g.edge_m = M;
    if (M) {
        DBuf<float> scale;
        if (g.emb) {
            scale.alloc(c, g.n);
            k_emb_scale<<<grid_for(g.n, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.n, g.emb, scale.get());
            SC_LAUNCH_CHECK();
            c.launches++;
        }
        DBuf<float2> nlog(c, g.n);
        k_node_logs<<<grid_for(g.n, TB), TB, 0, c.stream>>>(g.ptr, g.strength, g.n, nlog.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        const FeatArgs A{g.ptr,  g.nbr,       g.w,       g.strength, nlog.get(), 2.0 * g.total_weight, g.emb,
                         scale.get(), base.get(), g.edge_sf, g.edge_i,   g.edge_j,   g.edge_e};
        k_edge_rows<<<grid_for(g.n * 32, TB), TB, 0, c.stream>>>(A, g.n);
        SC_LAUNCH_CHECK();
        c.launches++;
        if (g.max_degree > (uint32_t)ROW_STAGE) {
            // rows a warp cannot stage: a block each
            DBuf<uint32_t> big(c, g.n);
            DBuf<unsigned> nbig(c, 1);
            zero(c, nbig.get(), 1);
            k_big_rows<<<grid_for(g.n, TB), TB, 0, c.stream>>>(g.ptr, g.n, ROW_STAGE, big.get(), nbig.get());
            SC_LAUNCH_CHECK();
            c.launches++;
            const unsigned nb = to_host(c, nbig.get());
            if (nb) {
                const size_t sm = (size_t)BIG_STAGE * (sizeof(uint32_t) + sizeof(float));
                SC_CUDA(cudaFuncSetAttribute(k_edge_big_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_edge_big_rows<<<std::min<unsigned>(nb, 148u * 8u), TB, sm, c.stream>>>(A, big.get(), nb);
                SC_LAUNCH_CHECK();
                c.launches++;
            }
        }
    }
    sync(c);
    g.edge_ready = true;
    if (trace)
        std::fprintf(stderr, "[sc] structural edge features M=%llu: %.2f ms (once per graph)\n", (unsigned long long)M,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}

// The MLP input of every undirected edge of g at gamma with the context
// partitions (nullable): the graph's structural values plus the
// resolution and context features.
void build_edges(Ctx& c, const DevGraph& g, double gamma, const uint32_t* coarse, const uint32_t* fine,
                 EdgeSet& es) {
    build_structural(c, g);
    const uint64_t M = g.edge_m;
    es.M = M;
    es.ei = g.edge_i;
    es.ej = g.edge_j;
    es.feat.alloc(c, M * MLP_F);
    if (!M) return;
    DBuf<float> share_c, share_f;
    DBuf<uint32_t> big;
    unsigned nb = 0;
    if ((coarse || fine) && g.max_degree > 32u * 32u) {
        // rows past 32 chunks: a block each
        big.alloc(c, g.n);
        DBuf<unsigned> nbig(c, 1);
        zero(c, nbig.get(), 1);
        k_big_rows<<<grid_for(g.n, TB), TB, 0, c.stream>>>(g.ptr, g.n, 32 * 32, big.get(), nbig.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        nb = to_host(c, nbig.get());
    }
    for (int t = 0; t < 2; ++t) {
        const uint32_t* lab = t == 0 ? coarse : fine;
        DBuf<float>& sh = t == 0 ? share_c : share_f;
        if (!lab) continue;
        sh.alloc(c, g.E);
        k_label_share<<<grid_for(g.n * 32, TB), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, lab, g.strength, g.n,
                                                                   sh.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        if (nb) {
            k_label_share_big<<<std::min<unsigned>(nb, 148u * 8u), TB, 0, c.stream>>>(g.ptr, g.nbr, g.w, lab,
                                                                                    g.strength, big.get(), nb,
                                                                                    sh.get());
            SC_LAUNCH_CHECK();
            c.launches++;
        }
    }
    k_assemble<<<grid_for(M, TB), TB, 0, c.stream>>>(M, g.edge_sf, g.edge_i, g.edge_j, g.edge_e, (float)log(gamma),
                                                     gamma, coarse, fine, share_c.get(), share_f.get(), es.feat.get());
    SC_LAUNCH_CHECK();
    c.launches++;
}

// Standardise es's features with the model's scaler, fitting it first if the
// model has none (and `fit` allows it).
void scale_edges(Ctx& c, Mlp& m, EdgeSet& es, bool fit) {
    if (!m.has_norm) {
        if (!fit) fail(SC_E_INVALID_ARGUMENT, "the model has no feature scaler yet: train it or set one first");
        const int nb = 148;
        DBuf<double> partial(c, (uint64_t)nb * 2 * MLP_F);
        k_feat_partials<<<nb, TB, 0, c.stream>>>(es.feat.get(), es.M, partial.get());
        k_feat_finalize<<<1, 32, 0, c.stream>>>(partial.get(), nb, es.M, m.norm);
        SC_LAUNCH_CHECK();
        sync(c);
        m.has_norm = true;
        c.launches += 2;
    }
    if (es.M) {
        k_normalize<<<grid_for(es.M * MLP_F, TB), TB, 0, c.stream>>>(es.feat.get(), es.M, m.norm);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
}

// Mean BCE loss and its gradient at the current BF16 weights.
double grad_at(Ctx& c, const Mlp& m, const EdgeSet& es, const uint8_t* labels, float* d_grad) {
    DBuf<__nv_bfloat16> wb(c, MLP_NPARAM);
    k_to_bf16<<<4, 256, 0, c.stream>>>(m.master, wb.get());
    DBuf<float> partial(c, (uint64_t)MLP_BLOCKS * MLP_NPARAM);
    DBuf<double> partial_loss(c, MLP_BLOCKS), loss(c, 1);
    launch_mlp_tc<true>(c, es.feat.get(), labels, es.M, wb.get(), nullptr, partial.get(), partial_loss.get());
    k_grad_reduce<<<8, 256, 0, c.stream>>>(partial.get(), partial_loss.get(), MLP_BLOCKS, es.M, d_grad, loss.get());
    SC_LAUNCH_CHECK();
    c.launches += 3;
    return to_host(c, loss.get());
}

// y_i[r] = sum_a X[i][a] P[a][r], P the d x EMB_R sign matrix (rows of X in
// chunks: the host embedding is uploaded piecewise).
__global__ void k_emb_project(const float* __restrict__ X, uint64_t rows, uint64_t d, const float* __restrict__ P,
                              float* y) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < rows * EMB_R;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = t / EMB_R;
        const int r = (int)(t % EMB_R);
        float acc = 0.0f;
        for (uint64_t a = 0; a < d; ++a) acc = __fmaf_rn(X[i * d + a], P[a * EMB_R + r], acc);
        y[t] = acc;
    }
}

}  // namespace

// P[a][r] = +-1/sqrt(EMB_R), the sign from the top bit of splitmix(a EMB_R + r):
// a fixed random projection (Johnson-Lindenstrauss with signs), the same for
// every graph and embedding width.
void graph_set_embedding(Ctx& c, DevGraph& g, const float* X, uint64_t d) {
    if (d == 0) fail(SC_E_INVALID_ARGUMENT, "embedding width must be positive");
    if (X == nullptr && g.n) fail(SC_E_INVALID_ARGUMENT, "embedding is NULL");
    std::vector<float> P(d * EMB_R);
    for (uint64_t a = 0; a < d; ++a)
        for (int r = 0; r < EMB_R; ++r) P[a * EMB_R + r] = (splitmix(a * EMB_R + r) >> 63) ? -0.25f : 0.25f;
    DBuf<float> dP(c, P.size());
    SC_CUDA(cudaMemcpyAsync(dP.get(), P.data(), P.size() * sizeof(float), cudaMemcpyHostToDevice, c.stream));
    float* y = nullptr;
    if (g.n) {
        cudaError_t e = cudaMallocFromPoolAsync((void**)&y, g.n * EMB_R * sizeof(float), user_graph_pool(c.device),
                                                c.stream);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            fail(SC_E_OUT_OF_MEMORY, "device allocation of the projected embedding failed");
        }
        if (e != cudaSuccess) throw_cuda(e, "cudaMallocFromPoolAsync", __FILE__, __LINE__);
    }
    const uint64_t chunk = std::max<uint64_t>(1, (64ull << 20) / (d * sizeof(float)));
    DBuf<float> xb(c, std::min(chunk, std::max<uint64_t>(g.n, 1)) * d);
    for (uint64_t r0 = 0; r0 < g.n; r0 += chunk) {
        const uint64_t rows = std::min(chunk, g.n - r0);
        SC_CUDA(cudaMemcpyAsync(xb.get(), X + r0 * d, rows * d * sizeof(float), cudaMemcpyHostToDevice, c.stream));
        k_emb_project<<<grid_for(rows * EMB_R, TB), TB, 0, c.stream>>>(xb.get(), rows, d, dP.get(),
                                                                      y + r0 * EMB_R);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    sync(c);
    std::lock_guard<std::mutex> lock(g.edge_mu);
    drop_edge_cache(g);  // the structural features read the embedding
    if (g.emb) {
        SC_CUDA(cudaDeviceSynchronize());
        SC_CUDA(cudaFreeAsync(g.emb, c.stream));
        sync(c);
    }
    g.emb = y;
}

Mlp* mlp_create(Ctx& c, uint64_t seed) {
    std::unique_ptr<Mlp> m(new Mlp());
    m->device = c.device;
    struct Guard {
        Mlp* m;
        ~Guard() { if (m) mlp_destroy(m); }
    } guard{m.get()};
    SC_CUDA(cudaMalloc(&m->master, MLP_NPARAM * sizeof(float)));
    SC_CUDA(cudaMalloc(&m->m, MLP_NPARAM * sizeof(float)));
    SC_CUDA(cudaMalloc(&m->v, MLP_NPARAM * sizeof(float)));
    SC_CUDA(cudaMalloc(&m->norm, 2 * MLP_F * sizeof(float)));
    k_init_params<<<4, 256, 0, c.stream>>>(m->master, seed);
    SC_LAUNCH_CHECK();
    zero(c, m->m, MLP_NPARAM);
    zero(c, m->v, MLP_NPARAM);
    zero(c, m->norm, 2 * MLP_F);
    sync(c);
    guard.m = nullptr;
    return m.release();
}

void mlp_destroy(Mlp* m) {
    if (!m) return;
    cudaFree(m->master);
    cudaFree(m->m);
    cudaFree(m->v);
    cudaFree(m->norm);
    delete m;
}

uint32_t mlp_param_count() { return MLP_NPARAM; }

uint32_t mlp_feature_count() { return MLP_F; }

bool mlp_get(Ctx& c, const Mlp& m, float* params, float* scaler) {
    if (params) d2h(c, params, m.master, MLP_NPARAM);
    if (scaler) d2h(c, scaler, m.norm, 2 * MLP_F);
    sync(c);
    return m.has_norm;
}

// New parameters (and optionally scaler); resets the Adam state.
void mlp_set(Ctx& c, Mlp& m, const float* params, const float* scaler) {
    if (params) {
        h2d(c, m.master, params, MLP_NPARAM);
        zero(c, m.m, MLP_NPARAM);
        zero(c, m.v, MLP_NPARAM);
        m.step = 0;
    }
    if (scaler) {
        h2d(c, m.norm, scaler, 2 * MLP_F);
        m.has_norm = true;
    }
    sync(c);
}

// Edge features of g at resolution gamma as the model sees them (standardised
// by its scaler, which this fits if the model has none), sorted by (i, j).
void mlp_features(Ctx& c, Mlp& m, const DevGraph& g, double gamma, const uint32_t* coarse, const uint32_t* fine,
                  float* feat_host, uint32_t* ei_host, uint32_t* ej_host, uint64_t cap, uint64_t* M_out) {
    EdgeSet es;
    build_edges(c, g, gamma, coarse, fine, es);
    *M_out = es.M;
    if (es.M > cap)
        fail(SC_E_INVALID_ARGUMENT, "capacity %llu is below the %llu undirected edges", (unsigned long long)cap,
             (unsigned long long)es.M);
    scale_edges(c, m, es, true);
    if (feat_host) d2h(c, feat_host, es.feat.get(), es.M * MLP_F);
    if (ei_host) d2h(c, ei_host, es.ei, es.M);
    if (ej_host) d2h(c, ej_host, es.ej, es.M);
    sync(c);
}

// `epochs` full-batch Adam steps on (g, membership) at gamma; returns the mean
// loss at the weights before the last step. epochs == 0 only evaluates the loss
// and gradient. grad_out_host (nullable) receives the last gradient.
double mlp_train(Ctx& c, Mlp& m, const DevGraph& g, const uint32_t* d_memb, double gamma, const uint32_t* coarse,
                 const uint32_t* fine, uint32_t epochs, double lr, float* grad_out_host) {
    EdgeSet es;
    build_edges(c, g, gamma, coarse, fine, es);
    scale_edges(c, m, es, true);
    DBuf<uint8_t> lab(c, es.M);
    if (es.M) {
        k_edge_labels<<<grid_for(es.M, TB), TB, 0, c.stream>>>(es.ei, es.ej, es.M, d_memb, lab.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    DBuf<float> grad(c, MLP_NPARAM);
    double loss = grad_at(c, m, es, lab.get(), grad.get());
    const float b1 = 0.9f, b2 = 0.999f;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        if (ep) loss = grad_at(c, m, es, lab.get(), grad.get());
        m.step++;
        const float bc1 = 1.0f - powf(b1, (float)m.step), bc2 = 1.0f - powf(b2, (float)m.step);
        k_adam<<<4, 256, 0, c.stream>>>(m.master, m.m, m.v, grad.get(), (float)lr, b1, b2, 1e-8f, bc1, bc2);
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    if (grad_out_host) {
        d2h(c, grad_out_host, grad.get(), MLP_NPARAM);
        sync(c);
    }
    return loss;
}

// Proposal: components of the edges whose predicted probability exceeds thr.
uint64_t mlp_propose(Ctx& c, Mlp& m, const DevGraph& g, double gamma, const uint32_t* coarse, const uint32_t* fine,
                     double thr, double core_fraction, uint32_t* d_labels, float* prob_host, uint64_t prob_cap) {
    // SC_TRACE: device time of the stages (events on the context's stream)
    static const bool trace = std::getenv("SC_TRACE") != nullptr;
    std::vector<cudaEvent_t> ev;
    auto mark = [&]() {
        if (!trace) return;
        cudaEvent_t e;
        SC_CUDA(cudaEventCreate(&e));
        SC_CUDA(cudaEventRecord(e, c.stream));
        ev.push_back(e);
    };
    mark();
    EdgeSet es;
    build_edges(c, g, gamma, coarse, fine, es);
    mark();
    scale_edges(c, m, es, false);
    DBuf<__nv_bfloat16> wb(c, MLP_NPARAM);
    k_to_bf16<<<4, 256, 0, c.stream>>>(m.master, wb.get());
    DBuf<float> p(c, es.M);
    if (es.M)
        launch_mlp_tc<false>(c, es.feat.get(), nullptr, es.M, wb.get(), p.get(), nullptr, nullptr);
    SC_LAUNCH_CHECK();
    mark();
    if (prob_host) {
        if (es.M > prob_cap) fail(SC_E_INVALID_ARGUMENT, "probability capacity too small");
        d2h(c, prob_host, p.get(), es.M);
    }
    const uint64_t n = g.n;
    DBuf<uint32_t> deg(c, n), conf(c, n);
    DBuf<uint8_t> keep(c, es.M);
    zero(c, deg.get(), n);
    zero(c, conf.get(), n);
    if (es.M) {
        k_conf_degree<<<grid_for(es.M, TB), TB, 0, c.stream>>>(es.ei, es.ej, p.get(), es.M, (float)thr,
                                                               deg.get(), conf.get());
        k_core_mask<<<grid_for(es.M, TB), TB, 0, c.stream>>>(es.ei, es.ej, p.get(), es.M, (float)thr,
                                                             core_fraction, deg.get(), conf.get(), keep.get());
        SC_LAUNCH_CHECK();
        c.launches += 3;
    }
    k_iota_u32<<<grid_for(n, TB), TB, 0, c.stream>>>(d_labels, n);
    DBuf<int> changed(c, 1);
    bool done = false;
    // Every round either hooks a root under a smaller label or shortens a path,
    // and labels only decrease, so the loop ends; the cap turns a bug into an error.
    for (int round = 0; round < 4096 && !done; ++round) {
        zero(c, changed.get(), 1);
        if (es.M)
            k_cc_hook<<<grid_for(es.M, TB), TB, 0, c.stream>>>(es.ei, es.ej, keep.get(), es.M, d_labels,
                                                               changed.get());
        for (int j = 0; j < 4; ++j) k_cc_jump<<<grid_for(n, TB), TB, 0, c.stream>>>(d_labels, n, changed.get());
        SC_LAUNCH_CHECK();
        c.launches += 5;
        done = !to_host(c, changed.get());
    }
    if (!done) fail(SC_E_INTERNAL, "proposal components did not converge");
    mark();
    DBuf<uint32_t> compact(c, n);
    const uint32_t K = renumber_ids(c, d_labels, n, n, compact.get());
    d2d(c, d_labels, compact.get(), n);
    mark();
    sync(c);
    if (trace) {
        float t[4] = {};
        for (int k = 0; k < 4; ++k) SC_CUDA(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
        std::fprintf(stderr, "[sc] mlp propose M=%llu: features %.2f ms, scale + infer %.2f ms, components %.2f ms, "
                     "renumber %.2f ms\n", (unsigned long long)es.M, t[0], t[1], t[2], t[3]);
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    return K;
}

}  // namespace sc
