// sc_knn.cu — Gaussian kNN graph builder (src/neighborhood/mod.rs) on sm_100a.
//
// 1. k_knn_prep       X (f32) -> A = [-2x, 1, 1, 0..] and B = [x, |x|^2 hi, |x|^2 lo, 0..]
//                     in BF16, KA = 32 (D <= 30) or 64 (D <= 62) columns.
//                     A . B = |c|^2 - 2 q.c = |q - c|^2 - |q|^2: the row-constant
//                     |q|^2 does not change a row's ranking, so the contraction
//                     yields ranking scores directly.
//    k_knn_prep_f8    the FP8 (e4m3) operands, 64 one-byte columns (D <= 61): B =
//                     [x / S, three e4m3 terms of |x|^2 / S_n, 0..] with one scale
//                     for the point set, A = f_q [-2 x S / S_n, 1, 1, 1, 0..] with a
//                     power-of-two scale f_q per query row. A . B = (f_q / S_n) (|c|^2
//                     - 2 q.c): a positive factor per row, so the ranking is kept
//                     (a per-point scale on B would rescale columns and break it).
//                     64-byte rows: the tile geometry, swizzle and descriptors of the
//                     BF16 KA = 32 path; each K step is one kind::f8f6f4 MMA of K = 32.
// 2. k_knn_tc         persistent tcgen05 kernel, one CTA per SM. A group of 256
//                     queries (two M = 128 tiles) stays in shared memory; every
//                     128-candidate tile of B streams in by TMA (no multicast)
//                     through a STAGES-deep ring; one thread issues
//                     tcgen05.mma (M=128, N=128, K=16, BF16 -> FP32) into a
//                     double-buffered TMEM accumulator (2 x 2 x 128 columns);
//                     8 epilogue warps read it with tcgen05.ld and keep, per
//                     query, the R best scores in shared memory (a candidate is
//                     rejected with one compare against the row's worst kept).
// 3. k_knn_rerank     exact FP32 distances sum (q_d - c_d)^2 of the R candidates
//                     (no norm expansion, so no cancellation), sorted by
//                     (distance, self first, index); the first k+1 are kept.
// 4. k_knn_sigma / k_knn_pairs / CSR: sigma (median of the positive distances,
//                     neighborhood/mod.rs:105-124, or the k-th distance), the
//                     Gaussian weight of :139-163, lower-id or union emission,
//                     sorted into a CSR that from_csr_parts then finishes.
//
// Every wait on an mbarrier is bounded: on timeout the CTA records
// DEV_TIMEOUT, drains the copies it issued (again bounded), frees its TMEM and
// returns; the host turns the status into SC_E_TIMEOUT.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cudaTypedefs.h>

#include "sc_prims.cuh"

namespace sc {

namespace {

constexpr int QT = 2;              // query tiles of 128 per CTA group
constexpr int TILE = 128;          // rows per tile (M and N of the MMA)
constexpr int HALVES = 2;          // each accumulator row is read as two 64-column halves
constexpr int RCAND = 32;          // candidates kept per (query, half) before the exact re-rank
constexpr int RTOTAL = RCAND * HALVES;  // candidates per query handed to the re-rank
constexpr int NUM_EPI_WARPS = 4 * QT * HALVES;  // a full set of 4 TMEM lane quarters per (tile, half)
constexpr int KNN_THREADS = 32 * (2 + NUM_EPI_WARPS);
template <int KA>
constexpr int stages_for() { return KA == 32 ? 6 : 3; }  // B ring depth within 227 KB
constexpr uint32_t WAIT_LIMIT = DEFAULT_WAIT_LIMIT;  // drain waits: copies / MMAs already issued
constexpr uint32_t TMEM_COLS = 512;

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait for the phase with the given parity to complete: at most
// `limit` try_wait attempts, false when they ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = WAIT_LIMIT) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, swizzled rows of KA * 2 bytes:
// start >> 4 at [0,14), stride between 8-row groups >> 4 at [32,46),
// version 1 at [46,48), layout at [61,64) (4 = 64B swizzle, 2 = 128B swizzle).
template <int KA>
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    constexpr uint64_t row_bytes = KA * 2;
    constexpr uint64_t sbo = 8 * row_bytes;
    constexpr uint64_t layout = (KA == 32) ? 4ull : 2ull;
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= 1ull << 46;
    d |= layout << 61;
    return d;
}

// Instruction descriptor, kind::f16: D f32, A/B bf16, both K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16_128x128() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TILE >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Instruction descriptor, kind::f8f6f4: D f32, A/B e4m3 (format 0), both K-major, N = 128, M = 128.
__host__ __device__ constexpr uint32_t idesc_e4m3_128x128() {
    return (1u << 4) | ((uint32_t)(TILE >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}

__device__ __forceinline__ void mma_e4m3(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
          "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
          "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Insert (v, idx) into a query's candidate slots over its current worst slot and
// return the new worst (value, slot). Kept out of line: it is the rare path,
// and inlining it into the unrolled filter loop overflows the instruction cache.
struct Worst {
    float thr;
    int slot;
};

// A chunk whose candidates fall in at most this many of a warp's 32 rows is
// processed by the whole warp, row by row; denser chunks by each lane alone.
constexpr int COOP_ROWS = 8;

template <int R>
__device__ __noinline__ Worst cand_insert(float* cs, uint32_t* ci, int qrow, int slot, float v, uint32_t idx) {
    constexpr int S = QT * HALVES * TILE;
    cs[slot * S + qrow] = v;
    ci[slot * S + qrow] = idx;
    Worst w{-INFINITY, 0};
    for (int s = 0; s < R; ++s) {
        const float x = cs[s * S + qrow];
        if (x > w.thr) {
            w.thr = x;
            w.slot = s;
        }
    }
    return w;
}

// ------------------------------------------------------------ prep
template <int KA>
__global__ void k_knn_prep(const float* __restrict__ X, uint64_t n, uint32_t d, __nv_bfloat16* A,
                           __nv_bfloat16* B) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float* x = X + i * d;
        float nrm = 0.0f;
        for (uint32_t j = 0; j < d; ++j) nrm = __fmaf_rn(x[j], x[j], nrm);
        __nv_bfloat16* a = A + i * KA;
        __nv_bfloat16* b = B + i * KA;
        for (uint32_t j = 0; j < d; ++j) {
            __nv_bfloat16 xb = __float2bfloat16_rn(x[j]);
            a[j] = __float2bfloat16_rn(-2.0f * __bfloat162float(xb));
            b[j] = xb;
        }
        __nv_bfloat16 hi = __float2bfloat16_rn(nrm);
        __nv_bfloat16 lo = __float2bfloat16_rn(nrm - __bfloat162float(hi));
        a[d] = __float2bfloat16_rn(1.0f);
        a[d + 1] = __float2bfloat16_rn(1.0f);
        b[d] = hi;
        b[d + 1] = lo;
        for (uint32_t j = d + 2; j < (uint32_t)KA; ++j) {
            a[j] = __float2bfloat16_rn(0.0f);
            b[j] = __float2bfloat16_rn(0.0f);
        }
    }
}

// max |x_ik| and max |x_i|^2 over the point set (non-negative floats order like
// their bit patterns, so an integer atomicMax finds them).
__global__ void k_knn_scales(const float* __restrict__ X, uint64_t n, uint32_t d, unsigned* maxabs,
                             unsigned* maxnorm) {
    float ma = 0.0f, mn = 0.0f;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float* x = X + i * d;
        float nrm = 0.0f;
        for (uint32_t j = 0; j < d; ++j) {
            ma = fmaxf(ma, fabsf(x[j]));
            nrm = __fmaf_rn(x[j], x[j], nrm);
        }
        mn = fmaxf(mn, nrm);
    }
    for (int o = 16; o; o >>= 1) {
        ma = fmaxf(ma, __shfl_xor_sync(0xFFFFFFFFu, ma, o));
        mn = fmaxf(mn, __shfl_xor_sync(0xFFFFFFFFu, mn, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(maxabs, __float_as_uint(ma));
        atomicMax(maxnorm, __float_as_uint(mn));
    }
}

__device__ __forceinline__ uint8_t to_e4m3(float x) { return (uint8_t)__nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3); }

__device__ __forceinline__ float from_e4m3(uint8_t b) {
    __nv_fp8_e4m3 v;
    v.__x = (__nv_fp8_storage_t)b;
    return (float)v;
}

// FP8 operands (64 one-byte columns, D <= 61): see the file comment.
__global__ void k_knn_prep_f8(const float* __restrict__ X, uint64_t n, uint32_t d, const unsigned* __restrict__ maxabs,
                              const unsigned* __restrict__ maxnorm, uint8_t* A, uint8_t* B) {
    constexpr uint32_t W = 64;
    const float ma = __uint_as_float(*maxabs), mn = __uint_as_float(*maxnorm);
    const float S = ma > 0.0f ? ma / 256.0f : 1.0f;
    const float Sn = mn > 0.0f ? mn / 256.0f : 1.0f;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float* x = X + i * d;
        uint8_t* a = A + i * W;
        uint8_t* b = B + i * W;
        float nrm = 0.0f, m = 0.0f;
        for (uint32_t j = 0; j < d; ++j) {
            nrm = __fmaf_rn(x[j], x[j], nrm);
            m = fmaxf(m, fabsf(2.0f * x[j] * S / Sn));
        }
        // power-of-two row factor f with m f <= 448, f in [2^-9, 2^8] (both e4m3-exact)
        int e = 8;
        if (m > 0.0f) {
            e = (int)floorf(log2f(448.0f / m));
            e = e < -9 ? -9 : (e > 8 ? 8 : e);
        }
        const float f = ldexpf(1.0f, e);
        for (uint32_t j = 0; j < d; ++j) {
            a[j] = to_e4m3(-2.0f * x[j] * S / Sn * f);
            b[j] = to_e4m3(x[j] / S);
        }
        // |x|^2 / S_n as three e4m3 terms (each takes the remainder of the last)
        float v = nrm / Sn;
        for (uint32_t t = 0; t < 3; ++t) {
            const uint8_t q = to_e4m3(v);
            b[d + t] = q;
            a[d + t] = to_e4m3(f);
            v -= from_e4m3(q);
        }
        for (uint32_t j = d + 3; j < W; ++j) {
            a[j] = 0;
            b[j] = 0;
        }
    }
}

// ------------------------------------------------------------ tensor-core candidate search
template <int KA, int R = RCAND>
struct KnnSmem {
    static constexpr int STAGES = stages_for<KA>();
    static constexpr uint32_t TILE_BYTES = TILE * KA * 2;
    static constexpr uint32_t SLOTS = QT * HALVES * TILE;                       // (tile, half, row) owners
    static constexpr uint32_t A_OFF = 0;
    static constexpr uint32_t B_OFF = A_OFF + QT * TILE_BYTES;
    static constexpr uint32_t C_OFF = B_OFF + STAGES * TILE_BYTES;               // candidate scores
    static constexpr uint32_t I_OFF = C_OFF + R * SLOTS * 4;                     // candidate ids
    static constexpr uint32_t BAR_OFF = I_OFF + R * SLOTS * 4;
    static constexpr uint32_t NBAR = 2 * STAGES + 4 + 2;
    static constexpr uint32_t MISC_OFF = BAR_OFF + NBAR * 8;
    static constexpr uint32_t ROW_OFF = MISC_OFF + 64;                       // one staged row chunk per epilogue warp
    static constexpr uint32_t BYTES = ROW_OFF + NUM_EPI_WARPS * 32 * 4 + 1024;  // + alignment slack
    static_assert(BYTES <= 227 * 1024, "shared memory of the kNN kernel exceeds 227 KB");
    static_assert(ROW_OFF % 16 == 0, "staged rows must be 16-byte aligned");
};

// The point tiles a query group scans, in order: every tile, or (a pruned
// search) the group's ranges of (first tile, tile count), which never overlap.
struct TileWalk {
    const uint2* r;
    uint32_t nr, ri, off, all;
    __device__ TileWalk(const uint32_t* rptr, const uint2* rngs, uint32_t g, uint32_t ntiles)
        : r(rptr ? rngs + rptr[g] : nullptr), nr(rptr ? rptr[g + 1] - rptr[g] : 0), ri(0), off(0), all(ntiles) {}
    __device__ uint32_t count() const {
        if (!r) return all;
        uint32_t c = 0;
        for (uint32_t i = 0; i < nr; ++i) c += r[i].y;
        return c;
    }
    __device__ uint32_t next() {
        if (!r) return off++;
        while (off >= r[ri].y) {
            ++ri;
            off = 0;
        }
        return r[ri].x + off++;
    }
};

// F8: the operands are e4m3 bytes with the row size of BF16 KA columns.
// rptr / rngs (nullable): the tile ranges of each query group (pruned search).
// qcap (nullable): per query, a score no kept candidate reaches (a proven
// bound of the pruned search's second pass); the rows start from it instead
// of +inf, so far points never enter the insertion path.
// R: candidates kept per (query, half), RCAND or fewer (a pass that only
// bounds the (k+1)-th distance); the slots past R are written empty.
template <int KA, bool F8, int R = RCAND>
__global__ void __launch_bounds__(KNN_THREADS, 1)
    k_knn_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, uint32_t n,
             uint32_t nq, float* __restrict__ cand_score, uint32_t* __restrict__ cand_idx, uint32_t* status,
             uint32_t lim, uint32_t hold_tiles, const uint32_t* __restrict__ rptr, const uint2* __restrict__ rngs,
             const float* __restrict__ qcap) {
    using L = KnnSmem<KA, R>;
    extern __shared__ __align__(1024) unsigned char raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
    unsigned char* sA = smem + L::A_OFF;
    unsigned char* sB = smem + L::B_OFF;
    float* cs = (float*)(smem + L::C_OFF);
    uint32_t* ci = (uint32_t*)(smem + L::I_OFF);
    uint64_t* bars = (uint64_t*)(smem + L::BAR_OFF);
    uint64_t* full = bars;                 // [L::STAGES] B tile landed
    uint64_t* empty = bars + L::STAGES;       // [L::STAGES] B tile consumed by the MMAs
    uint64_t* accfull = bars + 2 * L::STAGES;       // [2] accumulator ready
    uint64_t* accempty = bars + 2 * L::STAGES + 2;  // [2] accumulator drained
    uint64_t* afull = bars + 2 * L::STAGES + 4;     // query tiles landed
    uint64_t* aempty = bars + 2 * L::STAGES + 5;    // query tiles no longer read
    uint32_t* misc = (uint32_t*)(smem + L::MISC_OFF);
    volatile uint32_t* abort_flag = misc + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t ntiles = (n + TILE - 1) / TILE;          // point tiles (B)
    const uint32_t ngroups = (nq + QT * TILE - 1) / (QT * TILE);  // query tile groups (A)

    if (threadIdx.x == 0) {
        for (int s = 0; s < L::STAGES; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accfull + b, 1);
            mbar_init(accempty + b, NUM_EPI_WARPS);
        }
        mbar_init(afull, 1);
        mbar_init(aempty, 1);
        misc[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(misc)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = misc[0];

    if (warp == 0) {
        // ---------------- TMA producer
        if (lane == 0) {
            uint64_t it = 0;  // global B tile counter (all groups)
            uint32_t gi = 0;
            bool a_in_flight = false;
            for (uint32_t g = blockIdx.x; g < ngroups && !*abort_flag; g += gridDim.x, ++gi) {
                if (gi > 0 && !mbar_wait(aempty, (gi - 1) & 1, lim)) {
                    *abort_flag = 1;
                    break;
                }
                mbar_expect_tx(afull, QT * L::TILE_BYTES);
                a_in_flight = true;
                for (int q = 0; q < QT; ++q)
                    tma_load_2d(sA + q * L::TILE_BYTES, &tmA, afull, 0, (int)(g * QT * TILE + q * TILE));
                if (hold_tiles) {  // test hook: no point tile is ever issued
                    ++gi;
                    break;
                }
                TileWalk walk(rptr, rngs, g, ntiles);
                const uint32_t cnt = walk.count();
                for (uint32_t t = 0; t < cnt; ++t, ++it) {
                    const uint32_t tile = walk.next();
                    const uint32_t s = (uint32_t)(it % L::STAGES);
                    const uint64_t use = it / L::STAGES;
                    if (use > 0 && !mbar_wait(empty + s, (uint32_t)((use - 1) & 1), lim)) {
                        *abort_flag = 1;
                        break;
                    }
                    if (*abort_flag) break;
                    mbar_expect_tx(full + s, L::TILE_BYTES);
                    tma_load_2d(sB + s * L::TILE_BYTES, &tmB, full + s, 0, (int)(tile * TILE));
                }
            }
            // drain: the copies issued last (one per stage, and the query tiles)
            // must land before the CTA exits (waits with the default limit)
            if (*abort_flag || hold_tiles) {
                for (uint64_t x = it > L::STAGES ? it - L::STAGES : 0; x < it; ++x)
                    mbar_wait(full + (x % L::STAGES), (uint32_t)((x / L::STAGES) & 1));
                if (a_in_flight && gi > 0) mbar_wait(afull, (gi - 1) & 1);
            }
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = F8 ? idesc_e4m3_128x128() : idesc_bf16_128x128();
            uint64_t it = 0;
            uint32_t gi = 0;
            for (uint32_t g = blockIdx.x; g < ngroups && !*abort_flag; g += gridDim.x, ++gi) {
                if (!mbar_wait(afull, gi & 1, lim)) {
                    *abort_flag = 1;
                    break;
                }
                fence_after();
                const uint32_t cnt = TileWalk(rptr, rngs, g, ntiles).count();
                for (uint32_t t = 0; t < cnt; ++t, ++it) {
                    const uint32_t s = (uint32_t)(it % L::STAGES);
                    const uint32_t b = (uint32_t)(it & 1);
                    const uint64_t use_b = it >> 1;
                    if (!mbar_wait(full + s, (uint32_t)((it / L::STAGES) & 1), lim)) {
                        *abort_flag = 1;
                        break;
                    }
                    if (use_b > 0 && !mbar_wait(accempty + b, (uint32_t)((use_b - 1) & 1), lim)) {
                        *abort_flag = 1;
                        break;
                    }
                    fence_after();
                    const uint32_t bbase = smem_u32(sB + s * L::TILE_BYTES);
#pragma unroll
                    for (int q = 0; q < QT; ++q) {
                        const uint32_t abase = smem_u32(sA + q * L::TILE_BYTES);
                        const uint32_t d = tmem + b * (QT * TILE) + q * TILE;
#pragma unroll
                        for (int kk = 0; kk < KA / 16; ++kk) {  // 32 bytes of K per MMA
                            if constexpr (F8)
                                mma_e4m3(d, smem_desc<KA>(abase + kk * 32), smem_desc<KA>(bbase + kk * 32), idesc,
                                         kk > 0 ? 1u : 0u);
                            else
                                mma_bf16(d, smem_desc<KA>(abase + kk * 32), smem_desc<KA>(bbase + kk * 32), idesc,
                                         kk > 0 ? 1u : 0u);
                        }
                    }
                    mma_commit(empty + s);
                    mma_commit(accfull + b);
                }
                mma_commit(aempty);
            }
            // drain: MMAs complete in issue order, so once the last tile's
            // accumulator commit has arrived none is left writing TMEM or
            // arriving on this CTA's barriers (waits with the default limit)
            if (*abort_flag && it > 0) {
                const uint64_t x = it - 1;
                mbar_wait(accfull + (uint32_t)(x & 1), (uint32_t)((x >> 1) & 1));
            }
        }
    } else {
        // ---------------- epilogue: 16 warps; warp % 4 selects the TMEM lane quarter
        // (hardware rule), (warp - 2) / 4 the (query tile, column half) it reads
        const int ew = warp - 2;
        const int combo = ew >> 2;
        const int q = combo / HALVES;           // query tile
        const int h = combo % HALVES;           // column half
        const int lq = warp & 3;                // lane quarter
        const int row = lq * 32 + lane;         // row within the query tile
        const int owner = combo * TILE + row;   // candidate-buffer column
        constexpr int S = L::SLOTS;
        float* srow = (float*)(smem + L::ROW_OFF) + ew * 32;  // this warp's staged row chunk
        uint64_t it = 0;
        for (uint32_t g = blockIdx.x; g < ngroups && !*abort_flag; g += gridDim.x) {
            const uint64_t qrow = (uint64_t)g * QT * TILE + q * TILE + row;
            const float capv = (qcap && qrow < nq) ? qcap[qrow] : INFINITY;
            float thr = capv;
            int thr_slot = 0;
            for (int s2 = 0; s2 < R; ++s2) {
                cs[s2 * S + owner] = INFINITY;
                ci[s2 * S + owner] = 0xFFFFFFFFu;
            }
            TileWalk walk(rptr, rngs, g, ntiles);
            const uint32_t cnt = walk.count();
            for (uint32_t t = 0; t < cnt; ++t, ++it) {
                const uint32_t tile = walk.next();
                const uint32_t b = (uint32_t)(it & 1);
                if (!mbar_wait(accfull + b, (uint32_t)((it >> 1) & 1), lim)) {
                    *abort_flag = 1;
                    break;
                }
                fence_after();
                const uint32_t taddr =
                    tmem + ((uint32_t)(lq * 32) << 16) + b * (QT * TILE) + q * TILE + h * (TILE / HALVES);
#pragma unroll 1
                for (int c0 = 0; c0 < TILE / HALVES; c0 += 32) {
                    float r[32];
                    tmem_ld32(taddr + c0, r);
                    // branch-free prefilter: the chunk's minimum against the worst kept
                    float m[16];
#pragma unroll
                    for (int j = 0; j < 16; ++j) m[j] = fminf(r[j], r[j + 16]);
#pragma unroll
                    for (int w2 = 8; w2 >= 1; w2 >>= 1)
#pragma unroll
                        for (int j = 0; j < w2; ++j) m[j] = fminf(m[j], m[j + w2]);
                    const uint32_t base_idx = tile * TILE + h * (TILE / HALVES) + c0;
                    unsigned hits = __ballot_sync(0xFFFFFFFFu, m[0] < thr);
                    if (__popc(hits) > COOP_ROWS) {
                        // many rows have candidates: each lane scans its own row
                        if (m[0] < thr) {
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                if (r[j] < thr && base_idx + j < n) {
                                    const Worst w = cand_insert<R>(cs, ci, owner, thr_slot, r[j], base_idx + j);
                                    thr = fminf(w.thr, capv);
                                    thr_slot = w.slot;
                                }
                            }
                        }
                    } else {
                        // few rows: the warp takes them one at a time, lane j holding
                        // column j; inserts in ascending column order with a warp argmax
                        // over the row's kept slots (same operations as the lane path)
                        while (hits) {
                            const int L = __ffs(hits) - 1;
                            hits &= hits - 1;
                            if (lane == L) {
#pragma unroll
                                for (int j = 0; j < 32; j += 4)
                                    *(float4*)(srow + j) = make_float4(r[j], r[j + 1], r[j + 2], r[j + 3]);
                            }
                            __syncwarp();
                            const float v = srow[lane];
                            __syncwarp();
                            const int ownerL = owner - lane + L;
                            float thrL = __shfl_sync(0xFFFFFFFFu, thr, L);
                            int slotL = __shfl_sync(0xFFFFFFFFu, thr_slot, L);
                            const float capL = __shfl_sync(0xFFFFFFFFu, capv, L);
                            const bool inrange = base_idx + lane < n;
                            unsigned cand = __ballot_sync(0xFFFFFFFFu, inrange && v < thrL);
                            while (cand) {
                                const int jc = __ffs(cand) - 1;
                                if (lane == jc) {
                                    cs[slotL * S + ownerL] = v;
                                    ci[slotL * S + ownerL] = base_idx + jc;
                                }
                                __syncwarp();
                                // new worst of the row: highest score, lowest slot on ties
                                float wv = lane < R ? cs[lane * S + ownerL] : -INFINITY;
                                int ws = lane;
#pragma unroll
                                for (int o = 16; o; o >>= 1) {
                                    const float ov = __shfl_xor_sync(0xFFFFFFFFu, wv, o);
                                    const int os = __shfl_xor_sync(0xFFFFFFFFu, ws, o);
                                    if (ov > wv || (ov == wv && os < ws)) {
                                        wv = ov;
                                        ws = os;
                                    }
                                }
                                thrL = fminf(wv, capL);
                                slotL = ws;
                                // later columns of this row that still beat the new worst
                                cand &= ~((2u << jc) - 1u);
                                cand &= __ballot_sync(0xFFFFFFFFu, inrange && v < thrL);
                            }
                            if (lane == L) {
                                thr = thrL;
                                thr_slot = slotL;
                            }
                        }
                    }
                }
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(accempty + b);
            }
            if (*abort_flag) break;
            if (qrow < nq) {
                for (int s2 = 0; s2 < RCAND; ++s2) {
                    cand_score[qrow * RTOTAL + h * RCAND + s2] = s2 < R ? cs[s2 * S + owner] : INFINITY;
                    cand_idx[qrow * RTOTAL + h * RCAND + s2] = s2 < R ? ci[s2 * S + owner] : 0xFFFFFFFFu;
                }
            }
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (threadIdx.x == 0 && *abort_flag) atomicOr(status, DEV_TIMEOUT);
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

// ------------------------------------------------------------ FP32 candidate search
// The FP32 arm: squared distances computed on the CUDA cores as
// sum_t (q_t - c_t)^2, the re-rank's own operations in the same order
// (dimensions past d are zero on both sides and add exactly nothing), so the
// candidates are the exact FP32 nearest points, with no norm expansion and no
// reduced-precision operand. One thread per query, 256 queries per block, the
// query's coordinates in registers; points stream through shared memory in
// tiles of F32_TILE (every thread reads the same point: broadcast loads). Each
// query keeps its RCAND best (distance, id) in shared memory, the worst kept
// is the rejection threshold, so most points cost one compare after the
// distance. The other RCAND candidate slots are written empty.
constexpr int F32_THREADS = 256;
constexpr int F32_TILE = 64;

template <int DP>
__global__ void __launch_bounds__(F32_THREADS) k_knn_fp32(const float* __restrict__ X, uint64_t n, uint32_t d,
                                                          uint64_t q0, uint64_t nq, uint32_t* __restrict__ cand_idx) {
    extern __shared__ __align__(16) unsigned char smem[];
    float* tile = (float*)smem;                           // [F32_TILE][DP]
    float* cs = tile + F32_TILE * DP;                     // [RCAND][F32_THREADS]
    uint32_t* ci = (uint32_t*)(cs + RCAND * F32_THREADS);  // [RCAND][F32_THREADS]
    const uint32_t t = threadIdx.x;
    const uint64_t lq = (uint64_t)blockIdx.x * F32_THREADS + t;
    const bool have = lq < nq;
    float q[DP];
#pragma unroll
    for (int j = 0; j < DP; ++j) q[j] = (have && (uint32_t)j < d) ? X[(q0 + lq) * d + j] : 0.0f;
    for (int s2 = 0; s2 < RCAND; ++s2) {
        cs[s2 * F32_THREADS + t] = INFINITY;
        ci[s2 * F32_THREADS + t] = 0xFFFFFFFFu;
    }
    float thr = INFINITY;
    int thr_slot = 0;
    for (uint64_t base = 0; base < n; base += F32_TILE) {
        __syncthreads();  // the previous tile is no longer read
        for (uint32_t e = t; e < (uint32_t)(F32_TILE * DP); e += F32_THREADS) {
            const uint32_t p = e / DP, j = e % DP;
            tile[e] = (base + p < n && j < d) ? X[(base + p) * d + j] : 0.0f;
        }
        __syncthreads();
        const uint32_t cnt = (n - base < (uint64_t)F32_TILE) ? (uint32_t)(n - base) : (uint32_t)F32_TILE;
        for (uint32_t p = 0; p < cnt; ++p) {
            const float4* c4 = (const float4*)(tile + p * DP);
            float acc = 0.0f;
#pragma unroll
            for (int j4 = 0; j4 < DP / 4; ++j4) {
                const float4 c = c4[j4];
                float df = __fsub_rn(q[4 * j4], c.x);
                acc = __fmaf_rn(df, df, acc);
                df = __fsub_rn(q[4 * j4 + 1], c.y);
                acc = __fmaf_rn(df, df, acc);
                df = __fsub_rn(q[4 * j4 + 2], c.z);
                acc = __fmaf_rn(df, df, acc);
                df = __fsub_rn(q[4 * j4 + 3], c.w);
                acc = __fmaf_rn(df, df, acc);
            }
            if (acc < thr) {
                cs[thr_slot * F32_THREADS + t] = acc;
                ci[thr_slot * F32_THREADS + t] = (uint32_t)(base + p);
                thr = -INFINITY;
                for (int s2 = 0; s2 < RCAND; ++s2) {
                    const float x = cs[s2 * F32_THREADS + t];
                    if (x > thr) {
                        thr = x;
                        thr_slot = s2;
                    }
                }
            }
        }
    }
    if (have) {
        for (int s2 = 0; s2 < RCAND; ++s2) {
            cand_idx[lq * RTOTAL + s2] = ci[s2 * F32_THREADS + t];
            cand_idx[lq * RTOTAL + RCAND + s2] = 0xFFFFFFFFu;
        }
    }
}

template <int DP>
void candidates_fp32(Ctx& c, const float* dX, uint64_t n, uint32_t d, uint64_t q0, uint64_t nq, uint32_t* cand_idx) {
    const size_t sm = (size_t)F32_TILE * DP * 4 + (size_t)RCAND * F32_THREADS * 8;
    SC_CUDA(cudaFuncSetAttribute(k_knn_fp32<DP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const uint64_t blocks = (nq + F32_THREADS - 1) / F32_THREADS;
    k_knn_fp32<DP><<<(unsigned)blocks, F32_THREADS, sm, c.stream>>>(dX, n, d, q0, nq, cand_idx);
    SC_LAUNCH_CHECK();
    c.launches++;
}

// ------------------------------------------------------------ exact re-rank
__device__ __forceinline__ uint64_t rerank_key(const float* __restrict__ X, uint64_t n, uint32_t d, uint64_t q,
                                               uint32_t j) {
    if (j >= n) return ~0ull;
    const float* a = X + q * d;
    const float* b = X + (uint64_t)j * d;
    float acc = 0.0f;
    for (uint32_t t = 0; t < d; ++t) {
        const float diff = __fsub_rn(a[t], b[t]);
        acc = __fmaf_rn(diff, diff, acc);
    }
    // (distance, self first, index); acc >= 0 so its bits order like the value
    return ((uint64_t)__float_as_uint(acc) << 32) | (j == (uint32_t)q ? 0u : j + 1u);
}

__device__ __forceinline__ uint64_t warp_sort32(uint64_t key) {
    const unsigned lane = threadIdx.x & 31u;
    for (int size = 2; size <= 32; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, key, stride);
            const bool up = ((lane & size) == 0);
            const bool lower = (lane & stride) == 0;
            const uint64_t mn = key < other ? key : other, mx = key < other ? other : key;
            key = (lower == up) ? mn : mx;
        }
    }
    return key;
}

// One warp per query: exact FP32 distances of its RTOTAL = 64 candidates (two
// per lane), the 32 smallest kept by a merge-split of two sorted halves, then
// the first k+1 written.
// Queries are points q0 .. q0 + nq - 1; rows of cand_idx / out_* are local.
__global__ void k_knn_rerank(const float* __restrict__ X, uint64_t n, uint32_t d, uint32_t k, uint64_t q0,
                             uint64_t nq, const uint32_t* __restrict__ cand_idx, uint32_t* __restrict__ out_idx,
                             float* __restrict__ out_d2) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t lq = warp; lq < nq; lq += nwarps) {
        const uint64_t q = q0 + lq;
        uint64_t ka = warp_sort32(rerank_key(X, n, d, q, cand_idx[lq * RTOTAL + lane]));
        uint64_t kb = warp_sort32(rerank_key(X, n, d, q, cand_idx[lq * RTOTAL + 32 + lane]));
        const uint64_t kbr = __shfl_sync(0xFFFFFFFFu, kb, 31 - lane);
        uint64_t key = ka < kbr ? ka : kbr;  // the 32 smallest, as a bitonic sequence
        for (int stride = 16; stride > 0; stride >>= 1) {
            const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, key, stride);
            key = (lane & stride) == 0 ? (key < other ? key : other) : (key < other ? other : key);
        }
        if (lane <= k) {
            const uint32_t tag = (uint32_t)key;
            const uint32_t idx = (key == ~0ull) ? 0xFFFFFFFFu : (tag == 0 ? (uint32_t)q : tag - 1u);
            out_idx[lq * (k + 1) + lane] = idx;
            out_d2[lq * (k + 1) + lane] = key == ~0ull ? INFINITY : __uint_as_float((uint32_t)(key >> 32));
        }
    }
}

// ------------------------------------------------------------ sigma and connectivities
// sigma_i: median of the positive distances among the k+1 (neighborhood/mod.rs:480-499;
// the kd-tree path's sqrt(median(d^2)), :105-124, is the same element), 1 if none;
// or the k-th neighbour's distance.
__global__ void k_knn_sigma(const float* __restrict__ d2, uint64_t n, uint32_t k, int kth, float* sigma) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float* r = d2 + i * (k + 1);
        // with fewer than k + 1 points the trailing slots are empty (infinite):
        // only the neighbours the search returned count, as in the reference
        uint32_t m = 0;
        while (m <= k && isfinite(r[m])) ++m;
        if (kth) {
            sigma[i] = m ? sqrtf(r[m - 1]) : 1.0f;
            continue;
        }
        uint32_t pos = 0;
        for (uint32_t t = 0; t < m; ++t) pos += r[t] > 0.0f;
        if (pos == 0) {
            sigma[i] = 1.0f;
            continue;
        }
        // rows are sorted ascending, positive entries are the last `pos` of the m
        uint32_t first = m - pos;
        sigma[i] = sqrtf(r[first + pos / 2]);
    }
}

// Connectivity weight of :139-163 in f32, operation for operation.
__device__ __forceinline__ float gauss_w(float dist_sq, float si, float sj, bool* ok) {
    float si2 = __fmul_rn(si, si), sj2 = __fmul_rn(sj, sj);
    float den = __fadd_rn(si2, sj2);
    *ok = den > 0.0f;
    if (!*ok) return 0.0f;
    float num = __fmul_rn(__fmul_rn(2.0f, si), sj);
    float norm = sqrtf(__fdiv_rn(num, den));
    float ex = expf(__fdiv_rn(-dist_sq, den));
    return __fmul_rn(norm, ex);
}

// Emit (row << 32 | col) keys and weights. lower_id: only from the row i <= j,
// both directions (the reference's rule). union: every listed pair, both
// directions; duplicates are removed after the sort.
__global__ void k_knn_pairs(const uint32_t* __restrict__ idx, const float* __restrict__ d2, uint64_t n,
                            uint32_t k, const float* __restrict__ sigma, int sym_union, int squared,
                            unsigned long long* keys, float* w, unsigned long long* count) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        for (uint32_t t = 1; t <= k; ++t) {
            uint32_t j = idx[i * (k + 1) + t];
            if (j >= n) continue;
            if (!sym_union && !(i <= j)) continue;
            if (sym_union && j == i) continue;
            // HNSW path: squares the returned distance; kd-tree path: already squared
            float dist_sq = squared ? d2[i * (k + 1) + t] : __fmul_rn(sqrtf(d2[i * (k + 1) + t]),
                                                                       sqrtf(d2[i * (k + 1) + t]));
            bool ok;
            float wt = gauss_w(dist_sq, sigma[i], sigma[j], &ok);
            if (!ok || !(wt > 1e-14f)) continue;
            unsigned long long pos = atomicAdd(count, i == j ? 1ull : 2ull);
            keys[pos] = ((unsigned long long)i << 32) | j;
            w[pos] = wt;
            if (i != j) {
                keys[pos + 1] = ((unsigned long long)j << 32) | i;
                w[pos + 1] = wt;
            }
        }
    }
}

__global__ void k_dedupe_flags(const unsigned long long* __restrict__ keys, uint64_t N, uint8_t* keep) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x)
        keep[i] = (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void k_split_rowcol(const unsigned long long* __restrict__ keys, uint64_t N, uint32_t* rows,
                               uint32_t* cols) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        rows[i] = (uint32_t)(keys[i] >> 32);
        cols[i] = (uint32_t)keys[i];
    }
}

__global__ void k_ptr_from_rows(const uint32_t* __restrict__ rows, uint64_t N, uint64_t R, uint64_t* start) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= N;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = i < N ? rows[i] : R;
        uint64_t prev = i == 0 ? 0 : (uint64_t)rows[i - 1] + 1;
        for (uint64_t q = prev; q <= r && q <= R; ++q) start[q] = i;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        SC_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !p) fail(SC_E_CUDA, "cuTensorMapEncodeTiled is unavailable");
        fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

// 2-D map of n rows of `row_bytes` bytes, tiles of 128 rows, swizzled by the row size.
CUtensorMap make_map(const void* base, uint64_t n, uint32_t row_bytes, bool bytes_type) {
    CUtensorMap m;
    const uint32_t esize = bytes_type ? 1 : 2;
    cuuint64_t dims[2] = {(cuuint64_t)(row_bytes / esize), (cuuint64_t)n};
    cuuint64_t strides[1] = {(cuuint64_t)row_bytes};
    cuuint32_t box[2] = {(cuuint32_t)(row_bytes / esize), (cuuint32_t)TILE};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode_fn()(&m, bytes_type ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                             (void*)base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(SC_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return m;
}

// Tile ranges of each query group of a pruned search (device arrays).
struct TileLists {
    const uint32_t* rptr = nullptr;  // ngroups + 1
    const uint2* rngs = nullptr;     // (first tile, tile count)
    const float* cap = nullptr;      // per query (launch order): the score bound of k_knn_tc's qcap
};

template <int KA, bool F8, int R = RCAND>
void launch_tc(Ctx& c, const CUtensorMap& ta, const CUtensorMap& tb, uint64_t n, uint64_t nq, float* cand_score,
               uint32_t* cand_idx, const TileLists& tl = TileLists{}) {
    using L = KnnSmem<KA, R>;
    SC_CUDA(cudaFuncSetAttribute(k_knn_tc<KA, F8, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::BYTES));
    const uint32_t ngroups = (uint32_t)((nq + QT * TILE - 1) / (QT * TILE));
    const unsigned grid = std::min<unsigned>(ngroups, (unsigned)c.sm_count);
    k_knn_tc<KA, F8, R><<<grid, KNN_THREADS, L::BYTES, c.stream>>>(ta, tb, (uint32_t)n, (uint32_t)nq, cand_score,
                                                                 cand_idx, c.d_status, c.wait_limit,
                                                                 c.knn_hold_tiles, tl.rptr, tl.rngs, tl.cap);
    SC_LAUNCH_CHECK();
    c.launches++;
}

// Candidates of the queries q0 .. q0 + nq - 1 against all n points. A is the
// query operand: its tensor map starts at row q0 (KA * 2 bytes per row, a
// multiple of 16, so every row start is a legal TMA base).
template <int KA>
void candidates(Ctx& c, const float* dX, uint64_t n, uint32_t d, uint64_t q0, uint64_t nq, float* cand_score,
                uint32_t* cand_idx) {
    DBuf<__nv_bfloat16> A(c, n * KA), B(c, n * KA);
    k_knn_prep<KA><<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, A.get(), B.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    CUtensorMap ta = make_map(A.get() + q0 * KA, nq, KA * 2, false), tb = make_map(B.get(), n, KA * 2, false);
    launch_tc<KA, false>(c, ta, tb, n, nq, cand_score, cand_idx);
}

// The same search with e4m3 operands (64-byte rows, the geometry of BF16 KA = 32).
void candidates_f8(Ctx& c, const float* dX, uint64_t n, uint32_t d, uint64_t q0, uint64_t nq, float* cand_score,
                   uint32_t* cand_idx) {
    DBuf<uint8_t> A(c, n * 64), B(c, n * 64);
    DBuf<unsigned> mx(c, 2);
    zero(c, mx.get(), 2);
    k_knn_scales<<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, mx.get(), mx.get() + 1);
    k_knn_prep_f8<<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, mx.get(), mx.get() + 1, A.get(), B.get());
    SC_LAUNCH_CHECK();
    c.launches += 2;
    CUtensorMap ta = make_map(A.get() + q0 * 64, nq, 64, true), tb = make_map(B.get(), n, 64, true);
    launch_tc<32, true>(c, ta, tb, n, nq, cand_score, cand_idx);
}

// ------------------------------------------------------------ exact pruning
// Points are grouped by a deterministic k-means (fixed-point sums, ties to the
// lower centroid) and sorted by group, so every 128-row tile is spatially
// coherent. A query group first scans the tiles of its own clusters; the exact
// FP32 re-rank of those candidates bounds each query's (k+1)-th distance from
// above. A cluster b can hold a closer point only if a lower bound on
// |q - x| over x in b is at most that distance: the ball bound |q - c_b| - r_b
// and the slab bound of the direction u from the query's cluster centre to
// c_b (every x in b projects into [lo, hi] on u, so |q - x| >= the distance
// from <q, u> to [lo, hi]). The second pass scans the own tiles and those of
// every cluster some query of the group cannot exclude, narrowed to the fine
// cells (~256 points) a ball bound cannot exclude; skipped points are provably
// farther than the query's (k+1)-th neighbour, so the result is the full
// search's. The first pass keeps fewer candidates (it only yields the bound)
// and walks each group's nearest cells first; the second starts every query's
// candidate rows from a proven score bound derived from the first pass's
// distance (k_pass2_cap). Both passes take their tile lists from the device.
constexpr int KM_ITERS = 8;
constexpr uint32_t KM_SAMPLE = 65536;  // points the Lloyd steps run on

// Nearest centroid of every point (squared FP32 distance, ties to the lower id).
__global__ void k_km_assign(const float* __restrict__ X, uint64_t n, uint32_t d, const float* __restrict__ cent,
                            uint32_t K, uint32_t* assign) {
    // centroid rows padded to a multiple of 4 floats, read as float4
    extern __shared__ __align__(16) float s_cent[];
    const uint32_t dp = (d + 3) & ~3u;
    for (uint32_t i = threadIdx.x; i < K * dp; i += blockDim.x) {
        const uint32_t c = i / dp, j = i % dp;
        s_cent[i] = j < d ? cent[(uint64_t)c * d + j] : 0.0f;
    }
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        // the point in registers (d <= 62): the centroid loop then reads only
        // shared memory, every lane the same words (a broadcast)
        float x[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) x[j] = (uint32_t)j < d ? X[i * d + j] : 0.0f;
        float best = INFINITY;
        uint32_t bc = 0;
        for (uint32_t c = 0; c < K; ++c) {
            const float4* m4 = reinterpret_cast<const float4*>(s_cent + (uint64_t)c * dp);
            float acc = 0.0f;
#pragma unroll
            for (int q = 0; q < 16; ++q)
                if ((uint32_t)(4 * q) < d) {
                    const float4 mv = m4[q];
                    const float mm[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
                    for (int t = 0; t < 4; ++t)
                        if ((uint32_t)(4 * q + t) < d) {
                            const float df = __fsub_rn(x[4 * q + t], mm[t]);
                            acc = __fmaf_rn(df, df, acc);
                        }
                }
            if (acc < best) {
                best = acc;
                bc = c;
            }
        }
        assign[i] = bc;
    }
}

// Per-cluster coordinate sums in fixed point (x * 2^s rounded; integer adds are
// associative, so the centroids do not depend on the order) and counts.
__global__ void k_km_accum(const float* __restrict__ X, uint64_t n, uint32_t d, const uint32_t* __restrict__ assign,
                           uint32_t K, double scale, unsigned long long* sum, unsigned* cnt) {
    extern __shared__ unsigned long long s_sum[];
    unsigned* s_cnt = (unsigned*)(s_sum + K * d);
    for (uint32_t i = threadIdx.x; i < K * d; i += blockDim.x) s_sum[i] = 0;
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) s_cnt[i] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = assign[i];
        const float* x = X + i * d;
        for (uint32_t j = 0; j < d; ++j)
            atomicAdd(s_sum + c * d + j, (unsigned long long)__double2ll_rn((double)x[j] * scale));
        atomicAdd(s_cnt + c, 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < K * d; i += blockDim.x)
        if (s_sum[i]) atomicAdd(sum + i, s_sum[i]);
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x)
        if (s_cnt[i]) atomicAdd(cnt + i, s_cnt[i]);
}

// Farthest-point seeding: d2min[i] = min(d2min[i], |x_i - c|^2) for the newest
// centre c; the next centre is the sample point farthest from every centre
// chosen so far (ties to the lower index), so separated groups of points each
// get a centre before any group gets a second.
__global__ void k_seed_update(const float* __restrict__ Xs, uint64_t n, uint32_t d, const float* __restrict__ c,
                              float* d2min) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float acc = 0.0f;
        for (uint32_t j = 0; j < d; ++j) {
            const float df = __fsub_rn(Xs[i * d + j], c[j]);
            acc = __fmaf_rn(df, df, acc);
        }
        d2min[i] = fminf(d2min[i], acc);
    }
}

// One block: the index of the largest d2min (lowest index on ties); copies
// that point into centre slot `t`.
__global__ void k_seed_pick(const float* __restrict__ Xs, uint64_t n, uint32_t d, const float* __restrict__ d2min,
                            float* cent, uint32_t t) {
    __shared__ float sv[32];
    __shared__ uint32_t si[32];
    float bv = -1.0f;
    uint32_t bi = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const float v = d2min[i];
        if (v > bv) {
            bv = v;
            bi = i;
        }
    }
    for (int o = 16; o; o >>= 1) {
        const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
        const uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
        if (ov > bv || (ov == bv && oi < bi)) {
            bv = ov;
            bi = oi;
        }
    }
    if ((threadIdx.x & 31) == 0) {
        sv[threadIdx.x >> 5] = bv;
        si[threadIdx.x >> 5] = bi;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const uint32_t nw = blockDim.x >> 5;
        bv = threadIdx.x < nw ? sv[threadIdx.x] : -1.0f;
        bi = threadIdx.x < nw ? si[threadIdx.x] : 0xFFFFFFFFu;
        for (int o = 16; o; o >>= 1) {
            const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
            const uint32_t oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) {
                bv = ov;
                bi = oi;
            }
        }
        if (threadIdx.x == 0) si[0] = bi;
    }
    __syncthreads();
    const uint32_t pick = si[0];
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) cent[(uint64_t)t * d + j] = Xs[(uint64_t)pick * d + j];
}

// New centroids; an empty cluster keeps its centroid.
__global__ void k_km_update(const unsigned long long* __restrict__ sum, const unsigned* __restrict__ cnt, uint32_t K,
                            uint32_t d, double inv_scale, float* cent) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < K * d; i += gridDim.x * blockDim.x) {
        const uint32_t c = i / d;
        if (cnt[c]) cent[i] = (float)((double)(long long)sum[i] * inv_scale / (double)cnt[c]);
    }
}

__global__ void k_gather_rows(const float* __restrict__ X, const uint32_t* __restrict__ rows, uint64_t m, uint32_t d,
                              float* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m * d; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = X[(uint64_t)rows[i / d] * d + i % d];
}

__global__ void k_iota_u32(uint32_t* x, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        x[i] = (uint32_t)i;
}

// Order-preserving map of floats to unsigned integers (for atomic min / max).
__device__ __forceinline__ unsigned ord32(float x) {
    const unsigned b = __float_as_uint(x);
    return (b >> 31) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unord32(unsigned k) {
    return __uint_as_float((k >> 31) ? (k & 0x7FFFFFFFu) : ~k);
}

// Fine cell of every point inside its coarse cluster (points sorted by coarse
// cluster): the nearest of the cluster's fine centres, its points at local
// positions 0, FINE, 2 FINE, ... (ties to the lower cell). Sorting by fine cell
// then makes each group of 256 consecutive queries one spatially tight cell,
// so its queries need similar clusters.
constexpr uint32_t FINE = 256;

__global__ void k_fine_assign(const float* __restrict__ Xs, uint64_t n, uint32_t d, const uint32_t* __restrict__ cl,
                              const uint64_t* __restrict__ cstart, const uint32_t* __restrict__ fbase,
                              uint32_t* fine) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = cl[i];
        const uint64_t s0 = cstart[b], s1 = cstart[b + 1];
        float x[64];  // the point in registers (d <= 62)
#pragma unroll
        for (int j = 0; j < 64; ++j) x[j] = (uint32_t)j < d ? Xs[i * d + j] : 0.0f;
        float best = INFINITY;
        uint32_t bf = 0, f = 0;
        for (uint64_t p = s0; p < s1; p += FINE, ++f) {
            const float* m = Xs + p * d;
            float acc = 0.0f;
#pragma unroll
            for (int j = 0; j < 64; ++j)
                if ((uint32_t)j < d) {
                    const float df = __fsub_rn(x[j], m[j]);
                    acc = __fmaf_rn(df, df, acc);
                }
            if (acc < best) {
                best = acc;
                bf = f;
            }
        }
        fine[i] = fbase[b] + bf;
    }
}

// A chunk of consecutive sorted points of one cluster (blocks of the extent
// and bound kernels).
struct Chunk {
    uint32_t cluster;
    uint64_t begin, end;
};

// Per chunk (one block): the radius of its cluster around the centre, and the
// extent [lo, hi] of its points along every direction u_{a,b} from a centre a
// to its own centre b. Ub[b][a][j] (FP32) is staged in shared memory; warps
// reduce by shuffles, the block in shared memory, and one thread per direction
// updates the global extents (order-preserving integer min / max).
__global__ void k_cluster_extent(const float* __restrict__ Xs, uint32_t d, const Chunk* __restrict__ chunks,
                                 const float* __restrict__ cent, const float* __restrict__ Ub, uint32_t K,
                                 unsigned* rad, unsigned* lo, unsigned* hi) {
    extern __shared__ float sm[];
    float* su = sm;                                   // K * d
    unsigned* slo = (unsigned*)(su + (size_t)K * d);  // K
    unsigned* shi = slo + K;                          // K
    __shared__ unsigned srad;
    const Chunk ch = chunks[blockIdx.x];
    const uint32_t b = ch.cluster;
    for (uint32_t i = threadIdx.x; i < K * d; i += blockDim.x) su[i] = Ub[(uint64_t)b * K * d + i];
    for (uint32_t i = threadIdx.x; i < K; i += blockDim.x) {
        slo[i] = 0xFFFFFFFFu;
        shi[i] = 0u;
    }
    if (threadIdx.x == 0) srad = 0u;
    __syncthreads();
    const unsigned FULL = 0xFFFFFFFFu;
    for (uint64_t base = ch.begin; base < ch.end; base += blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t ii = i < ch.end ? i : ch.end - 1;  // idle lanes repeat a point: min / max unchanged
        float x[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) x[j] = (uint32_t)j < d ? Xs[ii * d + j] : 0.0f;
        float r2 = 0.0f;
#pragma unroll
        for (int j = 0; j < 64; ++j)
            if ((uint32_t)j < d) {
                const float df = x[j] - cent[b * d + j];
                r2 = __fmaf_rn(df, df, r2);
            }
        unsigned kr = ord32(sqrtf(r2));
        for (int o = 16; o; o >>= 1) kr = max(kr, __shfl_xor_sync(FULL, kr, o));
        if ((threadIdx.x & 31) == 0) atomicMax(&srad, kr);
        for (uint32_t a = 0; a < K; ++a) {
            const float* u = su + (size_t)a * d;
            float p = 0.0f;
#pragma unroll
            for (int j = 0; j < 64; ++j)
                if ((uint32_t)j < d) p = __fmaf_rn(x[j], u[j], p);
            unsigned kl = ord32(p), kh = kl;
            for (int o = 16; o; o >>= 1) {
                kl = min(kl, __shfl_xor_sync(FULL, kl, o));
                kh = max(kh, __shfl_xor_sync(FULL, kh, o));
            }
            if ((threadIdx.x & 31) == 0) {
                atomicMin(slo + a, kl);
                atomicMax(shi + a, kh);
            }
        }
    }
    __syncthreads();
    for (uint32_t a = threadIdx.x; a < K; a += blockDim.x) {
        atomicMin(lo + (uint64_t)a * K + b, slo[a]);
        atomicMax(hi + (uint64_t)a * K + b, shi[a]);
    }
    if (threadIdx.x == 0) atomicMax(rad + b, srad);
}

// For every sorted query (chunks of its own cluster a, one block each): the
// clusters whose lower bound does not exclude them given its current (k+1)-th
// distance, as the bits of its own mask (words 64-bit words per query). FP32 with margins: `eps` bounds the
// rounding of a projection or a distance (a few ulps of the largest |x| times
// d), so every bound used is below the exact one.
__global__ void k_cluster_needs(const float* __restrict__ Xs, uint32_t d, const Chunk* __restrict__ chunks,
                                const uint32_t* __restrict__ perm, const float* __restrict__ d2k, uint32_t k1,
                                const float* __restrict__ cent, const unsigned* __restrict__ rad,
                                const float* __restrict__ Ua, const unsigned* __restrict__ lo,
                                const unsigned* __restrict__ hi, uint32_t K, float eps, uint32_t words,
                                unsigned long long* mask) {
    extern __shared__ float sm[];
    float* su = sm;                       // K * d: directions from a to every b
    float* sc = su + (size_t)K * d;       // K * d: centres
    float* sr = sc + (size_t)K * d;       // K: radii
    float* sl = sr + K;                   // K: lo[a][b]
    float* sh = sl + K;                   // K: hi[a][b]
    const Chunk ch = chunks[blockIdx.x];
    const uint32_t a = ch.cluster;
    for (uint32_t i = threadIdx.x; i < K * d; i += blockDim.x) {
        su[i] = Ua[(uint64_t)a * K * d + i];
        sc[i] = cent[i];
    }
    for (uint32_t b = threadIdx.x; b < K; b += blockDim.x) {
        sr[b] = unord32(rad[b]);
        sl[b] = unord32(lo[(uint64_t)a * K + b]);
        sh[b] = unord32(hi[(uint64_t)a * K + b]);
    }
    __syncthreads();
    for (uint64_t base = ch.begin; base < ch.end; base += blockDim.x) {
        const uint64_t i = base + threadIdx.x;
        const bool ok = i < ch.end;
        const uint64_t ii = ok ? i : ch.end - 1;
        float x[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) x[j] = (uint32_t)j < d ? Xs[ii * d + j] : 0.0f;
        const float kd2 = d2k[(uint64_t)perm[ii] * k1 + (k1 - 1)];
        // no (k+1)-th neighbour among the own clusters: every cluster is needed
        const float kth = isfinite(kd2) ? sqrtf(kd2) * (1.0f + 1e-5f) + eps : INFINITY;
        unsigned long long m[4] = {0ull, 0ull, 0ull, 0ull};
        for (uint32_t b = 0; b < K; ++b) {
            bool need = false;
            if (b != a) {
                const float* m = sc + (size_t)b * d;
                const float* u = su + (size_t)b * d;
                float dc = 0.0f, p = 0.0f;
#pragma unroll
                for (int j = 0; j < 64; ++j)
                    if ((uint32_t)j < d) {
                        const float df = x[j] - m[j];
                        dc = __fmaf_rn(df, df, dc);
                        p = __fmaf_rn(x[j], u[j], p);
                    }
                const float ball = sqrtf(dc) * (1.0f - 1e-5f) - sr[b] - eps;
                const float slab = fmaxf(sl[b] - p, p - sh[b]) - 2.0f * eps;
                need = fmaxf(ball, slab) <= kth;
            }
            if (need) m[b / 64] |= 1ull << (b % 64);
        }
        if (ok)
            for (uint32_t w = 0; w < words; ++w) mask[ii * words + w] = m[w];
    }
}

// Pass-2 order of the queries: by own cluster, then by a hash of the set of
// clusters the query needs, so each group of 256 holds queries needing the
// same clusters and the union a group scans stays close to what one needs.
__global__ void k_need_keys(const unsigned long long* __restrict__ mask, const uint32_t* __restrict__ cl, uint64_t n,
                            uint32_t words, unsigned long long* keys, uint32_t* pos) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h = 0x2545F4914F6CDD1Dull;
        for (uint32_t w = 0; w < words; ++w) h = splitmix(h ^ mask[i * words + w]);
        keys[i] = ((unsigned long long)cl[i] << 32) | (h >> 32);
        pos[i] = (uint32_t)i;
    }
}

// Rows of an operand (row_bytes, a multiple of 16) gathered in the order `ord`.
__global__ void k_gather_operand_rows(const uint4* __restrict__ src, const uint32_t* __restrict__ ord, uint64_t n,
                                      uint32_t row_vec, uint4* dst) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n * row_vec;
         i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[(uint64_t)ord[i / row_vec] * row_vec + i % row_vec];
}

// Per pass-2 group (one warp): the OR of its queries' masks, and the clusters
// of its first and last query (the group's own clusters lie between them).
__global__ void k_group_needs(const unsigned long long* __restrict__ mask, const uint32_t* __restrict__ ord,
                              const uint32_t* __restrict__ cl, uint64_t n, uint32_t words, uint64_t ngroups,
                              unsigned long long* gmask, uint32_t* gown) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = warp; g < ngroups; g += nwarps) {
        const uint64_t b = g * (QT * TILE), e = min(n, b + QT * TILE);
        for (uint32_t w = 0; w < words; ++w) {
            unsigned long long acc = 0ull;
            for (uint64_t i = b + lane; i < e; i += 32) acc |= mask[(uint64_t)ord[i] * words + w];
            for (int o = 16; o; o >>= 1) acc |= __shfl_xor_sync(0xFFFFFFFFu, acc, o);
            if (lane == 0) gmask[g * words + w] = acc;
        }
        if (lane == 0) {
            gown[2 * g] = cl[ord[b]];
            gown[2 * g + 1] = cl[ord[e - 1]];
        }
    }
}

// Points per fine cell (cells numbered in sorted order: a cell's points are
// contiguous) and the radius of every cell around its centre (the sample
// point that defined it).
__global__ void k_cell_count(const uint32_t* __restrict__ cell, uint64_t n, unsigned* cnt) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + cell[i], 1u);
}

__global__ void k_cell_radius(const float* __restrict__ Xs, uint64_t n, uint32_t d, const uint32_t* __restrict__ cell,
                              const float* __restrict__ fcent, unsigned* crad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f = cell[i];
        float r2 = 0.0f;
        for (uint32_t j = 0; j < d; ++j) {
            const float df = Xs[i * d + j] - fcent[(uint64_t)f * d + j];
            r2 = __fmaf_rn(df, df, r2);
        }
        atomicMax(crad + f, ord32(sqrtf(r2)));
    }
}

// Per pass-2 group (one block, a thread per query): the fine cells of the
// group's candidate clusters (its own clusters and every cluster one of its
// queries needs) that the ball bound |q - c_f| - r_f cannot exclude for at
// least one query, as bits of the group's cell bitmap. The group's queries
// are neighbours in the sorted order (one or a few fine cells), so a ball
// around them (centre: their mean, radius: the farthest of them) first
// excludes, for all queries at once, every cell with
// |g - c_f| - r_g - r_f > max kth; only the remaining cells are tested per
// query. Both tests carry the same rounding margins, the group test twice.
__global__ void k_group_cells(const float* __restrict__ Xs, uint64_t n, uint32_t d, const uint32_t* __restrict__ ord,
                              const uint32_t* __restrict__ perm, const float* __restrict__ d2k, uint32_t k1,
                              const unsigned long long* __restrict__ gmask, const uint32_t* __restrict__ gown,
                              uint32_t words, uint32_t K, const uint32_t* __restrict__ fbase,
                              const float* __restrict__ fcent, const unsigned* __restrict__ crad, float eps,
                              uint32_t cwords, const unsigned long long* __restrict__ qmask,
                              const uint32_t* __restrict__ qcl, unsigned* gcell) {
    const uint64_t g = blockIdx.x;
    const uint64_t r = g * (QT * TILE) + threadIdx.x;
    const bool ok = r < n;
    const uint64_t sq = ok ? ord[r] : ord[n - 1];
    float x[64];
#pragma unroll
    for (int j = 0; j < 64; ++j) x[j] = (uint32_t)j < d ? Xs[sq * d + j] : 0.0f;
    const float kd2 = d2k[(uint64_t)perm[sq] * k1 + (k1 - 1)];
    const float kth = isfinite(kd2) ? sqrtf(kd2) * (1.0f + 1e-5f) + eps : INFINITY;
    extern __shared__ unsigned s_bits[];  // cwords: the result, then cwords: cells the group ball keeps
    unsigned* s_maybe = s_bits + cwords;
    __shared__ float s_c[64];
    __shared__ unsigned s_r, s_k;  // group radius and max kth (ordered bits)
    for (uint32_t w = threadIdx.x; w < cwords; w += blockDim.x) s_bits[w] = s_maybe[w] = 0u;
    for (uint32_t j = threadIdx.x; j < 64; j += blockDim.x) s_c[j] = 0.0f;
    if (threadIdx.x == 0) s_r = s_k = 0u;
    __syncthreads();
    // group centre: the mean of its queries, summed in a fixed order (a warp
    // per dimension, lanes over the queries, a fixed tree)
    const uint64_t g0 = g * (QT * TILE), gcount = n - g0 < (uint64_t)(QT * TILE) ? n - g0 : (uint64_t)(QT * TILE);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t j = wid; j < d; j += nw) {
        float acc = 0.0f;
        for (uint64_t t = lane; t < gcount; t += 32) acc += Xs[(uint64_t)ord[g0 + t] * d + j];
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        if (lane == 0) s_c[j] = acc / (float)gcount;
    }
    __syncthreads();
    if (ok) {
        float dq = 0.0f;
#pragma unroll
        for (int j = 0; j < 64; ++j)
            if ((uint32_t)j < d) {
                const float df = x[j] - s_c[j];
                dq = __fmaf_rn(df, df, dq);
            }
        atomicMax(&s_r, ord32(sqrtf(dq)));
        atomicMax(&s_k, ord32(kth));
    }
    __syncthreads();
    const float rg = unord32(s_r) * (1.0f + 1e-5f), kmax = unord32(s_k);
    const uint32_t a0 = gown[2 * g], a1 = gown[2 * g + 1];
    // the group-ball test, a thread per cell
    for (uint32_t b = 0; b < K; ++b) {
        const bool cand = (b >= a0 && b <= a1) || ((gmask[g * words + b / 64] >> (b % 64)) & 1ull);
        if (!cand) continue;  // uniform over the block
        for (uint32_t f = fbase[b] + threadIdx.x; f < fbase[b + 1]; f += blockDim.x) {
            const float* m = fcent + (uint64_t)f * d;
            float dc = 0.0f;
            for (uint32_t j = 0; j < d; ++j) {
                const float df = s_c[j] - m[j];
                dc = __fmaf_rn(df, df, dc);
            }
            if (!(sqrtf(dc) * (1.0f - 1e-5f) - rg - unord32(crad[f]) - 2.0f * eps > kmax))
                atomicOr(s_maybe + f / 32, 1u << (f % 32));
        }
    }
    __syncthreads();
    // the per-query test on the cells the group ball kept, for the queries
    // whose own cluster or needs hold the cell's cluster (the group scans the
    // union of its queries' needs; each query tests only its own)
    const uint32_t myown = qcl[sq];
    const unsigned long long* mym = qmask + sq * words;
    uint32_t b = 0;  // the cluster of cell f (cells ascend, so does b)
    for (uint32_t wd = 0; wd < cwords; ++wd) {
        unsigned bits = s_maybe[wd];  // uniform over the block
        while (bits) {
            const uint32_t f = wd * 32 + (uint32_t)(__ffs(bits) - 1);
            bits &= bits - 1;
            while (fbase[b + 1] <= f) ++b;
            const bool mine = ok && (b == myown || ((mym[b / 64] >> (b % 64)) & 1ull));
            if (!__any_sync(0xFFFFFFFFu, mine)) continue;
            const float* m = fcent + (uint64_t)f * d;
            float dc = 0.0f;
#pragma unroll
            for (int j = 0; j < 64; ++j)
                if ((uint32_t)j < d) {
                    const float df = x[j] - m[j];
                    dc = __fmaf_rn(df, df, dc);
                }
            const bool need = mine && sqrtf(dc) * (1.0f - 1e-5f) - unord32(crad[f]) - eps <= kth;
            // one shared OR per warp that needs the cell (most cells are needed by all or none)
            if (__ballot_sync(0xFFFFFFFFu, need) && lane == 0) atomicOr(s_bits + f / 32, 1u << (f % 32));
        }
    }
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < cwords; w += blockDim.x) gcell[g * cwords + w] = s_bits[w];
}

// Pass 1's tile order, a block per query group: the group's own-cluster tiles
// [tb[g], te[g]) sorted by the distance from the group's centre (the mean of
// its queries) to the centroid of the cell holding each tile's first point,
// nearest first, ties by tile id; each tile one range of length 1 at
// out[rptr[g] ..]. Nearest points first tighten the rows' thresholds within
// the first tiles. More tiles than ORDER_CAP keep ascending order from the
// group's own tile.
constexpr int ORDER_CAP = 2048;
__global__ void k_order_tiles(const float* __restrict__ Xs, uint64_t n, uint32_t d, const uint32_t* __restrict__ tb,
                              const uint32_t* __restrict__ te, const uint32_t* __restrict__ tile_cell,
                              const float* __restrict__ fcent, const uint32_t* __restrict__ rptr, uint2* out) {
    __shared__ float s_c[64];
    __shared__ float s_key[ORDER_CAP];
    __shared__ uint32_t s_tile[ORDER_CAP];
    const uint64_t g = blockIdx.x;
    const uint64_t g0 = g * (QT * TILE), gcount = n - g0 < (uint64_t)(QT * TILE) ? n - g0 : (uint64_t)(QT * TILE);
    const uint32_t t0 = tb[g], t1 = te[g], cnt = t1 - t0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (cnt > (uint32_t)ORDER_CAP) {  // ascending from the group's own tile, wrapping round
        const uint32_t own = (uint32_t)(g0 / TILE);
        const uint32_t first = own >= t0 && own < t1 ? own : t0;
        for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) {
            uint32_t t = first + k;
            if (t >= t1) t -= cnt;
            out[rptr[g] + k] = make_uint2(t, 1u);
        }
        return;
    }
    for (uint32_t j = wid; j < d; j += nw) {
        float acc = 0.0f;
        for (uint64_t t = lane; t < gcount; t += 32) acc += Xs[(g0 + t) * d + j];
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
        if (lane == 0) s_c[j] = acc / (float)gcount;
    }
    __syncthreads();
    uint32_t P = 1;
    while (P < cnt) P <<= 1;
    for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) {
        float key = INFINITY;
        uint32_t t = 0xFFFFFFFFu;
        if (k < cnt) {
            t = t0 + k;
            const float* m = fcent + (uint64_t)tile_cell[t] * d;
            key = 0.0f;
            for (uint32_t j = 0; j < d; ++j) {
                const float df = s_c[j] - m[j];
                key = __fmaf_rn(df, df, key);
            }
        }
        s_key[k] = key;
        s_tile[k] = t;
    }
    __syncthreads();
    // bitonic sort of (key, tile) ascending
    for (uint32_t size = 2; size <= P; size <<= 1)
        for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) {
                const uint32_t o = k ^ stride;
                if (o > k) {
                    const bool up = (k & size) == 0;
                    const float ka = s_key[k], kb = s_key[o];
                    const uint32_t ta = s_tile[k], tb2 = s_tile[o];
                    const bool gt = ka > kb || (ka == kb && ta > tb2);
                    if (gt == up) {
                        s_key[k] = kb;
                        s_key[o] = ka;
                        s_tile[k] = tb2;
                        s_tile[o] = ta;
                    }
                }
            }
            __syncthreads();
        }
    for (uint32_t k = threadIdx.x; k < cnt; k += blockDim.x) out[rptr[g] + k] = make_uint2(s_tile[k], 1u);
}

__global__ void k_u64_to_u32(const uint64_t* __restrict__ in, uint64_t n, uint32_t* out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)in[i];
}

// The pass-2 tile ranges of every group (a thread per group) from its cell
// bitmap: each run of consecutive set cells is a run of adjacent points
// [cstart[first], cstart[last + 1]); those become tile ranges, merged where
// they touch or overlap.
// Without rptr it counts the ranges into cnt; with it, it writes them from
// rptr[g] and adds the group's tile count to *tiles.
__global__ void k_group_ranges(const unsigned* __restrict__ gcell, uint32_t cwords, uint32_t F,
                               const uint64_t* __restrict__ cstart, uint64_t ngroups,
                               const uint32_t* __restrict__ rptr, uint64_t* cnt, uint2* rngs,
                               unsigned long long* tiles) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < ngroups;
         g += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned* bits = gcell + g * cwords;
        uint64_t cur_b = 0, cur_e = 0, sum = 0;
        bool open = false;
        uint32_t k = 0, out = rptr ? rptr[g] : 0;
        auto emit = [&](uint64_t b, uint64_t e) {
            if (rptr) rngs[out + k] = make_uint2((uint32_t)b, (uint32_t)(e - b));
            sum += e - b;
            ++k;
        };
        uint32_t f = 0;
        while (f < F) {
            const unsigned m = bits[f / 32] >> (f % 32);
            if (m == 0) {  // no set bit left in this word
                f = (f / 32 + 1) * 32;
                continue;
            }
            f += (uint32_t)(__ffs(m) - 1);
            const uint32_t run0 = f;
            while (f < F) {
                const uint32_t avail = 32 - f % 32;
                const unsigned zeros = ~bits[f / 32] >> (f % 32);  // first clear bit at or after f
                if (zeros == 0) {
                    f += avail;
                    continue;
                }
                f += (uint32_t)(__ffs(zeros) - 1);
                break;
            }
            const uint32_t run1 = f < F ? f : F;
            const uint64_t pb = cstart[run0], pe = cstart[run1];
            if (pe <= pb) continue;
            const uint64_t tb = pb / TILE, te = (pe + TILE - 1) / TILE;
            if (open && tb <= cur_e) {
                cur_e = cur_e > te ? cur_e : te;
            } else {
                if (open) emit(cur_b, cur_e);
                cur_b = tb;
                cur_e = te;
                open = true;
            }
        }
        if (open) emit(cur_b, cur_e);
        if (rptr) atomicAdd(tiles, (unsigned long long)sum);
        else cnt[g] = k;
    }
}

// The pass-2 score bound of every query (row r of the pass-2 order is the
// sorted query ord[r]). Scores are |y|^2 - 2 x.y from BF16 operands with FP32
// accumulation. A point that can reach the final list has an FP32 distance of
// at most d21 (the query's (k+1)-th FP32 distance from pass 1), so |y| <= Y =
// |x| + sqrt(d21), and its score lies within 2^-6 (1 + 2^-6) |x| Y + 2^-14 Y^2
// of d^2 - |x|^2. The terms: the BF16 roundings of x and y (unit roundoff
// u = 2^-8 each) move 2 x.y by at most (4u + 2u^2) |x| |y| (Cauchy-Schwarz
// over the products); the FP32 norm split into two BF16 terms and up to 64
// FP32 accumulations add under 2^-15 (|x| |y| + |y|^2). 2^-16 (d21 + |x|^2)
// covers the FP32 distances and norm; the sum is rounded up.
__global__ void k_pass2_cap(const float* __restrict__ Xs, uint64_t n, uint32_t d, const uint32_t* __restrict__ ord,
                            const uint32_t* __restrict__ perm, const float* __restrict__ d21, uint32_t k1,
                            float* __restrict__ cap) {
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t sq = ord[r];
        const float* x = Xs + sq * d;
        float nx2 = 0.0f;
        for (uint32_t t = 0; t < d; ++t) nx2 = __fmaf_rn(x[t], x[t], nx2);
        const float dk = d21[(uint64_t)perm[sq] * k1 + k1 - 1];
        if (!(dk < INFINITY)) {
            cap[r] = INFINITY;
            continue;
        }
        const double nx = sqrt((double)nx2), Y = nx + sqrt((double)dk);
        const double margin = ldexp(nx * Y, -6) * (1.0 + 0x1.0p-6) + ldexp(Y * Y, -14) +
                              ldexp((double)dk + (double)nx2, -16);
        cap[r] = __double2float_ru((double)dk - (double)nx2 + 1.01 * margin);
    }
}

// The exact re-rank on the cluster-sorted copy Xs (the same FP32 values as X,
// so the same distances): row r is the sorted query ord[r] (ord nullable:
// r itself), candidates are sorted positions, ties are broken on original ids
// exactly as k_knn_rerank, and the lists land in the original query's row.
__global__ void k_knn_rerank_sorted(const float* __restrict__ Xs, uint64_t n, uint32_t d, uint32_t k,
                                    const uint32_t* __restrict__ ord, const uint32_t* __restrict__ perm,
                                    const uint32_t* __restrict__ cand_idx, uint32_t* __restrict__ out_idx,
                                    float* __restrict__ out_d2) {
    const unsigned lane = threadIdx.x & 31u;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t r = warp; r < n; r += nwarps) {
        const uint64_t sq = ord ? ord[r] : r;
        const uint32_t q = perm[sq];
        auto key = [&](uint32_t js) -> uint64_t {
            if (js >= n) return ~0ull;
            const float* a = Xs + sq * d;
            const float* b = Xs + (uint64_t)js * d;
            float acc = 0.0f;
            for (uint32_t t = 0; t < d; ++t) {
                const float diff = __fsub_rn(a[t], b[t]);
                acc = __fmaf_rn(diff, diff, acc);
            }
            const uint32_t j = perm[js];
            return ((uint64_t)__float_as_uint(acc) << 32) | (j == q ? 0u : j + 1u);
        };
        uint64_t ka = warp_sort32(key(cand_idx[r * RTOTAL + lane]));
        uint64_t kb = warp_sort32(key(cand_idx[r * RTOTAL + 32 + lane]));
        const uint64_t kbr = __shfl_sync(0xFFFFFFFFu, kb, 31 - lane);
        uint64_t kk = ka < kbr ? ka : kbr;  // the 32 smallest, as a bitonic sequence
        for (int stride = 16; stride > 0; stride >>= 1) {
            const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, kk, stride);
            kk = (lane & stride) == 0 ? (kk < other ? kk : other) : (kk < other ? other : kk);
        }
        if (lane <= k) {
            const uint32_t tag = (uint32_t)kk;
            const uint32_t idx = (kk == ~0ull) ? 0xFFFFFFFFu : (tag == 0 ? q : tag - 1u);
            out_idx[(uint64_t)q * (k + 1) + lane] = idx;
            out_d2[(uint64_t)q * (k + 1) + lane] = kk == ~0ull ? INFINITY : __uint_as_float((uint32_t)(kk >> 32));
        }
    }
}

void knn_check(uint64_t n, uint64_t d, uint64_t k, const sc_knn_opts& opts) {
    if (d == 0 || d > 62) fail(SC_E_UNSUPPORTED, "kNN supports 1..62 dimensions, got %llu", (unsigned long long)d);
    if (k + 1 > 32) fail(SC_E_UNSUPPORTED, "kNN supports k <= 31");
    if (n >= 0xFFFFFFFFull) fail(SC_E_TOO_MANY_NODES, "too many points");
    if (opts.precision != SC_KNN_FP32 && opts.precision != SC_KNN_BF16 && opts.precision != SC_KNN_FP8)
        fail(SC_E_INVALID_ARGUMENT, "unknown kNN precision %d", opts.precision);
    if (opts.precision == SC_KNN_FP8 && d > 61)
        fail(SC_E_UNSUPPORTED, "the FP8 contraction supports 1..61 dimensions, got %llu", (unsigned long long)d);
}

constexpr uint64_t PRUNE_MIN_POINTS = 65536;

uint32_t prune_clusters(const Ctx& c, uint64_t n) {
    if (c.knn_clusters == 1 || n < PRUNE_MIN_POINTS) return 0;
    if (c.knn_clusters) return std::min<uint32_t>(c.knn_clusters, 256);
    // more clusters bound tighter (measured on 4M points x 30: 16% of the tiles
    // scanned with 256 clusters, 45% with 32); about 8192 points per cluster
    return (uint32_t)std::min<uint64_t>(256, std::max<uint64_t>(16, n / 8192));
}

// BF16 or FP8 operands of the points X (rows = queries = candidates).
struct TcOperands {
    DBuf<uint8_t> A, B;
    CUtensorMap ta{}, tb{};
    int kind = 0;  // 0: BF16 KA = 32, 1: BF16 KA = 64, 2: e4m3
};

void prep_operands(Ctx& c, const float* dX, uint64_t n, uint32_t d, int precision, TcOperands& op) {
    if (precision == SC_KNN_FP8) {
        op.kind = 2;
        op.A.alloc(c, n * 64);
        op.B.alloc(c, n * 64);
        DBuf<unsigned> mx(c, 2);
        zero(c, mx.get(), 2);
        k_knn_scales<<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, mx.get(), mx.get() + 1);
        k_knn_prep_f8<<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, mx.get(), mx.get() + 1, op.A.get(),
                                                              op.B.get());
        SC_LAUNCH_CHECK();
        c.launches += 2;
        op.ta = make_map(op.A.get(), n, 64, true);
        op.tb = make_map(op.B.get(), n, 64, true);
        return;
    }
    const uint32_t KA = d <= 30 ? 32 : 64;
    op.kind = KA == 32 ? 0 : 1;
    op.A.alloc(c, n * KA * 2);
    op.B.alloc(c, n * KA * 2);
    __nv_bfloat16* A = (__nv_bfloat16*)op.A.get();
    __nv_bfloat16* B = (__nv_bfloat16*)op.B.get();
    if (KA == 32) k_knn_prep<32><<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, A, B);
    else k_knn_prep<64><<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, A, B);
    SC_LAUNCH_CHECK();
    c.launches++;
    op.ta = make_map(A, n, KA * 2, false);
    op.tb = make_map(B, n, KA * 2, false);
}

// few: keep PASS1_CAND candidates per (query, half) instead of RCAND (BF16;
// for a pass whose lists only bound the (k+1)-th distance).
constexpr int PASS1_CAND = 16;
void launch_operands(Ctx& c, const TcOperands& op, uint64_t n, float* cscore, uint32_t* cidx, const TileLists& tl,
                     bool few = false) {
    if (op.kind == 2) launch_tc<32, true>(c, op.ta, op.tb, n, n, cscore, cidx, tl);
    else if (op.kind == 0 && few) launch_tc<32, false, PASS1_CAND>(c, op.ta, op.tb, n, n, cscore, cidx, tl);
    else if (op.kind == 0) launch_tc<32, false>(c, op.ta, op.tb, n, n, cscore, cidx, tl);
    else if (few) launch_tc<64, false, PASS1_CAND>(c, op.ta, op.tb, n, n, cscore, cidx, tl);
    else launch_tc<64, false>(c, op.ta, op.tb, n, n, cscore, cidx, tl);
}

// The exact k+1 nearest points of every point by the pruned search (see
// "exact pruning" above); the same lists as the full scan.
// Device time between events recorded on the context's stream.
struct StageTimer {
    Ctx& c;
    std::vector<cudaEvent_t> ev;
    explicit StageTimer(Ctx& ctx) : c(ctx) {}
    ~StageTimer() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    void mark() {
        cudaEvent_t e;
        SC_CUDA(cudaEventCreate(&e));
        ev.push_back(e);
        SC_CUDA(cudaEventRecord(e, c.stream));
    }
    double ms(size_t a, size_t b) {
        SC_CUDA(cudaEventSynchronize(ev[b]));
        float t = 0.0f;
        SC_CUDA(cudaEventElapsedTime(&t, ev[a], ev[b]));
        return t;
    }
};

void knn_search_pruned(Ctx& c, const float* dX, uint64_t n, uint32_t d, uint32_t k, int precision, uint32_t K,
                       uint32_t* idx, float* d2) {
    const uint32_t k1 = k + 1;
    static const bool trace = std::getenv("SC_TRACE") != nullptr;
    StageTimer tm(c);
    tm.mark();
    // 1. deterministic k-means: K centroids from evenly spaced points, KM_ITERS Lloyd steps
    DBuf<unsigned> mx(c, 2);
    zero(c, mx.get(), 2);
    k_knn_scales<<<grid_for(n, 256), 256, 0, c.stream>>>(dX, n, d, mx.get(), mx.get() + 1);
    SC_LAUNCH_CHECK();
    c.launches++;
    unsigned hmx[2];
    d2h(c, hmx, mx.get(), 2);
    DBuf<float> cent(c, (uint64_t)K * d);
    sync(c);
    float maxabs, maxnorm;
    std::memcpy(&maxabs, &hmx[0], 4);
    std::memcpy(&maxnorm, &hmx[1], 4);
    // sums of n coordinates of magnitude <= maxabs stay below 2^62 in fixed point
    const double span = std::max(1e-30, (double)maxabs * (double)n);
    const int e = std::min(40, (int)std::floor(62.0 - std::log2(span)) - 1);
    const double scale = std::ldexp(1.0, e), inv_scale = std::ldexp(1.0, -e);
    // Lloyd steps on an evenly spaced sample of the points (a few hundred per
    // centroid is plenty for bounds that hold whatever the clusters), then one
    // assignment of every point
    const uint64_t ns = std::min<uint64_t>(n, (uint64_t)KM_SAMPLE);
    std::vector<uint32_t> srows(ns);
    for (uint64_t i = 0; i < ns; ++i) srows[i] = (uint32_t)(i * n / ns);
    DBuf<uint32_t> d_srows(c, ns);
    DBuf<float> Xsub(c, ns * d);
    h2d(c, d_srows.get(), srows.data(), ns);
    k_gather_rows<<<grid_for(ns * d, 256), 256, 0, c.stream>>>(dX, d_srows.get(), ns, d, Xsub.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    {
        // farthest-point seeds: the first sample point, then the farthest from all chosen so far
        DBuf<float> d2min(c, ns);
        SC_CUDA(cudaMemsetAsync(d2min.get(), 0x7F, ns * sizeof(float), c.stream));  // a huge finite value
        d2d(c, cent.get(), Xsub.get(), d);
        for (uint32_t t = 1; t < K; ++t) {
            k_seed_update<<<grid_for(ns, 256), 256, 0, c.stream>>>(Xsub.get(), ns, d, cent.get() + (uint64_t)(t - 1) * d,
                                                                   d2min.get());
            k_seed_pick<<<1, 1024, 0, c.stream>>>(Xsub.get(), ns, d, d2min.get(), cent.get(), t);
        }
        SC_LAUNCH_CHECK();
        c.launches += 2 * (K - 1);
    }
    DBuf<uint32_t> assign(c, n);
    DBuf<unsigned long long> sums(c, (uint64_t)K * d);
    DBuf<unsigned> cnt(c, K);
    const size_t sm_assign = (size_t)K * ((d + 3) & ~3u) * 4, sm_accum = (size_t)K * d * 8 + (size_t)K * 4;
    SC_CUDA(cudaFuncSetAttribute(k_km_assign, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_assign));
    SC_CUDA(cudaFuncSetAttribute(k_km_accum, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_accum));
    for (int it = 0; it < KM_ITERS; ++it) {
        k_km_assign<<<grid_for(ns, 256, (unsigned)c.sm_count * 4), 256, sm_assign, c.stream>>>(
            Xsub.get(), ns, d, cent.get(), K, assign.get());
        zero(c, sums.get(), (uint64_t)K * d);
        zero(c, cnt.get(), K);
        k_km_accum<<<grid_for(ns, 256, (unsigned)c.sm_count), 256, sm_accum, c.stream>>>(
            Xsub.get(), ns, d, assign.get(), K, scale, sums.get(), cnt.get());
        k_km_update<<<grid_for((uint64_t)K * d, 256), 256, 0, c.stream>>>(sums.get(), cnt.get(), K, d, inv_scale,
                                                                         cent.get());
        SC_LAUNCH_CHECK();
        c.launches += 3;
    }
    k_km_assign<<<grid_for(n, 256, (unsigned)c.sm_count * 4), 256, sm_assign, c.stream>>>(dX, n, d, cent.get(), K,
                                                                                          assign.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    Xsub.release();
    tm.mark();  // 1: k-means
    // 2. points sorted by cluster (stable: ascending point id inside a cluster)
    DBuf<uint32_t> iota(c, n), cl_s(c, n), perm0(c, n);
    k_iota_u32<<<grid_for(n, 256), 256, 0, c.stream>>>(iota.get(), n);
    SC_LAUNCH_CHECK();
    c.launches++;
    sort_pairs(c, assign.get(), cl_s.get(), iota.get(), perm0.get(), n, bits_for(K - 1));
    assign.release();
    iota.release();
    DBuf<float> Xs(c, n * d);
    k_gather_rows<<<grid_for(n * d, 256), 256, 0, c.stream>>>(dX, perm0.get(), n, d, Xs.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    std::vector<uint32_t> h_cl(n);
    std::vector<float> h_cent((uint64_t)K * d);
    d2h(c, h_cl.data(), cl_s.get(), n);
    d2h(c, h_cent.data(), cent.get(), (uint64_t)K * d);
    sync(c);
    std::vector<uint64_t> start(K + 1, 0);
    for (uint64_t i = 0; i < n; ++i) start[h_cl[i] + 1]++;
    for (uint32_t q = 0; q < K; ++q) start[q + 1] += start[q];
    // 3. fine cells inside every cluster, then the final order: (cluster, cell)
    std::vector<uint32_t> fbase(K + 1, 0);
    for (uint32_t q = 0; q < K; ++q) fbase[q + 1] = fbase[q] + (uint32_t)((start[q + 1] - start[q] + FINE - 1) / FINE);
    DBuf<uint64_t> d_start(c, K + 1);
    DBuf<uint32_t> d_fbase(c, K + 1), fine(c, n), fine_s(c, n), perm(c, n);
    h2d(c, d_start.get(), start.data(), K + 1);
    h2d(c, d_fbase.get(), fbase.data(), K + 1);
    k_fine_assign<<<grid_for(n, 256), 256, 0, c.stream>>>(Xs.get(), n, d, cl_s.get(), d_start.get(), d_fbase.get(),
                                                           fine.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    // each cell's centre: the sample point that defined it (read before Xs is re-sorted)
    const uint32_t F = fbase[K];
    std::vector<uint32_t> cell_rows(F);
    for (uint32_t q = 0; q < K; ++q)
        for (uint32_t j = 0; j < fbase[q + 1] - fbase[q]; ++j) cell_rows[fbase[q] + j] = (uint32_t)(start[q] + (uint64_t)j * FINE);
    DBuf<uint32_t> d_cell_rows(c, std::max<uint32_t>(F, 1));
    DBuf<float> fcent(c, (uint64_t)std::max<uint32_t>(F, 1) * d);
    h2d(c, d_cell_rows.get(), cell_rows.data(), F);
    k_gather_rows<<<grid_for((uint64_t)F * d, 256), 256, 0, c.stream>>>(Xs.get(), d_cell_rows.get(), F, d, fcent.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    sort_pairs(c, fine.get(), fine_s.get(), perm0.get(), perm.get(), n, bits_for(std::max<uint32_t>(F, 2) - 1));
    fine.release();
    perm0.release();
    k_gather_rows<<<grid_for(n * d, 256), 256, 0, c.stream>>>(dX, perm.get(), n, d, Xs.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    // each cell's points (contiguous in the final order) and radius around its centre
    DBuf<unsigned> ccnt(c, std::max<uint32_t>(F, 1)), crad(c, std::max<uint32_t>(F, 1));
    zero(c, ccnt.get(), F);
    zero(c, crad.get(), F);
    k_cell_count<<<grid_for(n, 256), 256, 0, c.stream>>>(fine_s.get(), n, ccnt.get());
    k_cell_radius<<<grid_for(n, 256), 256, 0, c.stream>>>(Xs.get(), n, d, fine_s.get(), fcent.get(), crad.get());
    SC_LAUNCH_CHECK();
    c.launches += 2;
    std::vector<unsigned> h_ccnt(F);
    d2h(c, h_ccnt.data(), ccnt.get(), F);
    sync(c);
    fine_s.release();
    std::vector<uint64_t> cstart(F + 1, 0);
    for (uint32_t f = 0; f < F; ++f) cstart[f + 1] = cstart[f] + h_ccnt[f];
    tm.mark();  // 2: sorted by cluster and cell
    // 4. cluster extents: radius, and [lo, hi] along every direction between centres
    std::vector<float> Ua((uint64_t)K * K * d, 0.0f), Ub((uint64_t)K * K * d, 0.0f);
    for (uint32_t qa = 0; qa < K; ++qa)
        for (uint32_t qb = 0; qb < K; ++qb) {
            double nrm = 0.0;
            for (uint32_t j = 0; j < d; ++j) {
                const double t = (double)h_cent[qb * d + j] - (double)h_cent[qa * d + j];
                nrm += t * t;
            }
            nrm = std::sqrt(nrm);
            if (qa == qb || nrm == 0.0) continue;  // a zero direction bounds nothing
            for (uint32_t j = 0; j < d; ++j) {
                const float u = (float)(((double)h_cent[qb * d + j] - (double)h_cent[qa * d + j]) / nrm);
                Ua[((uint64_t)qa * K + qb) * d + j] = u;
                Ub[((uint64_t)qb * K + qa) * d + j] = u;
            }
        }
    DBuf<float> d_Ua(c, (uint64_t)K * K * d), d_Ub(c, (uint64_t)K * K * d);
    h2d(c, d_Ua.get(), Ua.data(), (uint64_t)K * K * d);
    h2d(c, d_Ub.get(), Ub.data(), (uint64_t)K * K * d);
    const uint64_t ngroups = (n + QT * TILE - 1) / (QT * TILE);
    const uint64_t ntiles = (n + TILE - 1) / TILE;
    // chunks: inside one cluster for the extents; inside one cluster and one query group for the bounds
    std::vector<Chunk> ch_ext, ch_need;
    for (uint32_t q = 0; q < K; ++q) {
        for (uint64_t p0 = start[q]; p0 < start[q + 1]; p0 += 2048)
            ch_ext.push_back(Chunk{q, p0, std::min<uint64_t>(start[q + 1], p0 + 2048)});
        for (uint64_t p0 = start[q]; p0 < start[q + 1];) {
            const uint64_t grp_end = (p0 / (QT * TILE) + 1) * (QT * TILE);
            const uint64_t p1 = std::min<uint64_t>(start[q + 1], grp_end);
            ch_need.push_back(Chunk{q, p0, p1});
            p0 = p1;
        }
    }
    DBuf<Chunk> d_ch_ext(c, ch_ext.size()), d_ch_need(c, ch_need.size());
    h2d(c, d_ch_ext.get(), ch_ext.data(), ch_ext.size());
    h2d(c, d_ch_need.get(), ch_need.data(), ch_need.size());
    DBuf<unsigned> rad(c, K), lo(c, (uint64_t)K * K), hi(c, (uint64_t)K * K);
    zero(c, rad.get(), K);
    zero(c, hi.get(), (uint64_t)K * K);
    SC_CUDA(cudaMemsetAsync(lo.get(), 0xFF, (uint64_t)K * K * 4, c.stream));
    const size_t sm_ext = (size_t)K * d * 4 + (size_t)K * 8;
    SC_CUDA(cudaFuncSetAttribute(k_cluster_extent, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_ext));
    k_cluster_extent<<<(unsigned)ch_ext.size(), 256, sm_ext, c.stream>>>(Xs.get(), d, d_ch_ext.get(), cent.get(),
                                                                         d_Ub.get(), K, rad.get(), lo.get(), hi.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    // 5. operands of the sorted points
    TcOperands op;
    prep_operands(c, Xs.get(), n, d, precision, op);
    tm.mark();  // 3: extents and operands
    auto own = [&](uint64_t g, std::vector<std::pair<uint64_t, uint64_t>>& pts) {
        const uint32_t a0 = h_cl[g * QT * TILE], a1 = h_cl[std::min<uint64_t>(n, (g + 1) * QT * TILE) - 1];
        pts.emplace_back(start[a0], start[a1 + 1]);
        return std::make_pair(a0, a1);
    };
    DBuf<float> cscore(c, n * RTOTAL);
    DBuf<uint32_t> cidx(c, n * RTOTAL);
    // queries in the order `ord` (nullable: the sorted order), operand `o`
    // a scan and its re-rank, the tile lists on the device
    auto run_pass_dev = [&](const TcOperands& o, const uint32_t* ord, const uint32_t* d_rptr, const uint2* d_rngs,
                            uint32_t* out_idx, float* out_d2, const float* qcap, bool few) {
        launch_operands(c, o, n, cscore.get(), cidx.get(), TileLists{d_rptr, d_rngs, qcap}, few);
        k_knn_rerank_sorted<<<grid_for(n * 32, 256), 256, 0, c.stream>>>(Xs.get(), n, d, k, ord, perm.get(),
                                                                        cidx.get(), out_idx, out_d2);
        SC_LAUNCH_CHECK();
        c.launches++;
    };
    // 6. pass 1: every query group against its own clusters, nearest cells first
    // (k_order_tiles: the rows' thresholds tighten within the first tiles, so
    // fewer later scores take the insertion path; pass 1 only yields the
    // bounds of pass 2)
    std::vector<uint32_t> rptr(ngroups + 1, 0);
    uint64_t tiles1 = 0;
    DBuf<uint32_t> idx1(c, n * k1);
    DBuf<float> d21(c, n * k1);
    {
        std::vector<uint32_t> h_tb(ngroups), h_te(ngroups);
        std::vector<std::pair<uint64_t, uint64_t>> pts;
        for (uint64_t g = 0; g < ngroups; ++g) {
            pts.clear();
            own(g, pts);
            h_tb[g] = (uint32_t)(pts[0].first / TILE);
            h_te[g] = (uint32_t)((pts[0].second + TILE - 1) / TILE);
            tiles1 += h_te[g] - h_tb[g];
            if (tiles1 > 0xFFFFFFFFull)
                fail(SC_E_UNSUPPORTED, "pruned kNN lists exceed 2^32 tiles: use more clusters or the full scan");
            rptr[g + 1] = (uint32_t)tiles1;
        }
        std::vector<uint32_t> tile_cell(ntiles);
        for (uint64_t t = 0, f = 0; t < ntiles; ++t) {
            while (f + 1 < F && cstart[f + 1] <= t * TILE) ++f;
            tile_cell[t] = (uint32_t)f;
        }
        DBuf<uint32_t> d_tb(c, ngroups), d_te(c, ngroups), d_tc(c, ntiles), d_rp(c, ngroups + 1);
        DBuf<uint2> d_rg(c, std::max<uint64_t>(tiles1, 1));
        h2d(c, d_tb.get(), h_tb.data(), ngroups);
        h2d(c, d_te.get(), h_te.data(), ngroups);
        h2d(c, d_tc.get(), tile_cell.data(), ntiles);
        h2d(c, d_rp.get(), rptr.data(), ngroups + 1);
        k_order_tiles<<<(unsigned)ngroups, 256, 0, c.stream>>>(Xs.get(), n, d, d_tb.get(), d_te.get(), d_tc.get(),
                                                               fcent.get(), d_rp.get(), d_rg.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        // pass 1 only bounds the (k+1)-th distance: fewer kept candidates suffice
        // (any k + 1 real points give a bound; 2 x PASS1_CAND of them are kept)
        run_pass_dev(op, nullptr, d_rp.get(), d_rg.get(), idx1.get(), d21.get(), nullptr,
                     2 * PASS1_CAND >= (int)k1 + 8);
        sync(c);  // the host arrays above must outlive the copies
    }
    tm.mark();  // 4: pass 1
    // 7. the clusters every group still needs
    const uint32_t words = (K + 63) / 64;
    DBuf<unsigned long long> mask(c, n * words);
    // rounding of an FP32 projection, distance or radius: a few ulps of the
    // largest coordinate norm times d
    const float R = std::sqrt(std::max(maxnorm, 0.0f)) + 1.0f;
    const float eps = 8.0f * (float)d * std::ldexp(1.0f, -24) * 2.0f * R;
    tm.mark();  // 5: bounds begin (after pass 1)
    const size_t sm_need = (size_t)K * d * 8 + (size_t)K * 12;
    SC_CUDA(cudaFuncSetAttribute(k_cluster_needs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_need));
    k_cluster_needs<<<(unsigned)ch_need.size(), QT * TILE, sm_need, c.stream>>>(
        Xs.get(), d, d_ch_need.get(), perm.get(), d21.get(), k1, cent.get(), rad.get(), d_Ua.get(), lo.get(), hi.get(),
        K, eps, words, mask.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    // pass-2 order: by own cluster, then by need set; groups of 256 in that order
    DBuf<unsigned long long> nkeys(c, n), nkeys_s(c, n);
    DBuf<uint32_t> npos(c, n), ord(c, n);
    k_need_keys<<<grid_for(n, 256), 256, 0, c.stream>>>(mask.get(), cl_s.get(), n, words, nkeys.get(), npos.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    tm.mark();  // 6: cluster needs done
    sort_pairs(c, nkeys.get(), nkeys_s.get(), npos.get(), ord.get(), n, 32 + bits_for(K - 1));
    nkeys.release();
    nkeys_s.release();
    npos.release();
    DBuf<unsigned long long> gmask(c, ngroups * words);
    DBuf<uint32_t> gown(c, ngroups * 2);
    k_group_needs<<<grid_for(ngroups * 32, 256), 256, 0, c.stream>>>(mask.get(), ord.get(), cl_s.get(), n, words,
                                                                   ngroups, gmask.get(), gown.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    // the cells each group scans: those of its candidate clusters a query cannot exclude
    tm.mark();  // 7: order and group needs done
    const uint32_t cwords = (F + 31) / 32;
    DBuf<unsigned> gcell(c, ngroups * cwords);
    zero(c, gcell.get(), ngroups * cwords);
    SC_CUDA(cudaFuncSetAttribute(k_group_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(cwords * 8)));
    k_group_cells<<<(unsigned)ngroups, QT * TILE, cwords * 8, c.stream>>>(Xs.get(), n, d, ord.get(), perm.get(), d21.get(), k1,
                                                                gmask.get(), gown.get(), words, K, d_fbase.get(),
                                                                fcent.get(), crad.get(), eps, cwords, mask.get(),
                                                                cl_s.get(), gcell.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    tm.mark();  // 8: group cells done
    // the query operand in pass-2 order
    TcOperands op2;
    {
        const uint32_t row_bytes = op.kind == 1 ? 128u : 64u;
        op2.kind = op.kind;
        op2.A.alloc(c, n * row_bytes);
        k_gather_operand_rows<<<grid_for(n * row_bytes / 16, 256), 256, 0, c.stream>>>(
            (const uint4*)op.A.get(), ord.get(), n, row_bytes / 16, (uint4*)op2.A.get());
        SC_LAUNCH_CHECK();
        c.launches++;
        op2.ta = make_map(op2.A.get(), n, row_bytes, op.kind == 2);
        op2.tb = op.tb;
    }
    // score bounds of the BF16 search from the pass-1 distances (FP8 scores
    // carry too coarse an error for a useful bound: none)
    DBuf<float> qcap;
    if (op.kind != 2) {
        qcap.alloc(c, n);
        k_pass2_cap<<<grid_for(n, 256), 256, 0, c.stream>>>(Xs.get(), n, d, ord.get(), perm.get(), d21.get(), k1,
                                                            qcap.get());
        SC_LAUNCH_CHECK();
        c.launches++;
    }
    sync(c);
    tm.mark();  // 9: bounds
    idx1.release();
    d21.release();
    mask.release();
    // 8. pass 2: every cell a query of the group cannot exclude (cells in point
    // order), the tile lists built on the device from the cell bitmaps
    DBuf<uint64_t> d_cstart(c, F + 1);
    h2d(c, d_cstart.get(), cstart.data(), F + 1);
    DBuf<uint64_t> gcnt(c, ngroups + 1), r64(c, ngroups + 1);
    DBuf<uint32_t> d_rptr2(c, ngroups + 1);
    zero(c, gcnt.get(), ngroups + 1);
    DBuf<unsigned long long> d_tiles2(c, 1);
    zero(c, d_tiles2.get(), 1);
    k_group_ranges<<<grid_for(ngroups, 128), 128, 0, c.stream>>>(gcell.get(), cwords, F, d_cstart.get(), ngroups,
                                                                 nullptr, gcnt.get(), nullptr, nullptr);
    exclusive_sum(c, gcnt.get(), r64.get(), ngroups + 1);
    const uint64_t nranges = to_host(c, r64.get() + ngroups);
    if (nranges > 0xFFFFFFFFull)
        fail(SC_E_UNSUPPORTED, "pruned kNN lists exceed 2^32 ranges: use more clusters or the full scan");
    k_u64_to_u32<<<grid_for(ngroups + 1, 256), 256, 0, c.stream>>>(r64.get(), ngroups + 1, d_rptr2.get());
    DBuf<uint2> d_rngs2(c, std::max<uint64_t>(nranges, 1));
    k_group_ranges<<<grid_for(ngroups, 128), 128, 0, c.stream>>>(gcell.get(), cwords, F, d_cstart.get(), ngroups,
                                                                 d_rptr2.get(), nullptr, d_rngs2.get(),
                                                                 d_tiles2.get());
    SC_LAUNCH_CHECK();
    c.launches += 3;
    const uint64_t tiles2 = to_host(c, d_tiles2.get());
    tm.mark();  // 10: lists built
    run_pass_dev(op2, ord.get(), d_rptr2.get(), d_rngs2.get(), idx, d2, qcap.get(), false);
    tm.mark();  // 11: pass 2
    c.knn_stats.ms_cluster = tm.ms(0, 3);
    c.knn_stats.ms_pass1 = tm.ms(3, 4);
    c.knn_stats.ms_bounds = tm.ms(4, 10);
    c.knn_stats.ms_pass2 = tm.ms(10, 11);
    c.knn_stats.clusters = K;
    c.knn_stats.tiles_scanned = tiles1 + tiles2;
    c.knn_stats.tiles_pass1 = tiles1;
    c.knn_stats.tiles_full = ngroups * ntiles;
    if (trace)
        std::fprintf(stderr,
                     "[sc] knn pruned n=%llu K=%u cells=%u: k-means %.1f ms, sort %.1f ms, extents %.1f ms, pass1 "
                     "%.1f ms (%.2f%% of tiles), needs %.1f ms, order %.1f ms, cells %.1f ms, copy %.1f ms, lists "
                     "%.1f ms, pass2 %.1f ms (%.2f%%)\n",
                     (unsigned long long)n, K, F, tm.ms(0, 1), tm.ms(1, 2), tm.ms(2, 3), tm.ms(3, 4),
                     100.0 * tiles1 / (double)(ngroups * ntiles), tm.ms(5, 6), tm.ms(6, 7), tm.ms(7, 8),
                     tm.ms(8, 9), tm.ms(9, 10), tm.ms(10, 11), 100.0 * tiles2 / (double)(ngroups * ntiles));
}

// Exact (brute-force) k+1 nearest points of the queries q0 .. q0 + nq - 1
// among all n points of the device array dX: 64 candidates per query (the 32
// best of each half of the candidate columns) from the BF16 or FP8 tensor-core
// scores, or the 32 best exact FP32 distances from the CUDA cores, ranked
// exactly in FP32. idx/d2 are nq x (k+1), self first, then ascending squared
// distance, ties by lower index.
void knn_search_device(Ctx& c, const float* dX, uint64_t n, uint64_t d, uint64_t k, uint64_t q0, uint64_t nq,
                       int precision, uint32_t* idx, float* d2) {
    c.knn_stats = sc_knn_stats{};
    if (!nq) return;
    if (precision != SC_KNN_FP32 && q0 == 0 && nq == n) {
        const uint32_t K = prune_clusters(c, n);
        if (K) {
            knn_search_pruned(c, dX, n, (uint32_t)d, (uint32_t)k, precision, K, idx, d2);
            check_device_status(c);
            return;
        }
    }
    {
        const uint64_t groups = (nq + QT * TILE - 1) / (QT * TILE), tiles = (n + TILE - 1) / TILE;
        c.knn_stats.tiles_scanned = c.knn_stats.tiles_full = groups * tiles;
    }
    DBuf<float> cscore(c, precision == SC_KNN_FP32 ? 0 : nq * RTOTAL);
    DBuf<uint32_t> cidx(c, nq * RTOTAL);
    if (precision == SC_KNN_FP32) {
        if (d <= 32) candidates_fp32<32>(c, dX, n, (uint32_t)d, q0, nq, cidx.get());
        else candidates_fp32<64>(c, dX, n, (uint32_t)d, q0, nq, cidx.get());
    } else if (precision == SC_KNN_FP8) {
        candidates_f8(c, dX, n, (uint32_t)d, q0, nq, cscore.get(), cidx.get());
    } else if (d <= 30) {
        candidates<32>(c, dX, n, (uint32_t)d, q0, nq, cscore.get(), cidx.get());
    } else {
        candidates<64>(c, dX, n, (uint32_t)d, q0, nq, cscore.get(), cidx.get());
    }
    k_knn_rerank<<<grid_for(nq * 32, 256), 256, 0, c.stream>>>(dX, n, (uint32_t)d, (uint32_t)k, q0, nq,
                                                                cidx.get(), idx, d2);
    SC_LAUNCH_CHECK();
    c.launches++;
    check_device_status(c);
}

// Gaussian connectivities (neighborhood/mod.rs:105-163, :480-544) from the
// device k+1 lists of all n points (squared distances): sigma per point,
// weights, symmetrisation, duplicate removal, CSR.
void knn_connectivities_device(Ctx& c, const uint32_t* idx, const float* d2, uint64_t n, uint64_t k,
                               const sc_knn_opts& opts, uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                               uint64_t conn_cap, uint64_t* conn_nnz, DevGraph** graph_out) {
    DBuf<float> sigma(c, n);
    DBuf<unsigned long long> keys(c, 2 * n * k + 1), keys_s(c, 2 * n * k + 1);
    DBuf<float> w(c, 2 * n * k + 1), w_s(c, 2 * n * k + 1);
    DBuf<unsigned long long> cnt(c, 1);
    zero(c, cnt.get(), 1);
    if (n) {
        k_knn_sigma<<<grid_for(n, 256), 256, 0, c.stream>>>(d2, n, (uint32_t)k, opts.sigma == SC_SIGMA_KTH,
                                                            sigma.get());
        k_knn_pairs<<<grid_for(n, 256), 256, 0, c.stream>>>(idx, d2, n, (uint32_t)k, sigma.get(),
                                                            opts.sym == SC_SYM_UNION, opts.squared_kiddo,
                                                            keys.get(), w.get(), cnt.get());
        SC_LAUNCH_CHECK();
        c.launches += 2;
    }
    uint64_t N = to_host(c, cnt.get());
    sort_pairs(c, keys.get(), keys_s.get(), w.get(), w_s.get(), N, 64);
    DBuf<uint8_t> keep(c, N);
    DBuf<unsigned long long> ukeys(c, N);
    DBuf<float> uw(c, N);
    uint64_t M = N;
    if (N) {
        k_dedupe_flags<<<grid_for(N, 256), 256, 0, c.stream>>>(keys_s.get(), N, keep.get());
        c.launches++;
        DBuf<uint64_t> m(c, 1);
        select_flagged(c, keys_s.get(), keep.get(), ukeys.get(), m.get(), N);
        select_flagged(c, w_s.get(), keep.get(), uw.get(), m.get(), N);
        M = to_host(c, m.get());
    }
    DBuf<uint32_t> rows(c, M), cols(c, M);
    DBuf<uint64_t> ptr(c, n + 1);
    if (M) {
        k_split_rowcol<<<grid_for(M, 256), 256, 0, c.stream>>>(ukeys.get(), M, rows.get(), cols.get());
        c.launches++;
    }
    k_ptr_from_rows<<<grid_for(M + 1, 256), 256, 0, c.stream>>>(rows.get(), M, n, ptr.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    if (conn_nnz) *conn_nnz = M;
    if (conn_ptrs) {
        if (M > conn_cap) fail(SC_E_INVALID_ARGUMENT, "conn_capacity %llu < %llu entries",
                               (unsigned long long)conn_cap, (unsigned long long)M);
        d2h(c, conn_ptrs, ptr.get(), n + 1);
        if (conn_nbrs) d2h(c, conn_nbrs, cols.get(), M);
        if (conn_w) d2h(c, conn_w, uw.get(), M);
    }
    if (graph_out) *graph_out = graph_from_csr(c, ptr.get(), n + 1, cols.get(), M, uw.get(), M, nullptr, 0, true);
    sync(c);
}

void copy_lists_out(Ctx& c, const uint32_t* idx, const float* d2, uint64_t rows, uint64_t k, int squared,
                    uint32_t* knn_index, float* knn_dist) {
    if (knn_index) d2h(c, knn_index, idx, rows * (k + 1));
    if (knn_dist) {
        std::vector<float> h(rows * (k + 1));
        d2h(c, h.data(), d2, rows * (k + 1));
        sync(c);
        for (uint64_t i = 0; i < h.size(); ++i) knn_dist[i] = squared ? h[i] : std::sqrt(h[i]);
    }
    sync(c);
}

}  // namespace

// knn_arrayd_* (neighborhood/mod.rs:51-202, :359-578) with exact search.
void knn_gaussian(Ctx& c, const float* X, uint64_t n, uint64_t d, uint64_t k, const sc_knn_opts& opts,
                  uint32_t* knn_index, float* knn_dist, uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                  uint64_t conn_cap, uint64_t* conn_nnz, DevGraph** graph_out) {
    knn_check(n, d, k, opts);
    DBuf<float> dX(c, n * d);
    upload(c, dX.get(), X, n * d * sizeof(float));
    DBuf<uint32_t> idx(c, n * (k + 1));
    DBuf<float> d2(c, n * (k + 1));
    knn_search_device(c, dX.get(), n, d, k, 0, n, opts.precision, idx.get(), d2.get());
    copy_lists_out(c, idx.get(), d2.get(), n, k, opts.squared_kiddo, knn_index, knn_dist);
    if (!conn_ptrs && !graph_out) return;
    knn_connectivities_device(c, idx.get(), d2.get(), n, k, opts, conn_ptrs, conn_nbrs, conn_w, conn_cap, conn_nnz,
                              graph_out);
}

// Times the search of all rows of X under candidate cluster counts (1: the
// full scan) and keeps the fastest on the context. Every candidate returns the
// same lists, so this changes speed only. Returns the number of candidates.
uint32_t knn_autotune(Ctx& c, const float* X, uint64_t n, uint64_t d, uint64_t k, const sc_knn_opts& opts,
                      uint32_t* chosen, double* ms_chosen, double* ms_full) {
    knn_check(n, d, k, opts);
    DBuf<float> dX(c, n * d);
    upload(c, dX.get(), X, n * d * sizeof(float));
    DBuf<uint32_t> idx(c, n * (k + 1));
    DBuf<float> d2(c, n * (k + 1));
    std::vector<uint32_t> cand{1};
    for (uint32_t K : {32u, 64u, 128u, 256u})
        if (n >= PRUNE_MIN_POINTS && (uint64_t)K * 4096 <= n) cand.push_back(K);
    const uint32_t saved = c.knn_clusters;
    double best = INFINITY, full = 0.0;
    uint32_t pick = 1;
    cudaEvent_t e0, e1;
    SC_CUDA(cudaEventCreate(&e0));
    SC_CUDA(cudaEventCreate(&e1));
    try {
        // warm-up: modules, pools, first-call costs
        c.knn_clusters = cand.back();
        knn_search_device(c, dX.get(), n, d, k, 0, n, opts.precision, idx.get(), d2.get());
        for (uint32_t K : cand) {
            c.knn_clusters = K;
            SC_CUDA(cudaEventRecord(e0, c.stream));
            knn_search_device(c, dX.get(), n, d, k, 0, n, opts.precision, idx.get(), d2.get());
            SC_CUDA(cudaEventRecord(e1, c.stream));
            SC_CUDA(cudaEventSynchronize(e1));
            float ms = 0.0f;
            SC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (K == 1) full = ms;
            if (ms < best) {
                best = ms;
                pick = K;
            }
        }
    } catch (...) {
        c.knn_clusters = saved;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c.knn_clusters = pick;
    if (chosen) *chosen = pick;
    if (ms_chosen) *ms_chosen = best;
    if (ms_full) *ms_full = full;
    return (uint32_t)cand.size();
}

// The k+1 lists of the query rows [q0, q1) only (one shard of a multi-GPU
// build); squared FP32 distances.
void knn_search(Ctx& c, const float* X, uint64_t n, uint64_t d, uint64_t k, uint64_t q0, uint64_t q1,
                const sc_knn_opts& opts, uint32_t* knn_index, float* knn_d2) {
    knn_check(n, d, k, opts);
    if (q0 > q1 || q1 > n) fail(SC_E_INVALID_ARGUMENT, "query rows [%llu, %llu) are not inside [0, %llu)",
                                (unsigned long long)q0, (unsigned long long)q1, (unsigned long long)n);
    const uint64_t nq = q1 - q0;
    DBuf<float> dX(c, n * d);
    upload(c, dX.get(), X, n * d * sizeof(float));
    DBuf<uint32_t> idx(c, nq * (k + 1));
    DBuf<float> d2(c, nq * (k + 1));
    knn_search_device(c, dX.get(), n, d, k, q0, nq, opts.precision, idx.get(), d2.get());
    copy_lists_out(c, idx.get(), d2.get(), nq, k, 1, knn_index, knn_d2);
}

// Connectivities from gathered host lists (all n rows, squared distances).
void knn_connectivities(Ctx& c, const uint32_t* knn_index, const float* knn_d2, uint64_t n, uint64_t k,
                        const sc_knn_opts& opts, uint64_t* conn_ptrs, uint32_t* conn_nbrs, float* conn_w,
                        uint64_t conn_cap, uint64_t* conn_nnz, DevGraph** graph_out) {
    if (k + 1 > 32) fail(SC_E_UNSUPPORTED, "kNN supports k <= 31");
    if (n >= 0xFFFFFFFFull) fail(SC_E_TOO_MANY_NODES, "too many points");
    DBuf<uint32_t> idx(c, n * (k + 1));
    DBuf<float> d2(c, n * (k + 1));
    h2d(c, idx.get(), knn_index, n * (k + 1));
    h2d(c, d2.get(), knn_d2, n * (k + 1));
    knn_connectivities_device(c, idx.get(), d2.get(), n, k, opts, conn_ptrs, conn_nbrs, conn_w, conn_cap, conn_nnz,
                              graph_out);
}

}  // namespace sc
