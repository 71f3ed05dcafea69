// sc_prims.cuh — device-wide primitives (stable radix sort, scans, reductions)
// on the context stream. Temporary storage comes from the stream-ordered pool.
#pragma once

#include <cub/cub.cuh>

#include "sc_internal.cuh"

namespace sc {

inline int bits_for(uint64_t max_value) {
    int b = 0;
    while (b < 64 && (max_value >> b) != 0) ++b;
    return b < 1 ? 1 : b;
}

// Stable LSD radix sort of (key, value) pairs on bits [0, end_bit).
template <class K, class V>
void sort_pairs(Ctx& c, const K* kin, K* kout, const V* vin, V* vout, size_t n, int end_bit) {
    if (n == 0) return;
    size_t bytes = 0;
    SC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit,
                                            c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), bytes, kin, kout, vin, vout, n, 0, end_bit,
                                            c.stream));
    c.launches += 4;
}

template <class T>
void exclusive_sum(Ctx& c, const T* in, T* out, size_t n) {
    if (n == 0) return;
    size_t bytes = 0;
    SC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, c.stream));
    c.launches += 2;
}

template <class T>
void inclusive_sum(Ctx& c, const T* in, T* out, size_t n) {
    if (n == 0) return;
    size_t bytes = 0;
    SC_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, in, out, n, c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceScan::InclusiveSum(tmp.get(), bytes, in, out, n, c.stream));
    c.launches += 2;
}

// out[0] = Σ in (device scalar)
template <class T>
void device_sum(Ctx& c, const T* in, T* out, size_t n) {
    size_t bytes = 0;
    SC_CUDA(cub::DeviceReduce::Sum(nullptr, bytes, in, out, n, c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceReduce::Sum(tmp.get(), bytes, in, out, n, c.stream));
    c.launches += 1;
}

template <class T>
void device_max(Ctx& c, const T* in, T* out, size_t n) {
    size_t bytes = 0;
    SC_CUDA(cub::DeviceReduce::Max(nullptr, bytes, in, out, n, c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceReduce::Max(tmp.get(), bytes, in, out, n, c.stream));
    c.launches += 1;
}

template <class T>
void device_min(Ctx& c, const T* in, T* out, size_t n) {
    size_t bytes = 0;
    SC_CUDA(cub::DeviceReduce::Min(nullptr, bytes, in, out, n, c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceReduce::Min(tmp.get(), bytes, in, out, n, c.stream));
    c.launches += 1;
}

// Stable compaction of `in` where flags != 0; *d_count receives the kept count.
template <class T, class F>
void select_flagged(Ctx& c, const T* in, const F* flags, T* out, uint64_t* d_count, size_t n) {
    size_t bytes = 0;
    SC_CUDA(cub::DeviceSelect::Flagged(nullptr, bytes, in, flags, out, d_count, n, c.stream));
    DBuf<uint8_t> tmp(c, bytes);
    SC_CUDA(cub::DeviceSelect::Flagged(tmp.get(), bytes, in, flags, out, d_count, n, c.stream));
    c.launches += 2;
}

// Small device->host reads through the context's pinned mailbox: get() queues
// an asynchronous copy and returns where its result will be; wait() completes
// every copy queued so far with one synchronisation of the context's stream.
// Results are valid until the next Mailbox of the same context is used.
struct Mailbox {
    Ctx& c;
    size_t off = 0;
    explicit Mailbox(Ctx& ctx) : c(ctx) {}
    template <class T>
    const T* get(const T* d, size_t n) {
        off = (off + 15) & ~size_t(15);
        if (off + n * sizeof(T) > MAILBOX_BYTES) fail(SC_E_INTERNAL, "mailbox overflow (%zu bytes)", off + n * sizeof(T));
        T* h = reinterpret_cast<T*>(c.mailbox + off);
        if (n) SC_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, c.stream));
        off += n * sizeof(T);
        return h;
    }
    void wait() { SC_CUDA(cudaStreamSynchronize(c.stream)); }
};

template <class T>
T to_host(Ctx& c, const T* d) {
    Mailbox mb(c);
    const T* h = mb.get(d, 1);
    mb.wait();
    return *h;
}

template <class T>
void h2d(Ctx& c, T* d, const T* h, size_t n) {
    if (n) SC_CUDA(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, c.stream));
}
template <class T>
void d2h(Ctx& c, T* h, const T* d, size_t n) {
    if (n) SC_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, c.stream));
}
template <class T>
void d2d(Ctx& c, T* dst, const T* src, size_t n) {
    if (n) SC_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, c.stream));
}
template <class T>
void zero(Ctx& c, T* d, size_t n) {
    if (n) SC_CUDA(cudaMemsetAsync(d, 0, n * sizeof(T), c.stream));
}
inline void sync(Ctx& c) { SC_CUDA(cudaStreamSynchronize(c.stream)); }


// Sum of x over this lane's peers (the lanes holding the same key; `peers` from
// __match_any_sync), complete in the lowest peer. A tree fold over each peer
// group's ranks: in round r a peer whose rank has bit r clear adds the value of
// the next peer above it that is still open, then the peers with bit r set
// close; five rounds at most. Use it where the grouping cannot change the sum:
// integers, or doubles whose every partial sum is exact. Neighbour entries of
// a node (or of a group's members) mostly share one or two keys, and without
// this fold each of them lands on the same table slot, one atomic after
// another. Every lane of the warp must call it.
template <class T>
__device__ __forceinline__ T peer_sum(unsigned peers, T x) {
    const unsigned FULL = 0xFFFFFFFFu;
    const unsigned lane = threadIdx.x & 31u;
    unsigned rank = __popc(peers & ((1u << lane) - 1u));
    unsigned above = peers & ~((2u << lane) - 1u);  // lane 31: (2u << 31) - 1 = ~0u, nothing above
    while (__any_sync(FULL, above != 0u)) {
        const int next = __ffs(above);
        const T t = __shfl_sync(FULL, x, next ? next - 1 : (int)lane);
        if (next) x += t;
        above &= ~__ballot_sync(FULL, rank & 1u);
        rank >>= 1;
    }
    return x;
}

// Σ_{i in [b, e)} f(i) in index order, by one warp: lanes load 32 terms at a
// time (coalesced), then every lane folds them in order through shuffles, so
// the result is the sequential left fold of the reference, bit for bit, while
// the loads stay memory-parallel. Every lane returns the same value.
template <class F>
__device__ __forceinline__ double warp_ordered_sum(uint64_t b, uint64_t e, double init, F f) {
    const unsigned lane = threadIdx.x & 31u;
    double acc = init;
    for (uint64_t base = b; base < e; base += 32) {
        const uint64_t i = base + lane;
        const double x = i < e ? f(i) : 0.0;
        const unsigned cnt = (unsigned)((e - base) < 32 ? (e - base) : 32);
        for (unsigned j = 0; j < cnt; ++j) acc = __dadd_rn(acc, __shfl_sync(0xFFFFFFFFu, x, (int)j));
    }
    return acc;
}

// init + Σ f(i) when every partial sum is exact (the exact regime): any order
// gives the same bits, so lanes accumulate strided and reduce by butterfly.
// Falls back to the ordered fold otherwise. Every lane returns the same value.
template <class F>
__device__ __forceinline__ double warp_fold(uint64_t b, uint64_t e, double init, bool exact, F f) {
    if (!exact) return warp_ordered_sum(b, e, init, f);
    const unsigned lane = threadIdx.x & 31u;
    double acc = 0.0;
    for (uint64_t i = b + lane; i < e; i += 32) acc = __dadd_rn(acc, f(i));
    for (int o = 16; o; o >>= 1) acc = __dadd_rn(acc, __shfl_xor_sync(0xFFFFFFFFu, acc, o));
    return e > b ? __dadd_rn(init, acc) : init;
}

}  // namespace sc
