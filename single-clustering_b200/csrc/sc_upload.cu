// sc_upload.cu — host -> device copies of large pageable buffers.
//
// A pageable cudaMemcpyAsync is staged by the CUDA driver through its own pinned
// buffers by one thread, about 10 GB/s here. For the graph arrays (hundreds
// of MB) that copy is most of an end-to-end call, so large uploads go through
// the context's own pinned staging instead: STAGE_LANES host threads each copy
// STAGE_CHUNK-byte chunks of the source into their two pinned buffers and queue
// each chunk's DMA on their own stream, so host copies, transfers and the other
// lanes overlap. The context's stream then waits for every lane.
#include <thread>

#include "sc_prims.cuh"

namespace sc {

struct Staging {
    cudaStream_t stream[STAGE_LANES] = {};
    cudaEvent_t done[STAGE_LANES][2] = {};  // the last DMA out of each buffer
    unsigned char* buf[STAGE_LANES][2] = {};
};

namespace {

void destroy(Staging* s) {
    for (int l = 0; l < STAGE_LANES; ++l) {
        if (s->stream[l]) cudaStreamSynchronize(s->stream[l]);
        for (int b = 0; b < 2; ++b) {
            if (s->done[l][b]) cudaEventDestroy(s->done[l][b]);
            if (s->buf[l][b]) cudaFreeHost(s->buf[l][b]);
        }
        if (s->stream[l]) cudaStreamDestroy(s->stream[l]);
    }
    delete s;
}

Staging* staging_of(Ctx& c) {
    if (c.staging) return c.staging;
    Staging* s = new Staging();
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < STAGE_LANES && e == cudaSuccess; ++l) {
        e = cudaStreamCreateWithFlags(&s->stream[l], cudaStreamNonBlocking);
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            e = cudaEventCreateWithFlags(&s->done[l][b], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaHostAlloc((void**)&s->buf[l][b], STAGE_CHUNK, cudaHostAllocDefault);
        }
    }
    if (e != cudaSuccess) {
        destroy(s);
        throw_cuda(e, "pinned staging set-up", __FILE__, __LINE__);
    }
    c.staging = s;
    return s;
}

}  // namespace

void release_staging(Ctx& c) {
    if (c.staging) destroy(c.staging);
    c.staging = nullptr;
}

void upload(Ctx& c, void* dst, const void* src, size_t bytes) {
    if (bytes < STAGE_MIN_BYTES) {
        if (bytes) SC_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c.stream));
        return;
    }
    Staging* s = staging_of(c);
    // dst may come from a stream-ordered allocation on the context's stream
    cudaEvent_t ready;
    SC_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ready, c.stream);
    for (int l = 0; l < STAGE_LANES && e == cudaSuccess; ++l) e = cudaStreamWaitEvent(s->stream[l], ready, 0);
    cudaEventDestroy(ready);
    if (e != cudaSuccess) throw_cuda(e, "staged upload set-up", __FILE__, __LINE__);

    const size_t nchunks = (bytes + STAGE_CHUNK - 1) / STAGE_CHUNK;
    cudaError_t lane_err[STAGE_LANES];
    auto lane = [&](int l) {
        cudaError_t le = cudaSetDevice(c.device);
        int which = 0;
        for (size_t k = (size_t)l; k < nchunks && le == cudaSuccess; k += STAGE_LANES) {
            const size_t off = k * STAGE_CHUNK;
            const size_t len = bytes - off < STAGE_CHUNK ? bytes - off : STAGE_CHUNK;
            unsigned char* b = s->buf[l][which];
            le = cudaEventSynchronize(s->done[l][which]);  // this buffer's previous DMA has finished
            if (le != cudaSuccess) break;
            std::memcpy(b, (const unsigned char*)src + off, len);
            le = cudaMemcpyAsync((unsigned char*)dst + off, b, len, cudaMemcpyHostToDevice, s->stream[l]);
            if (le == cudaSuccess) le = cudaEventRecord(s->done[l][which], s->stream[l]);
            which ^= 1;
        }
        lane_err[l] = le;
    };
    std::thread workers[STAGE_LANES - 1];
    for (int l = 1; l < STAGE_LANES; ++l) {
        try {
            workers[l - 1] = std::thread(lane, l);
        } catch (...) {
            lane(l);  // no thread to be had: this thread copies the lane's chunks itself
        }
    }
    lane(0);
    for (int t = 0; t < STAGE_LANES - 1; ++t)
        if (workers[t].joinable()) workers[t].join();
    for (int l = 0; l < STAGE_LANES; ++l)
        if (lane_err[l] != cudaSuccess) throw_cuda(lane_err[l], "staged upload", __FILE__, __LINE__);
    // the context's stream continues once every lane's DMAs are done
    for (int l = 0; l < STAGE_LANES; ++l) {
        cudaEvent_t fin;
        SC_CUDA(cudaEventCreateWithFlags(&fin, cudaEventDisableTiming));
        e = cudaEventRecord(fin, s->stream[l]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c.stream, fin, 0);
        cudaEventDestroy(fin);
        if (e != cudaSuccess) throw_cuda(e, "staged upload join", __FILE__, __LINE__);
    }
}

namespace {
__global__ void k_widen_labels(const uint32_t* __restrict__ a, uint64_t n, uint64_t* b) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}
}  // namespace

void download_labels(Ctx& c, const uint32_t* d_labels, uint64_t n, uint64_t* host_out) {
    if (n == 0) return;
    DBuf<uint64_t> wide(c, n);
    k_widen_labels<<<grid_for(n, 256), 256, 0, c.stream>>>(d_labels, n, wide.get());
    SC_LAUNCH_CHECK();
    c.launches++;
    SC_CUDA(cudaMemcpyAsync(host_out, wide.get(), n * sizeof(uint64_t), cudaMemcpyDeviceToHost, c.stream));
    sync(c);
}

}  // namespace sc
