// host_stage.cpp -- host-to-device uploads of large pageable buffers through
// pinned staging memory.
//
// A copy from pageable memory is staged by the driver through its own small
// pinned buffers, one chunk at a time, at the speed of one host thread's
// memcpy.  Volumes are uploaded whole (hundreds of MB to GB), so this path
// pipelines the upload instead: the host buffer is copied in chunks into one
// of two pinned staging buffers by several threads while the DMA engine
// moves the other buffer's previous chunk to the device.  The staging
// buffers (2 x 32 MB, allocated on first use with cudaHostAllocPortable so
// that every device can read them) are shared by the process and kept until
// it exits; uploads that run at the same time take turns on them.
#include <cuda_runtime.h>
#include <omp.h>
#include <string.h>

#include <algorithm>
#include <mutex>

#include "mk_internal.h"

namespace mk {

namespace {

constexpr size_t kStageChunk = 32u << 20;
constexpr size_t kStageMin = 8u << 20;      // smaller uploads copy directly
constexpr int kStageThreads = 8;

std::mutex g_stage_mu;
void *g_stage_buf[2] = {nullptr, nullptr};
bool g_stage_failed = false;

// Copy n bytes with up to kStageThreads threads, 1 MB or more each.
void parallel_copy(void *dst, const void *src, size_t n) {
    const size_t piece = 1u << 20;
    const long pieces = (long)((n + piece - 1) / piece);
    const int threads = std::max(1, std::min(kStageThreads, (int)std::min<long>(pieces, omp_get_max_threads())));
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long i = 0; i < pieces; ++i) {
        const size_t off = (size_t)i * piece;
        memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, std::min(piece, n - off));
    }
}

}  // namespace

cudaError_t stage_to_device(void *dst, const void *src, size_t bytes, cudaStream_t s) {
    if (bytes < kStageMin) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    std::lock_guard<std::mutex> lk(g_stage_mu);
    if (!g_stage_buf[0] && !g_stage_failed) {
        for (int b = 0; b < 2; ++b) {
            if (cudaHostAlloc(&g_stage_buf[b], kStageChunk, cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                if (b == 1) cudaFreeHost(g_stage_buf[0]);
                g_stage_buf[0] = g_stage_buf[1] = nullptr;
                g_stage_failed = true;
                break;
            }
        }
    }
    if (!g_stage_buf[0]) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool used[2] = {false, false};
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) e = cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming);
    for (size_t off = 0, i = 0; e == cudaSuccess && off < bytes; off += kStageChunk, ++i) {
        const int b = (int)(i & 1);
        const size_t n = std::min(kStageChunk, bytes - off);
        if (used[b]) e = cudaEventSynchronize(ev[b]);    // its previous chunk has left the buffer
        if (e != cudaSuccess) break;
        parallel_copy(g_stage_buf[b], static_cast<const char *>(src) + off, n);
        e = cudaMemcpyAsync(static_cast<char *>(dst) + off, g_stage_buf[b], n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaEventRecord(ev[b], s);
        used[b] = true;
    }
    // the buffers are free for the next upload only once both copies are done
    for (int b = 0; b < 2; ++b) {
        if (ev[b]) {
            if (used[b]) {
                const cudaError_t w = cudaEventSynchronize(ev[b]);
                if (e == cudaSuccess) e = w;
            }
            cudaEventDestroy(ev[b]);
        }
    }
    return e;
}

}  // namespace mk
