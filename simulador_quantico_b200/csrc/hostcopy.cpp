// Large copies between pageable host memory and a device state.
//
// cudaMemcpy from pageable memory stages through one driver buffer on one
// thread: 11 GB/s host->device and 21 GB/s device->host for a 16 GiB state
// on the B200 systems this engine targets.  Here a few host threads each
// own two page-locked chunks and a stream; a thread copies its share of the
// buffer chunk by chunk between host memory and a chunk (memcpy) and between
// the chunk and the device (cudaMemcpyAsync), with the two chunks taking
// turns, so the host copies, the page faults of first-touch host memory and
// the DMA all run in parallel (27-45 GB/s host->device and 42 GB/s
// device->host with four threads, the fastest count measured; more threads
// contend).  Registering the caller's
// buffer instead (cudaHostRegister) copies at 55 GB/s but registering and
// unregistering 16 GiB takes 2.8 s, more than the copy itself.
//
// The chunks (kThreads x 2 x kChunk = 256 MiB of page-locked memory) are
// allocated on the first large copy and kept until exit; copies below
// kStagedMin use a plain cudaMemcpyAsync.  One staged copy runs at a time.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "hgm_internal.h"

namespace hgm {

namespace {

constexpr int kThreads = 4;
constexpr size_t kChunk = size_t(32) << 20;
constexpr size_t kStagedMin = size_t(256) << 20;

struct Stager {
    int device = -1;
    char *buf[kThreads][2] = {};
    cudaStream_t stream[kThreads] = {};
    cudaEvent_t done[kThreads][2] = {};
    bool ready = false;
};

std::mutex g_stage_mu;
Stager g_stage;
bool g_stage_failed = false;

void stager_free() {
    for (int t = 0; t < kThreads; t++) {
        for (int k = 0; k < 2; k++) {
            if (g_stage.buf[t][k]) cudaFreeHost(g_stage.buf[t][k]);
            if (g_stage.done[t][k]) cudaEventDestroy(g_stage.done[t][k]);
        }
        if (g_stage.stream[t]) cudaStreamDestroy(g_stage.stream[t]);
    }
    g_stage = Stager();
}

int stager_alloc() {
    for (int t = 0; t < kThreads; t++) {
        cudaError_t e;
        if ((e = cudaStreamCreateWithFlags(&g_stage.stream[t], cudaStreamNonBlocking)) != cudaSuccess)
            return fail(HGM_ERR_CUDA, "staging stream: %s", cudaGetErrorString(e));
        for (int k = 0; k < 2; k++) {
            if ((e = cudaMallocHost(&g_stage.buf[t][k], kChunk)) != cudaSuccess)
                return fail(HGM_ERR_NOMEM, "staging chunk: %s", cudaGetErrorString(e));
            if ((e = cudaEventCreateWithFlags(&g_stage.done[t][k], cudaEventDisableTiming)) != cudaSuccess)
                return fail(HGM_ERR_CUDA, "staging event: %s", cudaGetErrorString(e));
        }
    }
    return HGM_OK;
}

int stager_init(int device) {
    if (g_stage.ready) return HGM_OK;
    if (g_stage_failed) return HGM_ERR_NOMEM;  // tried once; copy directly from now on
    int rc = stager_alloc();
    if (rc == HGM_OK) {
        g_stage.device = device;
        g_stage.ready = true;
    } else {
        stager_free();
        cudaGetLastError();
        g_stage_failed = true;
    }
    return rc;
}


// Thread t's share: chunks t, t + kThreads, t + 2 kThreads, ...
void stage_h2d(int t, char *dev, const char *host, size_t bytes, std::atomic<int> *err) {
    cudaSetDevice(g_stage.device);
    int k = 0;
    for (size_t off = (size_t)t * kChunk; off < bytes; off += (size_t)kThreads * kChunk, k ^= 1) {
        const size_t n = off + kChunk <= bytes ? kChunk : bytes - off;
        if (cudaEventSynchronize(g_stage.done[t][k]) != cudaSuccess) err->store(1);  // chunk free again
        memcpy(g_stage.buf[t][k], host + off, n);
        if (cudaMemcpyAsync(dev + off, g_stage.buf[t][k], n, cudaMemcpyHostToDevice, g_stage.stream[t]) != cudaSuccess ||
            cudaEventRecord(g_stage.done[t][k], g_stage.stream[t]) != cudaSuccess)
            err->store(1);
    }
    if (cudaStreamSynchronize(g_stage.stream[t]) != cudaSuccess) err->store(1);
}

void stage_d2h(int t, char *host, const char *dev, size_t bytes, std::atomic<int> *err) {
    cudaSetDevice(g_stage.device);
    size_t pending_off = 0, pending_n = 0;
    int pending_k = -1, k = 0;
    for (size_t off = (size_t)t * kChunk; off < bytes; off += (size_t)kThreads * kChunk, k ^= 1) {
        const size_t n = off + kChunk <= bytes ? kChunk : bytes - off;
        if (cudaMemcpyAsync(g_stage.buf[t][k], dev + off, n, cudaMemcpyDeviceToHost, g_stage.stream[t]) != cudaSuccess ||
            cudaEventRecord(g_stage.done[t][k], g_stage.stream[t]) != cudaSuccess)
            err->store(1);
        if (pending_k >= 0) {  // the previous chunk lands while this one is in flight
            if (cudaEventSynchronize(g_stage.done[t][pending_k]) != cudaSuccess) err->store(1);
            memcpy(host + pending_off, g_stage.buf[t][pending_k], pending_n);
        }
        pending_off = off;
        pending_n = n;
        pending_k = k;
    }
    if (pending_k >= 0) {
        if (cudaEventSynchronize(g_stage.done[t][pending_k]) != cudaSuccess) err->store(1);
        memcpy(host + pending_off, g_stage.buf[t][pending_k], pending_n);
    }
}

}  // namespace

int plain_copy(void *dst, const void *src, size_t bytes, bool to_device, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? HGM_OK : fail(HGM_ERR_CUDA, "state copy: %s", cudaGetErrorString(e));
}

int copy_state(void *dst, const void *src, size_t bytes, bool to_device, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (bytes < kStagedMin) return plain_copy(dst, src, bytes, to_device, st);
    // earlier work on the state's stream must be done before the staging
    // streams read or overwrite the state
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(HGM_ERR_CUDA, "state copy: %s", cudaGetErrorString(e));
    int device = 0;
    cudaGetDevice(&device);
    std::unique_lock<std::mutex> lk(g_stage_mu);
    // the chunks belong to the first device that made a large copy; other
    // devices, and hosts where page-locked memory ran out, copy directly
    if (stager_init(device) != HGM_OK || g_stage.device != device) {
        lk.unlock();
        return plain_copy(dst, src, bytes, to_device, st);
    }
    std::atomic<int> err{0};
    std::vector<std::thread> th;
    for (int t = 0; t < kThreads; t++) {
        if (to_device) th.emplace_back(stage_h2d, t, (char *)dst, (const char *)src, bytes, &err);
        else th.emplace_back(stage_d2h, t, (char *)dst, (const char *)src, bytes, &err);
    }
    for (std::thread &x : th) x.join();
    return err.load() ? fail(HGM_ERR_CUDA, "staged state copy failed") : HGM_OK;
}

}  // namespace hgm
