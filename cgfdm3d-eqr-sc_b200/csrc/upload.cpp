// Host -> device upload of large pageable arrays (the medium volume of a
// session, hundreds of MB): a pageable cudaMemcpy runs at about 10 GB/s on
// the B200 hosts, one host thread copying into the driver's staging buffer.
// Here several host threads copy chunks into pinned staging slots, each
// thread issuing its slots' DMA on its own stream as soon as a slot is
// filled, so the host copies and the DMA overlap.  The staging slots (pinned
// host memory) are made on first use and kept for the process: pinning them
// again for every session would cost more than it saves.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "upload.hpp"

namespace cgfdm {

namespace {
constexpr int UP_THREADS = 8;               // host copy threads
constexpr size_t UP_CHUNK = 8u << 20;       // bytes per staging slot
constexpr size_t UP_MIN = 64u << 20;        // smaller uploads: one plain copy

struct Staging {
    std::mutex lock;                        // one pipelined upload at a time
    bool ready = false;
    char *slot[UP_THREADS][2] = {};
    cudaStream_t stream[UP_THREADS] = {};
    cudaEvent_t done[UP_THREADS][2] = {};
    int device = -1;
};
Staging &staging()
{
    static Staging s;
    return s;
}

// the pinned slots, streams and events, on `device` (made once per process;
// remade if a later upload targets another device)
cudaError_t prepare(Staging &s, int device)
{
    if (s.ready && s.device == device) return cudaSuccess;
    if (s.ready) {
        for (int t = 0; t < UP_THREADS; t++) {
            cudaStreamDestroy(s.stream[t]);
            for (int b = 0; b < 2; b++) cudaEventDestroy(s.done[t][b]);
        }
    } else {
        for (int t = 0; t < UP_THREADS; t++)
            for (int b = 0; b < 2; b++) {
                void *p = nullptr;
                cudaError_t e = cudaHostAlloc(&p, UP_CHUNK, cudaHostAllocPortable);
                if (e != cudaSuccess) {
                    // give back what was pinned; the caller copies plainly
                    for (int u = 0; u < UP_THREADS; u++)
                        for (int c = 0; c < 2; c++)
                            if (s.slot[u][c]) cudaFreeHost(s.slot[u][c]), s.slot[u][c] = nullptr;
                    cudaGetLastError();
                    return e;
                }
                s.slot[t][b] = (char *)p;
            }
    }
    for (int t = 0; t < UP_THREADS; t++) {
        cudaError_t e = cudaStreamCreateWithFlags(&s.stream[t], cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
        for (int b = 0; b < 2; b++) {
            e = cudaEventCreateWithFlags(&s.done[t][b], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    s.ready = true;
    s.device = device;
    return cudaSuccess;
}
}  // namespace

cudaError_t upload_h2d(void *dst, const void *src, size_t bytes, int device, cudaStream_t st)
{
    if (bytes < UP_MIN) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
    // the caller's stream may still be writing dst (a memset): the copies wait
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    Staging &s = staging();
    std::lock_guard<std::mutex> guard(s.lock);
    if ((e = prepare(s, device)) != cudaSuccess) return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    const size_t nchunk = (bytes + UP_CHUNK - 1) / UP_CHUNK;
    std::atomic<int> failed{0};
    auto worker = [&](int t) {
        if (cudaSetDevice(device) != cudaSuccess) {
            failed = 1;
            return;
        }
        int use = 0;
        for (size_t c = t; c < nchunk && !failed; c += UP_THREADS, use++) {
            const int b = use & 1;
            // the slot's previous DMA must have read it
            if (use >= 2 && cudaEventSynchronize(s.done[t][b]) != cudaSuccess) {
                failed = 1;
                return;
            }
            const size_t off = c * UP_CHUNK, len = std::min(UP_CHUNK, bytes - off);
            std::memcpy(s.slot[t][b], (const char *)src + off, len);
            if (cudaMemcpyAsync((char *)dst + off, s.slot[t][b], len, cudaMemcpyHostToDevice, s.stream[t]) !=
                    cudaSuccess ||
                cudaEventRecord(s.done[t][b], s.stream[t]) != cudaSuccess) {
                failed = 1;
                return;
            }
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < UP_THREADS; t++) th.emplace_back(worker, t);
    worker(0);
    for (auto &x : th) x.join();
    for (int t = 0; t < UP_THREADS; t++) {
        cudaError_t es = cudaStreamSynchronize(s.stream[t]);
        if (es != cudaSuccess) e = es;
    }
    if (e == cudaSuccess && failed) e = cudaErrorUnknown;
    return e;
}

}  // namespace cgfdm
