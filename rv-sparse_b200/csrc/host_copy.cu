// Results that leave the device for pageable host memory: the host arrays
// the one-shot entry points allocate for C, and the device->host copies that
// fill them (and a caller's own pageable C arrays on the plan path).
//
// A plain cudaMemcpy into pageable memory moves the bytes through the
// driver's small pinned bounce buffers on the calling thread, and a freshly
// allocated destination takes a page fault for every 4 KiB page inside that
// copy: about 2 GB/s for a C of several GB. Here the device copies C in
// CHUNK-byte pieces into a ring of pinned buffers, and a team of host
// threads moves each finished piece into the destination, so the PCIe
// transfer, the destination's page faults and the host copies overlap.
// Large pageable operands go up the same way in reverse (copy_to_device):
// host threads fill the pinned pieces, each piece's upload is enqueued as
// soon as it is full. The
// arrays host_alloc hands out are 2 MiB aligned with transparent huge pages
// advised, which cuts their page faults 512-fold, and free() releases them.
//
// Result arrays of 64 MiB and more that the library releases itself
// (rvsp_csr_destroy, host_free) are kept in a small cache and handed out
// again by host_alloc: a fresh array's pages are faulted in and zeroed by
// the kernel inside the copy (38 GB/s with 16 threads into fresh pages),
// while a cached one's are already mapped. The cache holds at most 4
// arrays and a sixteenth of the host memory (32 GiB at most), frees the
// oldest first, and RVSP_HOST_CACHE=0 turns it off. It keeps allocations
// only: every product computes and copies its C in full.
#include <malloc.h>
#include <sched.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <unistd.h>

#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "rvsp_cuda.h"
#include "rvsp_internal.h"

namespace rvsp {

namespace {

constexpr size_t HUGE_PAGE = 2u << 20;
constexpr size_t CHUNK = 32u << 20;      // one piece between device and host
constexpr int RING = 16;                 // pinned pieces in flight
constexpr size_t STAGED_MIN = 64u << 20;  // smaller copy-backs go direct
constexpr size_t STAGED_MIN_UP = 16u << 20;  // smaller uploads go direct
constexpr int MAX_DEVICES = 16;
constexpr int MAX_THREADS = 16;

// One ring per device: pinned pieces and the events that mark each piece's
// device copy done, tied to the context that made them (a device reset
// frees pinned memory, so a ring of an older context is dropped, not freed).
struct Ring {
    unsigned long long ctx = 0;
    char* pin[RING] = {};
    cudaEvent_t ev[RING] = {};
};
Ring g_ring[MAX_DEVICES];
std::mutex g_ring_mu[MAX_DEVICES];

bool ring_ready(Ring& r) {
    const unsigned long long ctx = current_context_id();
    if (ctx == 0) return false;  // no way to tell the ring's context is live
    if (r.ctx == ctx) return true;
    Ring fresh;
    for (int i = 0; i < RING; ++i) {
        if (cudaHostAlloc((void**)&fresh.pin[i], CHUNK, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&fresh.ev[i], cudaEventDisableTiming | cudaEventBlockingSync) !=
                cudaSuccess) {
            for (int j = 0; j <= i; ++j) {
                if (fresh.pin[j]) cudaFreeHost(fresh.pin[j]);
                if (fresh.ev[j]) cudaEventDestroy(fresh.ev[j]);
            }
            cudaGetLastError();
            return false;
        }
    }
    // a previous ring belongs to a context that a reset destroyed (or that
    // the caller left without a reset): either way it is not freed here
    fresh.ctx = ctx;
    r = fresh;
    return true;
}

int copy_threads() {
    static const int n = [] {
        const char* env = getenv("RVSP_HOST_COPY_THREADS");
        if (env && atoi(env) > 0) return atoi(env) < MAX_THREADS ? atoi(env) : MAX_THREADS;
        cpu_set_t set;
        int cpus = 1;
        if (sched_getaffinity(0, sizeof(set), &set) == 0) cpus = CPU_COUNT(&set);
        return cpus < 1 ? 1 : (cpus > MAX_THREADS ? MAX_THREADS : cpus);
    }();
    return n;
}

// the released-array cache (see the top of this file)
constexpr int CACHE_MAX_ARRAYS = 4;
struct CachedArray {
    void* p;
    size_t bytes;  // malloc_usable_size
};
std::mutex g_cache_mu;
std::vector<CachedArray> g_cache;  // oldest first
size_t g_cache_bytes = 0;

bool cache_on() {
    static const bool on = [] {
        const char* env = getenv("RVSP_HOST_CACHE");
        return !(env && env[0] == '0');
    }();
    return on;
}

size_t cache_cap() {
    static const size_t cap = [] {
        const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
        // a sixteenth of host memory: one process per GPU, eight on a box,
        // keep half of it at most between them
        const size_t share = pages > 0 && page > 0 ? (size_t)pages * (size_t)page / 16 : 0;
        const size_t max = (size_t)32 << 30;
        return share < max ? share : max;
    }();
    return cap;
}

// a stream recording a CUDA graph takes no host waits: plain copies there
bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return st != cudaStreamCaptureStatusNone;
}

bool pinned_host(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

void* host_alloc(size_t bytes) {
    if (bytes < STAGED_MIN) return malloc(bytes ? bytes : 1);
    if (cache_on()) {
        // the smallest cached array that holds bytes and wastes at most half
        std::lock_guard<std::mutex> hold(g_cache_mu);
        int best = -1;
        for (int i = 0; i < (int)g_cache.size(); ++i)
            if (g_cache[i].bytes >= bytes && g_cache[i].bytes / 2 <= bytes &&
                (best < 0 || g_cache[i].bytes < g_cache[best].bytes))
                best = i;
        if (best >= 0) {
            void* p = g_cache[best].p;
            g_cache_bytes -= g_cache[best].bytes;
            g_cache.erase(g_cache.begin() + best);
            return p;
        }
    }
    void* p = nullptr;
    if (posix_memalign(&p, HUGE_PAGE, bytes) != 0) return nullptr;
    madvise(p, bytes & ~(HUGE_PAGE - 1), MADV_HUGEPAGE);  // advice only: failure is harmless
    return p;
}

void host_free(void* p) {
    if (!p) return;
    const size_t bytes = malloc_usable_size(p);
    if (cache_on() && bytes >= STAGED_MIN && bytes <= cache_cap()) {
        std::vector<void*> evict;
        {
            std::lock_guard<std::mutex> hold(g_cache_mu);
            g_cache.push_back({p, bytes});
            g_cache_bytes += bytes;
            while (g_cache.size() > (size_t)CACHE_MAX_ARRAYS || g_cache_bytes > cache_cap()) {
                evict.push_back(g_cache.front().p);
                g_cache_bytes -= g_cache.front().bytes;
                g_cache.erase(g_cache.begin());
            }
        }
        for (void* q : evict) free(q);
        return;
    }
    free(p);
}

cudaError_t copy_to_host(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (capturing(stream))  // recorded into the graph; no host wait allowed
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream)
                     : cudaSuccess;
    if (bytes == 0) return cudaStreamSynchronize(stream);
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int threads = copy_threads();
    if (bytes < STAGED_MIN || dev < 0 || dev >= MAX_DEVICES || threads < 2 || pinned_host(dst)) {
        e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream);
        return e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
    }
    std::lock_guard<std::mutex> hold(g_ring_mu[dev]);
    Ring& r = g_ring[dev];
    trace_point("host copy-back: start");
    if (!ring_ready(r)) {
        e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream);
        return e == cudaSuccess ? cudaStreamSynchronize(stream) : e;
    }
    const size_t n = (bytes + CHUNK - 1) / CHUNK;
    auto piece = [&](size_t i) { return i + 1 < n ? CHUNK : bytes - i * CHUNK; };
    // issued: pieces whose device copy is enqueued; done[i % RING]: the last
    // piece whose host copy left that ring slot, + 1.
    std::mutex mu;
    std::condition_variable cv;
    size_t issued = 0;
    size_t done[RING] = {};
    std::atomic<size_t> next{0};
    std::atomic<int> err{cudaSuccess};
    auto issue = [&](size_t i) -> cudaError_t {
        const int b = (int)(i % RING);
        cudaError_t x = cudaMemcpyAsync(r.pin[b], (const char*)src + i * CHUNK, piece(i),
                                        cudaMemcpyDeviceToHost, stream);
        if (x == cudaSuccess) x = cudaEventRecord(r.ev[b], stream);
        return x;
    };
    auto worker = [&] {
        cudaSetDevice(dev);  // the ring's events belong to this device
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= n) return;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return issued > i || err.load() != cudaSuccess; });
            }
            if (err.load() != cudaSuccess) return;
            const int b = (int)(i % RING);
            const cudaError_t x = cudaEventSynchronize(r.ev[b]);
            if (x != cudaSuccess) {
                {
                    std::lock_guard<std::mutex> lk(mu);  // a waiter sees it under the lock
                    int none = cudaSuccess;
                    err.compare_exchange_strong(none, (int)x);
                }
                cv.notify_all();
                return;
            }
            memcpy((char*)dst + i * CHUNK, r.pin[b], piece(i));
            {
                std::lock_guard<std::mutex> lk(mu);
                done[b] = i + 1;
            }
            cv.notify_all();
        }
    };
    // the first RING pieces need no free slot
    const size_t first = n < (size_t)RING ? n : (size_t)RING;
    for (size_t i = 0; i < first && err.load() == cudaSuccess; ++i) {
        const cudaError_t x = issue(i);
        if (x != cudaSuccess) err = (int)x;
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        issued = first;
    }
    std::vector<std::thread> team;
    team.reserve(threads);
    for (int t = 0; t < threads; ++t) team.emplace_back(worker);
    for (size_t i = first; i < n && err.load() == cudaSuccess; ++i) {
        const int b = (int)(i % RING);
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return done[b] == i - RING + 1 || err.load() != cudaSuccess; });
        }
        if (err.load() != cudaSuccess) break;
        const cudaError_t x = issue(i);
        {
            std::lock_guard<std::mutex> lk(mu);
            if (x != cudaSuccess) err = (int)x;
            else issued = i + 1;
        }
        cv.notify_all();
    }
    cv.notify_all();
    for (auto& t : team) t.join();
    trace_point("host copy-back (staged)");
    // every issued device copy has ended before a ring slot is used again
    const cudaError_t s = cudaStreamSynchronize(stream);
    return err.load() != cudaSuccess ? (cudaError_t)err.load() : s;
}

cudaError_t copy_to_device(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes == 0) return cudaSuccess;
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const int threads = copy_threads();
    if (bytes < STAGED_MIN_UP || dev < 0 || dev >= MAX_DEVICES || threads < 2 ||
        pinned_host(src) || capturing(stream))
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    std::lock_guard<std::mutex> hold(g_ring_mu[dev]);
    Ring& r = g_ring[dev];
    if (!ring_ready(r)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
    trace_point("host upload: start");
    const size_t n = (bytes + CHUNK - 1) / CHUNK;
    auto piece = [&](size_t i) { return i + 1 < n ? CHUNK : bytes - i * CHUNK; };
    // filled[i % RING]: the last piece copied into that slot, + 1; issued:
    // pieces whose upload is enqueued (a slot is free again once the upload
    // of the piece RING before has completed: its event)
    std::mutex mu;
    std::condition_variable cv;
    size_t issued = 0;
    size_t filled[RING] = {};
    std::atomic<size_t> next{0};
    std::atomic<int> err{cudaSuccess};
    auto worker = [&] {
        cudaSetDevice(dev);
        for (;;) {
            const size_t i = next.fetch_add(1);
            if (i >= n) return;
            const int b = (int)(i % RING);
            if (i >= (size_t)RING) {
                {
                    std::unique_lock<std::mutex> lk(mu);
                    cv.wait(lk, [&] { return issued > i - RING || err.load() != cudaSuccess; });
                }
                if (err.load() != cudaSuccess) return;
                const cudaError_t x = cudaEventSynchronize(r.ev[b]);
                if (x != cudaSuccess) {
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        int none = cudaSuccess;
                        err.compare_exchange_strong(none, (int)x);
                    }
                    cv.notify_all();
                    return;
                }
            }
            memcpy(r.pin[b], (const char*)src + i * CHUNK, piece(i));
            {
                std::lock_guard<std::mutex> lk(mu);
                filled[b] = i + 1;
            }
            cv.notify_all();
        }
    };
    std::vector<std::thread> team;
    team.reserve(threads);
    for (int t = 0; t < threads; ++t) team.emplace_back(worker);
    for (size_t i = 0; i < n; ++i) {
        const int b = (int)(i % RING);
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return filled[b] == i + 1 || err.load() != cudaSuccess; });
            if (err.load() != cudaSuccess) break;
        }
        cudaError_t x = cudaMemcpyAsync((char*)dst + i * CHUNK, r.pin[b], piece(i),
                                        cudaMemcpyHostToDevice, stream);
        if (x == cudaSuccess) x = cudaEventRecord(r.ev[b], stream);
        {
            std::lock_guard<std::mutex> lk(mu);
            if (x != cudaSuccess) err = (int)x;
            else issued = i + 1;
        }
        cv.notify_all();
        if (x != cudaSuccess) break;
    }
    cv.notify_all();
    for (auto& t : team) t.join();
    // the ring's pieces are free for the next user only once every upload
    // from them has completed
    const cudaError_t s = cudaStreamSynchronize(stream);
    trace_point("host upload (staged)");
    return err.load() != cudaSuccess ? (cudaError_t)err.load() : s;
}

}  // namespace rvsp

extern "C" RVSP_CUDA_API void rvsp_cuda_host_free(void* p) { rvsp::host_free(p); }
