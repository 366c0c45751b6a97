// Shared host-side plumbing: error capture and optional per-kernel event timing.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace g16 {

// thread-local last error text, surfaced through g16_last_error()
void set_error(const char* fmt, ...);

#define G16_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            ::g16::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                             cudaGetErrorString(e_));                               \
            return e_;                                                              \
        }                                                                           \
    } while (0)

// Kernel-class timing with CUDA events on the launching stream.  Disabled by
// default; when enabled every tagged launch is bracketed by two events and the
// elapsed times are folded in at collect() (after the stream has synchronised).
struct KernelTimer {
    bool enabled = false;
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    std::map<std::string, std::pair<double, long>> totals;   // ms, launches
    std::map<std::string, double> units;                     // algorithmic work, per kernel class
    std::map<std::string, double> bytes;                     // algorithmic HBM bytes, per kernel class
    std::atomic<uint64_t> launches{0};                        // every kernel this library launched
    std::atomic<uint64_t> device_allocs{0};                   // every cudaMalloc this library made
    std::atomic<uint64_t> device_alloc_bytes{0};              // and their bytes
    std::mutex mu;

    void add_units(const char* name, double u) {
        if (!enabled) return;
        std::lock_guard<std::mutex> g(mu);
        units[name] += u;
    }
    void add_bytes(const char* name, double b) {
        if (!enabled) return;
        std::lock_guard<std::mutex> g(mu);
        bytes[name] += b;
    }

    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
    void begin(const char* name, cudaStream_t s) {
        if (!enabled) return;
        std::lock_guard<std::mutex> g(mu);
        Pending p;
        p.name = name;
        p.a = take();
        p.b = take();
        cudaEventRecord(p.a, s);
        pending.push_back(p);
    }
    void end(cudaStream_t s) {
        if (!enabled) return;
        std::lock_guard<std::mutex> g(mu);
        if (!pending.empty()) cudaEventRecord(pending.back().b, s);
    }
    void collect() {
        std::lock_guard<std::mutex> g(mu);
        for (auto& p : pending) {
            float ms = 0.f;
            if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                auto& t = totals[p.name];
                t.first += ms;
                t.second += 1;
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void reset() {
        collect();
        std::lock_guard<std::mutex> g(mu);
        totals.clear();
        units.clear();
        bytes.clear();
    }
};

KernelTimer& timer();

struct TimedLaunch {
    cudaStream_t s;
    TimedLaunch(const char* name, cudaStream_t st) : s(st) {
        timer().launches.fetch_add(1, std::memory_order_relaxed);
        timer().begin(name, st);
    }
    ~TimedLaunch() { timer().end(s); }
};

// Every device allocation of the library goes through here, so that the number
// of allocations it has made is observable (g16_device_alloc_count).
template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes) {
    timer().device_allocs.fetch_add(1, std::memory_order_relaxed);
    timer().device_alloc_bytes.fetch_add(bytes, std::memory_order_relaxed);
    return cudaMalloc((void**)p, bytes);
}

// Byte that new value buffers are filled with, or -1 (the default):
// G16_FILL_VALUES=<0..255>.  A fresh process gets zeroed pages from the
// driver, and zeros read as points at infinity and as zero scalars, so a read
// of a point or a scalar that no kernel wrote goes unnoticed there; a filled
// buffer exposes it.  Only buffers of values (points, scalars, and tables that
// are uploaded whole before use) take the fill, never index arrays.
inline int value_fill_byte() {
    static const int v = [] {
        const char* e = std::getenv("G16_FILL_VALUES");
        if (!e || !*e) return -1;
        const int b = std::atoi(e);
        return b >= 0 && b <= 255 ? b : -1;
    }();
    return v;
}

// dev_malloc for a buffer of values (value_fill_byte).
template <class T>
inline cudaError_t dev_malloc_values(T** p, size_t bytes) {
    cudaError_t e = dev_malloc(p, bytes);
    const int fill = value_fill_byte();
    // the legacy stream does not order against the library's non-blocking
    // streams: the fill completes before the buffer is handed out
    if (e == cudaSuccess && fill >= 0 && bytes) e = cudaMemset((void*)*p, fill, bytes);
    if (e == cudaSuccess && fill >= 0 && bytes) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}

// Growable scratch (sort, bucket and engine buffers) is allocated and freed in
// stream order, from the device's default memory pool.  cudaMalloc and cudaFree
// are not: an allocation serialises every stream of the device and a free waits
// for all of its work, so a buffer that grows while other proofs run would stall
// them all.  The old buffer goes back on the same stream, which must be the only
// one with work on it in flight (a workspace or engine is idle when it grows).
// Such memory may still be released with cudaFree, which for it does not wait
// for the device: every owner's release synchronises the owner's streams first
// (Workspace, BatchEngine, the backend's own MSM scratch).  No buffer grows
// inside a stream capture: there the allocation would belong to the graph.
template <class T>
inline cudaError_t dev_realloc_async(T** p, size_t bytes, cudaStream_t st, bool values) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return e;
    if (cs != cudaStreamCaptureStatusNone) return cudaErrorStreamCaptureUnsupported;
    if (*p) e = cudaFreeAsync((void*)*p, st);
    *p = nullptr;
    if (e != cudaSuccess) return e;
    timer().device_allocs.fetch_add(1, std::memory_order_relaxed);
    timer().device_alloc_bytes.fetch_add(bytes, std::memory_order_relaxed);
    e = cudaMallocAsync((void**)p, bytes, st);
    const int fill = values ? value_fill_byte() : -1;
    if (e == cudaSuccess && fill >= 0 && bytes) e = cudaMemsetAsync((void*)*p, fill, bytes, st);
    return e;
}

inline unsigned blocks_for(size_t n, unsigned threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace g16
