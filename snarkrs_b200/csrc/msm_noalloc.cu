// A G1 MSM entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc.  One example is a process whose device
// memory is owned by another allocator, such as a framework's caching pool
// that has reserved the whole card. Another is a latency-critical loop where
// cudaMalloc's implicit device synchronisation or the chance of it failing
// mid-request is not acceptable. A third is code that must never grow the
// process's device footprint after start-up. g16_msm_g1_device and g16_msm_g1
// grow their scratch buffers on demand with cudaMalloc.  This entry point instead
// works entirely inside one fixed scratch array that is part of the library
// image: a file-scope __device__ array of NOALLOC_SCRATCH_BYTES (about 12 MiB)
// that every GPU which loads the library holds until the process exits.
//
// Limits and behaviour:
//   * at most NOALLOC_MAX_POINTS (16384) points per call; larger inputs are
//     refused with G16_ERR_INVALID_ARGUMENT before anything is launched;
//   * fixed 11-bit windows (24 windows, 1024 buckets each), which is what
//     bounds the scratch size;
//   * work runs on the device's legacy default stream and the call returns
//     after the result is on the host;
//   * every call on a device shares the one array and leaves the previous
//     call's data in it; the counters that must start at zero are cleared by
//     each call, everything else is overwritten before it is read.  Calls
//     whose device work overlaps (several host threads, or several streams
//     touching the same device) race on the array and must be serialised by
//     the caller;
//   * the first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and caches it; make that
//     first call before any stream capture begins.  With CUDA's lazy module
//     loading (the default since CUDA 12.2) that first call is also when the
//     device commits the array's memory and loads the MSM kernels, so make it
//     at start-up: on a device whose memory is already full it can fail, with
//     G16_ERR_DEVICE_MEMORY;
//   * the cached address belongs to the device's context at the first call:
//     resetting the device (cudaDeviceReset) after it is not supported;
//   * kernel timing (g16_kernel_timing_enable) must be off, since timing
//     creates CUDA events.
#include <mutex>
#include "common.cuh"
#include "g16b200.h"
#include "host_bn254.hpp"
#include "msm.cuh"

namespace {

constexpr size_t NOALLOC_MAX_POINTS = 1u << 14;
constexpr int NOALLOC_C = 11;
constexpr int NOALLOC_W = (255 + NOALLOC_C - 1) / NOALLOC_C;      // 24 windows
constexpr size_t NOALLOC_B = (size_t)1 << (NOALLOC_C - 1);        // 1024 buckets per window
constexpr size_t NOALLOC_K = NOALLOC_W * NOALLOC_B;               // 24576 buckets in all
constexpr size_t NOALLOC_CHUNK = 16;                              // entries per accumulate thread
constexpr g16::MsmReducePlan NOALLOC_PLAN =
    g16::msm_reduce_plan(NOALLOC_W, NOALLOC_B, false, g16::msm_reduce_pieces(false));

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// byte offsets of each region inside the scratch array
constexpr size_t OFF_SCALARS = 0;
constexpr size_t OFF_COUNTS = align256(OFF_SCALARS + 32 * NOALLOC_MAX_POINTS);
constexpr size_t U32_K = align256(4 * (NOALLOC_K + 1));
constexpr size_t OFF_OFFSETS = OFF_COUNTS + U32_K;
constexpr size_t OFF_CURSOR = OFF_OFFSETS + U32_K;
constexpr size_t OFF_SEGBASE = OFF_CURSOR + U32_K;
constexpr size_t OFF_FAT = OFF_SEGBASE + U32_K;
constexpr size_t OFF_SCANTMP = OFF_FAT + U32_K;
constexpr size_t SCANTMP_ELEMS = NOALLOC_K / 1024 + 2;
constexpr size_t OFF_ENTRIES = align256(OFF_SCANTMP + 4 * SCANTMP_ELEMS);
constexpr size_t ENTRIES_ELEMS = NOALLOC_MAX_POINTS * NOALLOC_W;
constexpr size_t OFF_TOTAL = align256(OFF_ENTRIES + 4 * ENTRIES_ELEMS);
constexpr size_t OFF_PARTIALS = align256(OFF_TOTAL + 16);
constexpr size_t PARTIALS_BYTES =
    g16::XYZZ_G1_BYTES * (NOALLOC_K + (ENTRIES_ELEMS + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK + 1);
constexpr size_t OFF_BUCKETS = align256(OFF_PARTIALS + PARTIALS_BYTES);
constexpr size_t BUCKETS_BYTES = g16::XYZZ_G1_BYTES * NOALLOC_K;
constexpr size_t OFF_SEGMENTS = align256(OFF_BUCKETS + BUCKETS_BYTES);
constexpr size_t SEGMENTS_BYTES = g16::XYZZ_G1_BYTES * NOALLOC_PLAN.block_points();
constexpr size_t OFF_WINDOWS = align256(OFF_SEGMENTS + SEGMENTS_BYTES);
constexpr size_t WINDOWS_BYTES = g16::XYZZ_G1_BYTES * NOALLOC_PLAN.result_points();
constexpr size_t OFF_WORK = align256(OFF_WINDOWS + WINDOWS_BYTES);
constexpr size_t NOALLOC_SCRATCH_BYTES = align256(OFF_WORK + 8);

// The scratch itself.  In host code this name is only a stand-in for the
// device symbol; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_msm_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_addr[MAX_DEVICES] = {};

}  // namespace

namespace g16 {
int cuda_fail(cudaError_t e, const char* what);   // prover.cu: status of a failed CUDA call, sticky faults recorded
int device_fault(int ordinal);                     // prover.cu: the sticky fault that took a device out of use
}  // namespace g16

namespace {

int fail_noalloc(int code, const char* msg) {
    g16::set_error("%s", msg);
    return code;
}

}  // namespace

extern "C" int g16_msm_g1_device_noalloc(int device, const void* d_bases, const void* d_scalars, size_t n,
                                         int scalars_form, uint8_t* out64) {
    if (!out64 || (n && (!d_bases || !d_scalars)))
        return fail_noalloc(G16_ERR_INVALID_ARGUMENT, "g16_msm_g1_device_noalloc: null argument");
    if (scalars_form != G16_SCALARS_STANDARD && scalars_form != G16_SCALARS_MONTGOMERY)
        return fail_noalloc(G16_ERR_INVALID_ARGUMENT, "g16_msm_g1_device_noalloc: unknown scalar form");
    if (n > NOALLOC_MAX_POINTS) {
        g16::set_error("g16_msm_g1_device_noalloc: %zu points exceed the fixed scratch limit of %zu points", n,
                       (size_t)NOALLOC_MAX_POINTS);
        return G16_ERR_INVALID_ARGUMENT;
    }
    if (device < 0 || device >= MAX_DEVICES)
        return fail_noalloc(G16_ERR_INVALID_ARGUMENT, "g16_msm_g1_device_noalloc: device ordinal out of range");
    if (const int f = g16::device_fault(device)) {
        g16::set_error("g16_msm_g1_device_noalloc: CUDA device %d is out of use after %s: a sticky fault earlier in "
                       "this process", device, cudaGetErrorString((cudaError_t)f));
        return G16_ERR_DEVICE;
    }
    if (g16::timer().enabled)
        return fail_noalloc(G16_ERR_INVALID_ARGUMENT,
                            "g16_msm_g1_device_noalloc: kernel timing creates CUDA events; disable it first");
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        g16::set_error("g16_msm_g1_device_noalloc: cudaSetDevice(%d): %s", device, cudaGetErrorString(e));
        return G16_ERR_DEVICE;
    }
    if (n == 0) {
        std::memset(out64, 0, 64);
        return G16_OK;
    }
    unsigned char* base;
    {
        // once per device, with that device current
        std::lock_guard<std::mutex> g(g_setup_mu);
        if (!g_scratch_addr[device]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_msm_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                g16::set_error("g16_msm_g1_device_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                // lazy module loading commits the array here: a full device is a memory error
                return e == cudaErrorMemoryAllocation ? G16_ERR_DEVICE_MEMORY : G16_ERR_DEVICE;
            }
            g_scratch_addr[device] = (unsigned char*)p;
        }
        base = g_scratch_addr[device];
    }
    g16::host_init();
    // views into the scratch, with capacities that make every grow() a no-op
    g16::MsmSort s;
    s.fixed = true;
    s.d_scalars_std = (uint32_t*)(base + OFF_SCALARS);
    s.cap_scalars = 8 * NOALLOC_MAX_POINTS;
    s.d_counts = (uint32_t*)(base + OFF_COUNTS);
    s.d_offsets = (uint32_t*)(base + OFF_OFFSETS);
    s.d_cursor = (uint32_t*)(base + OFF_CURSOR);
    s.d_seg_base = (uint32_t*)(base + OFF_SEGBASE);
    s.d_fat_list = (uint32_t*)(base + OFF_FAT);
    s.cap_k = NOALLOC_K + 1;
    s.d_scan_tmp = (uint32_t*)(base + OFF_SCANTMP);
    s.cap_tmp = SCANTMP_ELEMS;
    s.d_entries = (uint32_t*)(base + OFF_ENTRIES);
    s.cap_entries = ENTRIES_ELEMS;
    s.d_total = (uint32_t*)(base + OFF_TOTAL);
    g16::MsmAccum acc;
    acc.fixed = true;
    acc.d_partials = base + OFF_PARTIALS;
    acc.cap_partials = PARTIALS_BYTES;
    acc.d_buckets = base + OFF_BUCKETS;
    acc.cap_buckets = BUCKETS_BYTES;
    acc.d_segments = base + OFF_SEGMENTS;
    acc.cap_segments = SEGMENTS_BYTES;
    acc.d_windows = base + OFF_WINDOWS;
    acc.cap_windows = WINDOWS_BYTES;
    acc.d_work = (unsigned long long*)(base + OFF_WORK);
    cudaStream_t st = 0;   // the legacy default stream: no stream is created
    e = g16::msm_sort(s, d_scalars, n, scalars_form == G16_SCALARS_MONTGOMERY, NOALLOC_C, st);
    if (e == cudaSuccess) e = g16::msm_accumulate_g1(s, acc, d_bases, 0, (uint32_t)n, st);
    static_assert(WINDOWS_BYTES <= 64 * 1024, "the reduction's result is read into a stack buffer");
    uint8_t windows[WINDOWS_BYTES];
    const g16::MsmReducePlan plan = acc.plan;
    if (e == cudaSuccess && acc.result_bytes(g16::XYZZ_G1_BYTES) != WINDOWS_BYTES) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaMemcpy(windows, acc.d_windows, sizeof windows, cudaMemcpyDeviceToHost);
    // the views must not free the library's array
    s = g16::MsmSort();
    acc = g16::MsmAccum();
    if (e != cudaSuccess) {
        g16::set_error("%s", "");
        return g16::cuda_fail(e, "g16_msm_g1_device_noalloc");
    }
    g16::pack(out64, g16::msm_combine_g1(windows, plan, NOALLOC_C).to_affine());
    return G16_OK;
}
