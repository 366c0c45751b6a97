// Pippenger MSM kernels and engine (see msm.cuh for the pipeline).
#include "msm.cuh"
#include <type_traits>
#include "common.cuh"
#include "curve.cuh"
#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <vector>

namespace g16d {

using g16::MSM_DEAD;
using g16::MSM_MAX_SETS;
using g16::MSM_MAX_TARGETS;

// Bits [off, off + width) of a 256-bit little-endian scalar held in shared
// memory (8 words, row stride 9 to spread banks); reads past bit 255 are 0.
__device__ __forceinline__ uint32_t read_bits(const uint32_t* s, int off, int width) {
    int idx = off >> 5;
    if (idx >= 8) return 0;
    int sh = off & 31;
    uint64_t w = s[idx];
    if (idx + 1 < 8) w |= (uint64_t)s[idx + 1] << 32;
    return (uint32_t)(w >> sh) & ((1u << width) - 1u);
}

// Window w's digit of the carry-free signed recoding, in [-2^(c-1), 2^(c-1)]:
// the raw window b borrows 2^c when its top bit is set, and the bit just below
// the window repays the borrow of the window beneath.  255 recoding bits keep
// the top window's borrow zero for every scalar below 2^254.
__device__ __forceinline__ int signed_digit(const uint32_t* s, int w, int c) {
    int off = w * c;
    int b = (int)read_bits(s, off, c);
    int d = b - ((b >> (c - 1)) << c);
    int carry = off ? (int)read_bits(s, off - 1, 1) : 0;
    return d + carry;
}

constexpr uint32_t NO_KEY = 0xffffffffu;

// kw: key stride per window (B when every window has its own buckets, 0 when
// all windows share one bucket set over window-shifted bases)
// sink: the key of a zero digit (NO_KEY: not sorted; the constant-work sink bucket otherwise)
__global__ void __launch_bounds__(256) k_digits_count(const uint4* __restrict__ scalars, int mont, uint32_t n, int c,
                                                      int W, uint32_t kw, uint32_t sink, uint4* __restrict__ scalars_std,
                                                      uint32_t* __restrict__ counts) {
    __shared__ uint32_t sh[256 * 9];
    uint32_t i = blockIdx.x * 256 + threadIdx.x;
    bool valid = i < n;
    Fr s = Fr::zero();
    if (valid) {
        uint4 a = __ldg(scalars + 2 * (size_t)i), b = __ldg(scalars + 2 * (size_t)i + 1);
        s.v[0] = a.x; s.v[1] = a.y; s.v[2] = a.z; s.v[3] = a.w;
        s.v[4] = b.x; s.v[5] = b.y; s.v[6] = b.z; s.v[7] = b.w;
        if (mont) s = from_mont(s);
        scalars_std[2 * (size_t)i] = make_uint4(s.v[0], s.v[1], s.v[2], s.v[3]);
        scalars_std[2 * (size_t)i + 1] = make_uint4(s.v[4], s.v[5], s.v[6], s.v[7]);
    }
    uint32_t* row = sh + threadIdx.x * 9;
#pragma unroll
    for (int j = 0; j < 8; j++) row[j] = s.v[j];
    unsigned lane = threadIdx.x & 31;
    for (int w = 0; w < W; w++) {
        int d = signed_digit(row, w, c);
        uint32_t key = !valid ? NO_KEY : d != 0 ? (uint32_t)w * kw + (uint32_t)(d < 0 ? -d : d) - 1u : sink;
        unsigned mask = __match_any_sync(0xffffffffu, key);
        if (key != NO_KEY && lane == (unsigned)(__ffs(mask) - 1)) atomicAdd(&counts[key], (uint32_t)__popc(mask));
    }
}

// ew: entry-index stride per window (0, or n for window-shifted bases: entry
// w*n + i names base 2^(c w) P_i)
__global__ void __launch_bounds__(256) k_scatter(const uint4* __restrict__ scalars_std, uint32_t n, int c, int W,
                                                 uint32_t kw, uint32_t ew, uint32_t sink, uint32_t* __restrict__ cursor,
                                                 uint32_t* __restrict__ entries) {
    __shared__ uint32_t sh[256 * 9];
    uint32_t i = blockIdx.x * 256 + threadIdx.x;
    bool valid = i < n;
    uint32_t* row = sh + threadIdx.x * 9;
    if (valid) {
        uint4 a = scalars_std[2 * (size_t)i], b = scalars_std[2 * (size_t)i + 1];
        row[0] = a.x; row[1] = a.y; row[2] = a.z; row[3] = a.w;
        row[4] = b.x; row[5] = b.y; row[6] = b.z; row[7] = b.w;
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) row[j] = 0;
    }
    unsigned lane = threadIdx.x & 31;
    unsigned lt = (1u << lane) - 1u;
    for (int w = 0; w < W; w++) {
        int d = signed_digit(row, w, c);
        uint32_t key = !valid ? NO_KEY : d != 0 ? (uint32_t)w * kw + (uint32_t)(d < 0 ? -d : d) - 1u : sink;
        unsigned mask = __match_any_sync(0xffffffffu, key);
        int leader = __ffs(mask) - 1;
        uint32_t base = 0;
        if (key != NO_KEY && (int)lane == leader) base = atomicAdd(&cursor[key], (uint32_t)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (key != NO_KEY) entries[base + __popc(mask & lt)] = ((uint32_t)w * ew + i) | (d < 0 ? 0x80000000u : 0u);
    }
}

// ---- one scalar vector sorted for several live sets (the prover's witness MSMs) ----
// Set j keeps scalar i when rank[j][i] != MSM_DEAD; its entries name row
// rank[j][i] of the set's own window-shifted table: w * rows[j] + rank[j][i].
// The digits are computed once and sorted into every set the scalar is live
// in, so a base at infinity never becomes an entry (a lockstep step of the
// accumulate that adds nothing).
// With per-window bucket sets instead (plain bases, a compact key) window w's
// digit d goes to bucket w B + |d| - 1 and its entry is rank[j][i] itself:
// key_stride = B and rows = 0.
struct LiveSetArgs {
    const uint32_t* rank[MSM_MAX_SETS];
    uint32_t* counts[MSM_MAX_SETS];
    uint32_t* cursor[MSM_MAX_SETS];
    uint32_t* entries[MSM_MAX_SETS];
    uint32_t rows[MSM_MAX_SETS];   // entry stride per window: the table rows, or 0
    uint32_t key_stride;           // bucket offset per window: 0 (one shared set), or B
};

__global__ void __launch_bounds__(256) k_digits_count_sets(const uint4* __restrict__ scalars, int mont, uint32_t n,
                                                           int c, int W, uint32_t sink, int nsets, LiveSetArgs a,
                                                           uint4* __restrict__ scalars_std) {
    __shared__ uint32_t sh[256 * 9];
    uint32_t i = blockIdx.x * 256 + threadIdx.x;
    bool valid = i < n;
    Fr s = Fr::zero();
    bool live[MSM_MAX_SETS];
#pragma unroll
    for (int j = 0; j < MSM_MAX_SETS; j++) live[j] = valid && j < nsets && __ldg(a.rank[j] + i) != MSM_DEAD;
    if (valid) {
        uint4 x = __ldg(scalars + 2 * (size_t)i), y = __ldg(scalars + 2 * (size_t)i + 1);
        s.v[0] = x.x; s.v[1] = x.y; s.v[2] = x.z; s.v[3] = x.w;
        s.v[4] = y.x; s.v[5] = y.y; s.v[6] = y.z; s.v[7] = y.w;
        if (mont) s = from_mont(s);
        scalars_std[2 * (size_t)i] = make_uint4(s.v[0], s.v[1], s.v[2], s.v[3]);
        scalars_std[2 * (size_t)i + 1] = make_uint4(s.v[4], s.v[5], s.v[6], s.v[7]);
    }
    uint32_t* row = sh + threadIdx.x * 9;
#pragma unroll
    for (int j = 0; j < 8; j++) row[j] = s.v[j];
    unsigned lane = threadIdx.x & 31;
    for (int w = 0; w < W; w++) {
        int d = signed_digit(row, w, c);
        uint32_t key = d != 0 ? (uint32_t)w * a.key_stride + (uint32_t)(d < 0 ? -d : d) - 1u : sink;
#pragma unroll
        for (int j = 0; j < MSM_MAX_SETS; j++) {
            if (j >= nsets) break;
            uint32_t kj = live[j] ? key : NO_KEY;
            unsigned mask = __match_any_sync(0xffffffffu, kj);
            if (kj != NO_KEY && lane == (unsigned)(__ffs(mask) - 1)) atomicAdd(&a.counts[j][kj], (uint32_t)__popc(mask));
        }
    }
}

__global__ void __launch_bounds__(256) k_scatter_sets(const uint4* __restrict__ scalars_std, uint32_t n, int c, int W,
                                                      uint32_t sink, int nsets, LiveSetArgs a) {
    __shared__ uint32_t sh[256 * 9];
    uint32_t i = blockIdx.x * 256 + threadIdx.x;
    bool valid = i < n;
    uint32_t rank[MSM_MAX_SETS];
#pragma unroll
    for (int j = 0; j < MSM_MAX_SETS; j++) rank[j] = valid && j < nsets ? __ldg(a.rank[j] + i) : MSM_DEAD;
    uint32_t* row = sh + threadIdx.x * 9;
    if (valid) {
        uint4 x = scalars_std[2 * (size_t)i], y = scalars_std[2 * (size_t)i + 1];
        row[0] = x.x; row[1] = x.y; row[2] = x.z; row[3] = x.w;
        row[4] = y.x; row[5] = y.y; row[6] = y.z; row[7] = y.w;
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) row[j] = 0;
    }
    unsigned lane = threadIdx.x & 31;
    unsigned lt = (1u << lane) - 1u;
    for (int w = 0; w < W; w++) {
        int d = signed_digit(row, w, c);
        uint32_t key = d != 0 ? (uint32_t)w * a.key_stride + (uint32_t)(d < 0 ? -d : d) - 1u : sink;
        const uint32_t sign = d < 0 ? 0x80000000u : 0u;
#pragma unroll
        for (int j = 0; j < MSM_MAX_SETS; j++) {
            if (j >= nsets) break;
            uint32_t kj = rank[j] != MSM_DEAD ? key : NO_KEY;
            unsigned mask = __match_any_sync(0xffffffffu, kj);
            int leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (kj != NO_KEY && (int)lane == leader) base = atomicAdd(&a.cursor[j][kj], (uint32_t)__popc(mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (kj != NO_KEY) a.entries[j][base + __popc(mask & lt)] = ((uint32_t)w * a.rows[j] + rank[j]) | sign;
        }
    }
}

// ---- exclusive scan (three kernels) ----
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tot, uint32_t& total) {
    unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    unsigned nw = blockDim.x >> 5;
    if (wid == 0) {
        uint32_t t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= (unsigned)o) t += y;
        }
        if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    uint32_t before = wid ? warp_tot[wid - 1] : 0;
    total = warp_tot[nw - 1];
    __syncthreads();
    return before + x - v;
}

// 1024 elements per block of 256 threads (4 consecutive each)
__global__ void __launch_bounds__(256) k_scan_blocks(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                     uint32_t len, uint32_t* __restrict__ block_sums) {
    __shared__ uint32_t wt[32];
    size_t base = (size_t)blockIdx.x * 1024 + threadIdx.x * 4;
    uint32_t v[4], s = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        v[j] = base + j < len ? in[base + j] : 0;
        s += v[j];
    }
    uint32_t total;
    uint32_t pre = block_excl_scan(s, wt, total);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (base + j < len) out[base + j] = pre;
        pre += v[j];
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

// one block of 1024 threads scans nb block sums in place; writes the grand total
__global__ void __launch_bounds__(1024) k_scan_top(uint32_t* __restrict__ sums, uint32_t nb,
                                                   uint32_t* __restrict__ total_out) {
    __shared__ uint32_t wt[32];
    uint32_t per = (nb + 1023) / 1024;
    uint32_t lo = threadIdx.x * per, hi = min(lo + per, nb);
    uint32_t s = 0;
    for (uint32_t j = lo; j < hi; j++) s += sums[j];
    uint32_t total;
    uint32_t pre = block_excl_scan(s, wt, total);
    for (uint32_t j = lo; j < hi; j++) {
        uint32_t x = sums[j];
        sums[j] = pre;
        pre += x;
    }
    if (threadIdx.x == 0) *total_out = total;
}

__global__ void __launch_bounds__(256) k_scan_add(uint32_t* __restrict__ out, uint32_t len,
                                                  const uint32_t* __restrict__ sums,
                                                  const uint32_t* __restrict__ total) {
    size_t i = (size_t)blockIdx.x * 256 + threadIdx.x;
    if (i < len) out[i] += sums[i / 1024];
    if (i == 0) out[len] = *total;
}

// Partial sums per bucket (one per chunk the bucket touches).  Buckets with
// more than FAT_PARTIALS of them -- a repeated scalar, most often 1 -- go on
// the fat list and are folded in parallel before the bucket sums.
constexpr uint32_t FAT_PARTIALS = 16;
constexpr uint32_t FAT_JOBS = 64;

// partials per job of a fat bucket: at least one per thread of the folding
// block (FAT_JOB_MIN), at most FAT_JOBS jobs
constexpr uint32_t FAT_JOB_MIN = 128;
__device__ __forceinline__ uint32_t fat_job_len(uint32_t ns) {
    uint32_t j = (ns + FAT_JOBS - 1) / FAT_JOBS;
    return j < FAT_JOB_MIN ? FAT_JOB_MIN : j;
}

// Entries per accumulate thread, chosen on the device from the sorted count
// M and the K real buckets: at least L_min, no more than ACC_THREADS threads,
// and about M / (4 K) or more, so that an average bucket gets at most ~4
// partial sums and only skewed buckets (a repeated scalar such as 1) take the
// fat-bucket path.  Sparse scalars (witnesses of zeros and ones) still spread
// over the whole GPU.  Last, the chunks are fitted to whole waves of `wave`
// threads (one 512-thread G1 block per SM) when that saves 5% or more: a
// launch takes about (waves x L) additions per thread, so 2.4 waves of 16
// entries lose to 2 waves of 20 (a sparse witness MSM of the 2^21 prove).
constexpr uint32_t ACC_THREADS = 1u << 19;

__device__ __forceinline__ uint32_t chunk_len(uint32_t M, uint32_t K, uint32_t L_min, uint32_t wave) {
    uint32_t L = (uint32_t)(((uint64_t)M + ACC_THREADS - 1) / ACC_THREADS);
    uint32_t per_bucket = (uint32_t)(((uint64_t)M + 4ull * K - 1) / (4ull * K));
    if (per_bucket > L) L = per_bucket;
    if (L < L_min) L = L_min;
    if (wave && M) {
        const uint64_t chunks = ((uint64_t)M + L - 1) / L;
        const uint64_t waves = (chunks + wave - 1) / wave;
        if (waves > 1) {
            const uint64_t L2 = ((uint64_t)M + (waves - 1) * wave - 1) / ((waves - 1) * wave);
            // only for a clear gain: block times vary, and more, shorter waves balance better
            if (20 * (waves - 1) * L2 < 19 * waves * L) L = (uint32_t)L2;
        }
    }
    return L;
}

// partials per bucket for the Ks sorted buckets; only the K real ones can be
// fat (the constant-work sink bucket K is accumulated but never reduced).
// Also stores the chunk length L in total[3] for the kernels that follow.
__global__ void k_nseg(const uint32_t* __restrict__ offsets, uint32_t Ks, uint32_t K, uint32_t L_min, uint32_t wave,
                       uint32_t* __restrict__ nseg, uint32_t* __restrict__ fat_list, uint32_t* __restrict__ fat_count,
                       uint32_t* __restrict__ total) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t L = chunk_len(total[0], K, L_min, wave);
    if (g == 0) total[3] = L;
    if (g >= Ks) return;
    uint32_t lo = offsets[g], hi = offsets[g + 1];
    uint32_t ns = hi > lo ? ((hi - 1) / L - lo / L + 1) : 0;
    nseg[g] = ns;
    if (g < K && ns > FAT_PARTIALS) fat_list[atomicAdd(fat_count, 1u)] = g;
}

__global__ void k_copy_u32(uint32_t* dst, const uint32_t* src, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

// One MSM of a multi-segment space, as the accumulate kernel reads it.
struct MsmSegDev {
    const uint4* bases;   // window-shifted base table
    uint32_t key_start;   // first bucket of the segment in the space
    uint32_t n_bases;     // table entries
};

// ---- accumulate: one thread per chunk of L sorted entries ----
// LOCKSTEP: a block-wide barrier after every entry keeps the block's warps on
// the same instructions.  A fully inlined G1 madd is too long for the
// instruction cache, and warps that drift apart stall on instruction fetch
// (ncu: no_instruction was the top stall); in lockstep, one fetch serves the
// whole block.  G2 calls out-of-line Fq2 products and runs without it.
// MULTI: the buckets belong to several MSMs (segments, msm_space_*), each
// with its own base table; the segment of bucket g is the last one whose
// key_start is <= g, followed forward as g grows.
template <class F, bool LOCKSTEP, bool MULTI = false>
__device__ __forceinline__ void accumulate_chunks(const uint32_t* __restrict__ entries,
                                                  const uint32_t* __restrict__ offsets,
                                                  const uint32_t* __restrict__ seg_base, uint32_t K, uint32_t M,
                                                  uint32_t L, const uint4* __restrict__ bases, uint32_t base_offset,
                                                  uint32_t n_bases, uint4* __restrict__ partials,
                                                  unsigned long long* __restrict__ work,
                                                  const MsmSegDev* __restrict__ segs = nullptr, uint32_t nsegs = 0) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t start = t * L;
    const bool active = start < M;
    if (!LOCKSTEP && !active) return;
    size_t end = active ? (start + L < M ? start + L : M) : start;
    // last bucket g with offsets[g] <= start; then offsets[g+1] > start
    uint32_t g = 0, next = 0;
    if (active) {
        uint32_t lo = 0, hi = K;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (offsets[mid] <= start) lo = mid; else hi = mid;
        }
        g = lo;
        next = offsets[g + 1];
    }
    uint32_t si = 0, seg_end = 0xffffffffu;
    if (MULTI && active) {
        uint32_t lo = 0, hi = nsegs;
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (segs[mid].key_start <= g) lo = mid; else hi = mid;
        }
        si = lo;
        bases = segs[si].bases;
        n_bases = segs[si].n_bases;
        base_offset = 0;
        seg_end = si + 1 < nsegs ? segs[si + 1].key_start : 0xffffffffu;
    }
    Xyzz<F> acc = Xyzz<F>::identity();
    unsigned adds = 0;
    const size_t stop = LOCKSTEP ? start + L : end;   // lockstep: every thread runs L steps
    for (size_t k = start; k < stop; k++) {
        if (!LOCKSTEP || k < end) {
            if (k == next) {
                st_xyzz<F>(partials, seg_base[g] + (uint32_t)(t - offsets[g] / L), acc);
                acc = Xyzz<F>::identity();
                do {
                    g++;
                    next = offsets[g + 1];
                } while (next <= k);
                if (MULTI) {
                    while (g >= seg_end) {
                        si++;
                        bases = segs[si].bases;
                        n_bases = segs[si].n_bases;
                        seg_end = si + 1 < nsegs ? segs[si + 1].key_start : 0xffffffffu;
                    }
                }
            }
            uint32_t e = entries[k];
            if (k + 1 < end) {   // bring the next entry's base towards L1 while this one is added
                uint32_t nx = (entries[k + 1] & 0x7fffffffu) - base_offset;
                if (nx < n_bases)
                    asm volatile("prefetch.global.L1 [%0];" ::"l"(bases + (size_t)nx * (2 * Codec<F>::U4)));
            }
            uint32_t idx = e & 0x7fffffffu;
            if (idx >= base_offset && idx - base_offset < n_bases) {
                Affine<F> p = ld_affine<F>(bases, idx - base_offset);
                if (!p.is_inf()) {
                    if (e >> 31) p.y = neg(p.y);
                    // G1 keeps its products inlined; the Fq2 body is large enough
                    // that one out-of-line Fq2 product (three Fq chains) runs
                    // faster than inlined code that misses the instruction cache
                    acc = xyzz_add_affine<F, !std::is_same<F, Fq2>::value>(acc, p.x, p.y);
                    adds++;
                }
            }
        }
        if (LOCKSTEP) __syncthreads();
    }
    if (active) st_xyzz<F>(partials, seg_base[g] + (uint32_t)(t - offsets[g] / L), acc);
    // mixed additions performed, one atomic per warp (every lane reaches here in lockstep mode)
    unsigned mask = __activemask();
    unsigned total = __reduce_add_sync(mask, adds);
    if ((threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1) && total) atomicAdd(work, (unsigned long long)total);
}

constexpr int ACC_BLOCK_G1 = 512;   // lockstep block: 16 warps, one block per SM (<= 128 registers)
constexpr int ACC_BLOCK_G2 = 128;
// G2 accumulate blocks resident per SM that the register budget must allow
// (1: the compiler may take 255 registers, which leaves room for 2)
#ifndef ACC_G2_MIN_BLOCKS
#define ACC_G2_MIN_BLOCKS 1
#endif

// Multiprocessors of the current device (148 on a B200), cached per device.
static uint32_t device_sms() {
    static std::atomic<uint32_t> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    uint32_t v = cache[dev].load(std::memory_order_relaxed);
    if (!v) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 148;
        v = (uint32_t)sms;
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// Threads in one wave of G1 accumulate blocks on the current device (one
// block per SM), for chunk_len; 0 (no fitting) if the device cannot be read.
static uint32_t accumulate_wave() {
    static std::atomic<uint32_t> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    uint32_t w = cache[dev].load(std::memory_order_relaxed);
    if (!w) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return 0;
        w = (uint32_t)sms * ACC_BLOCK_G1;
        cache[dev].store(w, std::memory_order_relaxed);
    }
    return w;
}

__global__ void __launch_bounds__(ACC_BLOCK_G1, 1) k_accumulate_g1(const uint32_t* __restrict__ entries,
                                                                   const uint32_t* __restrict__ offsets,
                                                                   const uint32_t* __restrict__ seg_base, uint32_t K,
                                                                   const uint32_t* __restrict__ d_M,
                                                                   const uint32_t* __restrict__ d_L,
                                                                   const uint4* __restrict__ bases, uint32_t base_offset,
                                                                   uint32_t n_bases, uint4* __restrict__ partials,
                                                                   unsigned long long* __restrict__ work) {
    const uint32_t M = *d_M, L = *d_L;
    if ((size_t)blockIdx.x * blockDim.x * L >= M) return;   // the whole block has no entries
    accumulate_chunks<Fq, true>(entries, offsets, seg_base, K, M, L, bases, base_offset, n_bases, partials, work);
}

__global__ void __launch_bounds__(ACC_BLOCK_G2, ACC_G2_MIN_BLOCKS) k_accumulate_g2(const uint32_t* __restrict__ entries,
                                                               const uint32_t* __restrict__ offsets,
                                                               const uint32_t* __restrict__ seg_base, uint32_t K,
                                                               const uint32_t* __restrict__ d_M,
                                                               const uint32_t* __restrict__ d_L,
                                                               const uint4* __restrict__ bases, uint32_t base_offset,
                                                               uint32_t n_bases, uint4* __restrict__ partials,
                                                               unsigned long long* __restrict__ work) {
    accumulate_chunks<Fq2, false>(entries, offsets, seg_base, K, *d_M, *d_L, bases, base_offset, n_bases, partials,
                                  work);
}

__device__ __forceinline__ uint32_t n_partials(const uint32_t* offsets, uint32_t g, uint32_t L) {
    uint32_t lo = offsets[g], hi = offsets[g + 1];
    return hi > lo ? ((hi - 1) / L - lo / L + 1) : 0;
}

// Block-wide sum of one XYZZ point per thread through shared memory; the
// result is valid in thread 0.
template <class F>
__device__ __forceinline__ Xyzz<F> block_sum(Xyzz<F> acc, uint4* smem) {
    st_xyzz<F>(smem, threadIdx.x, acc);
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            acc = xyzz_add<F, false>(acc, ld_xyzz<F>(smem, threadIdx.x + s));
            st_xyzz<F>(smem, threadIdx.x, acc);
        }
        __syncthreads();
    }
    return acc;
}

// Fat buckets, stage 1: each of a fat bucket's partials is assigned to one of
// FAT_JOBS contiguous jobs; a block folds one job into the job's first slot.
template <class F>
__global__ void __launch_bounds__(128) k_fat_merge_jobs(uint4* __restrict__ partials,
                                                        const uint32_t* __restrict__ offsets,
                                                        const uint32_t* __restrict__ seg_base,
                                                        const uint32_t* __restrict__ fat_list,
                                                        const uint32_t* __restrict__ fat_count,
                                                        const uint32_t* __restrict__ d_L) {
    extern __shared__ uint4 smem[];
    const uint32_t L = *d_L;
    uint32_t items = *fat_count * FAT_JOBS;
    for (uint32_t item = blockIdx.x; item < items; item += gridDim.x) {
        uint32_t g = fat_list[item / FAT_JOBS], j = item % FAT_JOBS;
        uint32_t ns = n_partials(offsets, g, L), J = fat_job_len(ns);
        uint32_t a = j * J;
        if (a >= ns) continue;   // uniform across the block
        uint32_t b = min(a + J, ns), base = seg_base[g];
        Xyzz<F> acc = Xyzz<F>::identity();
        for (uint32_t i = a + threadIdx.x; i < b; i += blockDim.x) acc = xyzz_add<F, false>(acc, ld_xyzz<F>(partials, base + i));
        acc = block_sum(acc, smem);
        if (threadIdx.x == 0) st_xyzz<F>(partials, base + a, acc);
        __syncthreads();
    }
}

// Fat buckets, stage 2: fold the (at most FAT_JOBS) job results into the
// bucket's first partial slot.
template <class F>
__global__ void __launch_bounds__(64) k_fat_merge_final(uint4* __restrict__ partials,
                                                        const uint32_t* __restrict__ offsets,
                                                        const uint32_t* __restrict__ seg_base,
                                                        const uint32_t* __restrict__ fat_list,
                                                        const uint32_t* __restrict__ fat_count,
                                                        const uint32_t* __restrict__ d_L) {
    extern __shared__ uint4 smem[];
    const uint32_t L = *d_L;
    uint32_t nf = *fat_count;
    for (uint32_t f = blockIdx.x; f < nf; f += gridDim.x) {
        uint32_t g = fat_list[f];
        uint32_t ns = n_partials(offsets, g, L), J = fat_job_len(ns);
        uint32_t base = seg_base[g];
        uint32_t a = threadIdx.x * J;
        Xyzz<F> acc = a < ns ? ld_xyzz<F>(partials, base + a) : Xyzz<F>::identity();
        acc = block_sum(acc, smem);
        if (threadIdx.x == 0) st_xyzz<F>(partials, base, acc);
        __syncthreads();
    }
}

// Whether the bucket-sum and reduction kernels inline the G1 addition's
// products (G16_REDUCE_INLINE_G1=1) or call them out of line (the default).
#ifndef G16_REDUCE_INLINE_G1
#define G16_REDUCE_INLINE_G1 0
#endif
template <class F>
constexpr bool REDUCE_INL = std::is_same<F, g16d::Fq>::value && G16_REDUCE_INLINE_G1;
// Blocks per SM the bucket-sum and pieces kernels' register budget must allow.
#ifndef REDUCE_MIN_BLOCKS
#define REDUCE_MIN_BLOCKS 1
#endif

// Threads per k_bucket_sums block.
#ifndef G16_BUCKET_SUMS_BLOCK
#define G16_BUCKET_SUMS_BLOCK 128
#endif
constexpr unsigned BUCKET_SUMS_BLOCK = G16_BUCKET_SUMS_BLOCK;

// Bucket sums S_g: one thread per bucket folds its few partials (a fat
// bucket's total already sits in its first slot).
template <class F>
__global__ void __launch_bounds__(BUCKET_SUMS_BLOCK, REDUCE_MIN_BLOCKS) k_bucket_sums(const uint4* __restrict__ partials,
                                                     const uint32_t* __restrict__ offsets,
                                                     const uint32_t* __restrict__ seg_base, uint32_t K,
                                                     const uint32_t* __restrict__ d_L, uint4* __restrict__ buckets) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= K) return;
    const uint32_t L = *d_L;
    uint32_t ns = n_partials(offsets, g, L), base = seg_base[g];
    Xyzz<F> acc = Xyzz<F>::identity();
    if (ns > FAT_PARTIALS) {
        acc = ld_xyzz<F>(partials, base);
    } else {
        for (uint32_t s = 0; s < ns; s++) acc = xyzz_add<F, REDUCE_INL<F>>(acc, ld_xyzz<F>(partials, base + s));
    }
    st_xyzz<F>(buckets, g, acc);
}

// Bucket reduction, step 1.  A set's buckets S_0 .. S_{B-1} (S_b holds the
// points whose digit is b + 1) are cut into pieces of seg buckets; thread t of
// block j owns piece p = j 2^LB + t and folds it by running sums into
//   run_p = sum_i S_{p seg + i},   tot_p = sum_i (i + 1) S_{p seg + i},
// so that the set's sum_b (b + 1) S_b = sum_p tot_p + seg sum_p p run_p.
// The weights p are split over their bits instead of being multiplied out (a
// double-and-add per piece costs more than the piece's running sums): the
// block halves its 2^LB run values LB times in shared memory, v_t += v_(t+h)
// for h = 2^(LB-1) .. 1, and the upper half [h, 2h) that a halving reads holds
// exactly the folded values whose piece index has bit log2(h) set.  Once
// frozen, each upper half is summed by a tree that runs alongside the later
// halvings, so G_j = sum over the pieces with bit j set of run_p ends in slot
// 2^j after LB steps.  The tot values halve into T on the threads [h, 2h),
// which the run halving leaves idle (with seg = 1, tot = run and T = R).  Each
// step costs a thread at most one addition: a dependent XYZZ addition takes
// microseconds on an otherwise idle SM, so the depth is what counts here.
// The block writes T, G_0 .. G_(LB-1) and its run total R (LB + 2 points).
template <class F, int LB>
__global__ void __launch_bounds__(1 << LB, REDUCE_MIN_BLOCKS) k_reduce_pieces(const uint4* __restrict__ buckets, uint32_t B,
                                                           uint32_t seg, uint4* __restrict__ out) {
    constexpr uint32_t N = 1u << LB;
    extern __shared__ uint4 smem[];
    uint4* s_run = smem;
    uint4* s_tot = smem + N * 4 * Codec<F>::U4;
    const uint32_t t = threadIdx.x, set = blockIdx.y;
    const uint32_t p = blockIdx.x * N + t;
    const bool weighted = seg > 1;   // uniform: tot differs from run
    // G2: tot waits in shared memory while run is added, so that the two
    // 64-register points and the addition's operands fit without spilling
    constexpr bool TOT_SHARED = sizeof(F) > sizeof(g16d::Fq);
    Xyzz<F> run = Xyzz<F>::identity(), tot = Xyzz<F>::identity();
    if (TOT_SHARED && weighted) st_xyzz<F>(s_tot, t, tot);
    if ((size_t)p * seg < B) {
        const size_t g0 = (size_t)set * B + (size_t)p * seg;
#pragma unroll 1
        for (int i = (int)seg - 1; i >= 0; i--) {
            run = xyzz_add<F, REDUCE_INL<F>>(run, ld_xyzz<F>(buckets, g0 + i));
            if (weighted) {
                if constexpr (TOT_SHARED) st_xyzz<F>(s_tot, t, xyzz_add<F, REDUCE_INL<F>>(ld_xyzz<F>(s_tot, t), run));
                else tot = xyzz_add<F, REDUCE_INL<F>>(tot, run);
            }
        }
    }
    // run stays equal to slot t of s_run: thread t is the only writer of slot t
    st_xyzz<F>(s_run, t, run);
    if (!TOT_SHARED && weighted) st_xyzz<F>(s_tot, t, tot);
    const uint32_t lg = t ? 31 - __clz(t) : 0;   // slot t lies in the upper half [2^lg, 2^(lg+1))
#pragma unroll 1
    for (uint32_t k = 1; k <= (uint32_t)LB; k++) {
        __syncthreads();
        const uint32_t h = N >> k;
        // a step reads no slot that another thread writes in the same step:
        // run halving reads [h, 2h) and writes [0, h); the tot halving on
        // thread t in [h, 2h) reads t - h and t and writes t - h; the trees
        // stay at 2h and above
        if (t < h) {
            run = xyzz_add<F, REDUCE_INL<F>>(run, ld_xyzz<F>(s_run, t + h));
            st_xyzz<F>(s_run, t, run);
        } else if (t < 2 * h) {
            if (weighted) {
                tot = xyzz_add<F, REDUCE_INL<F>>(ld_xyzz<F>(s_tot, t - h), ld_xyzz<F>(s_tot, t));
                st_xyzz<F>(s_tot, t - h, tot);   // at the last step (t = 1) this is T
            }
        } else {
            // the half [2^lg, 2^(lg+1)) froze at step LB - lg; tree level k - (LB - lg) - 1 now
            const uint32_t hs = 1u << lg, s = 1u << (k - (LB - lg) - 1), o = t - hs;
            if ((o & (2 * s - 1)) == 0 && o + s < hs) {
                run = xyzz_add<F, REDUCE_INL<F>>(run, ld_xyzz<F>(s_run, t + s));
                st_xyzz<F>(s_run, t, run);
            }
        }
    }
    const size_t o0 = ((size_t)set * gridDim.x + blockIdx.x) * (LB + 2);
    if (t == 0) {
        if (!weighted) st_xyzz<F>(out, o0, run);
        st_xyzz<F>(out, o0 + LB + 1, run);
    } else if ((t & (t - 1)) == 0) {
        st_xyzz<F>(out, o0 + 1 + lg, run);   // G_lg
        if (t == 1 && weighted) st_xyzz<F>(out, o0, tot);
    }
}

// Bucket reduction, step 2 (when a set has more than a couple of blocks):
// block (o, set) sums one term over the set's nb blocks: o = 0 gives T,
// o = 1 .. LB gives G_(o-1), o = LB + 1 + i gives Gb_i, the sum of the run
// totals R of the blocks whose index has bit i set.  The host then forms
// T + seg (sum_j 2^j G_j + 2^LB sum_i 2^i Gb_i) by doublings and additions.
template <class F, int LB>
__global__ void __launch_bounds__(128) k_reduce_sets(const uint4* __restrict__ in, uint32_t nb,
                                                     uint4* __restrict__ out) {
    extern __shared__ uint4 smem[];
    const uint32_t o = blockIdx.x, set = blockIdx.y;
    const size_t base = (size_t)set * nb * (LB + 2);
    Xyzz<F> acc = Xyzz<F>::identity();
    for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x) {
        if (o <= (uint32_t)LB) acc = xyzz_add<F, false>(acc, ld_xyzz<F>(in, base + (size_t)j * (LB + 2) + o));
        else if ((j >> (o - LB - 1)) & 1u)
            acc = xyzz_add<F, false>(acc, ld_xyzz<F>(in, base + (size_t)j * (LB + 2) + LB + 1));
    }
    acc = block_sum(acc, smem);
    if (threadIdx.x == 0) st_xyzz<F>(out, (size_t)set * gridDim.x + o, acc);
}

// ---- batched MSMs: several scalar vectors, many MSMs, one launch per step ----
// A space holds the buckets of many MSMs (segments) back to back; sources are
// scalar vectors, each feeding up to MSM_MAX_TARGETS segments (the witness
// feeds A, B1 and L in the G1 space and B2 in the G2 space; an H vector feeds
// its H segment).  One digits pass and one scatter pass sort every source into
// every space; one accumulate launch per space adds every entry.

struct MsmTargetDev {
    uint32_t* counts;        // the space's sort buffers
    uint32_t* cursor;
    uint32_t* entries;
    const uint32_t* rank;    // scalar -> table row, MSM_DEAD where the base is infinity; nullptr: the scalar's index
    uint32_t key_start;      // the segment's first bucket in its space
    uint32_t rows;           // the segment's table rows
};

struct MsmSourceDev {
    const uint4* scalars;    // Montgomery Fr
    uint4* std_out;          // standard-form copy, for the scatter pass
    uint32_t n, c, W, ntargets;
    MsmTargetDev t[MSM_MAX_TARGETS];
};

// the source of block b: the last s with blk_start[s] <= b
__device__ __forceinline__ uint32_t source_of(const uint32_t* __restrict__ blk_start, uint32_t nsrc, uint32_t b) {
    uint32_t lo = 0, hi = nsrc;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (blk_start[mid] <= b) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_digits_multi(const MsmSourceDev* __restrict__ srcs,
                                                      const uint32_t* __restrict__ blk_start, uint32_t nsrc) {
    __shared__ uint32_t sh[256 * 9];
    const uint32_t si = source_of(blk_start, nsrc, blockIdx.x);
    const MsmSourceDev& S = srcs[si];
    const uint32_t i = (blockIdx.x - blk_start[si]) * 256 + threadIdx.x;
    const bool valid = i < S.n;
    const uint32_t nt = S.ntargets, c = S.c, W = S.W;
    Fr x = Fr::zero();
    bool live[MSM_MAX_TARGETS];
#pragma unroll
    for (int j = 0; j < MSM_MAX_TARGETS; j++)
        live[j] = valid && (uint32_t)j < nt && (!S.t[j].rank || __ldg(S.t[j].rank + i) != MSM_DEAD);
    if (valid) {
        uint4 a = __ldg(S.scalars + 2 * (size_t)i), b = __ldg(S.scalars + 2 * (size_t)i + 1);
        x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
        x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
        x = from_mont(x);
        S.std_out[2 * (size_t)i] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
        S.std_out[2 * (size_t)i + 1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
    }
    uint32_t* row = sh + threadIdx.x * 9;
#pragma unroll
    for (int j = 0; j < 8; j++) row[j] = x.v[j];
    const unsigned lane = threadIdx.x & 31;
    for (uint32_t w = 0; w < W; w++) {
        const int d = signed_digit(row, (int)w, (int)c);
        const uint32_t key = d != 0 ? (uint32_t)(d < 0 ? -d : d) - 1u : NO_KEY;
#pragma unroll
        for (int j = 0; j < MSM_MAX_TARGETS; j++) {
            if ((uint32_t)j >= nt) break;
            const uint32_t kj = live[j] && key != NO_KEY ? S.t[j].key_start + key : NO_KEY;
            const unsigned mask = __match_any_sync(0xffffffffu, kj);
            if (kj != NO_KEY && lane == (unsigned)(__ffs(mask) - 1)) atomicAdd(&S.t[j].counts[kj], (uint32_t)__popc(mask));
        }
    }
}

__global__ void __launch_bounds__(256) k_scatter_multi(const MsmSourceDev* __restrict__ srcs,
                                                       const uint32_t* __restrict__ blk_start, uint32_t nsrc) {
    __shared__ uint32_t sh[256 * 9];
    const uint32_t si = source_of(blk_start, nsrc, blockIdx.x);
    const MsmSourceDev& S = srcs[si];
    const uint32_t i = (blockIdx.x - blk_start[si]) * 256 + threadIdx.x;
    const bool valid = i < S.n;
    const uint32_t nt = S.ntargets, c = S.c, W = S.W;
    uint32_t rowi[MSM_MAX_TARGETS];
#pragma unroll
    for (int j = 0; j < MSM_MAX_TARGETS; j++)
        rowi[j] = valid && (uint32_t)j < nt ? (S.t[j].rank ? __ldg(S.t[j].rank + i) : i) : MSM_DEAD;
    uint32_t* row = sh + threadIdx.x * 9;
    if (valid) {
        uint4 a = S.std_out[2 * (size_t)i], b = S.std_out[2 * (size_t)i + 1];
        row[0] = a.x; row[1] = a.y; row[2] = a.z; row[3] = a.w;
        row[4] = b.x; row[5] = b.y; row[6] = b.z; row[7] = b.w;
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) row[j] = 0;
    }
    const unsigned lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
    for (uint32_t w = 0; w < W; w++) {
        const int d = signed_digit(row, (int)w, (int)c);
        const uint32_t key = d != 0 ? (uint32_t)(d < 0 ? -d : d) - 1u : NO_KEY;
        const uint32_t sign = d < 0 ? 0x80000000u : 0u;
#pragma unroll
        for (int j = 0; j < MSM_MAX_TARGETS; j++) {
            if ((uint32_t)j >= nt) break;
            const uint32_t kj = rowi[j] != MSM_DEAD && key != NO_KEY ? S.t[j].key_start + key : NO_KEY;
            const unsigned mask = __match_any_sync(0xffffffffu, kj);
            const int leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (kj != NO_KEY && (int)lane == leader) base = atomicAdd(&S.t[j].cursor[kj], (uint32_t)__popc(mask));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (kj != NO_KEY) S.t[j].entries[base + __popc(mask & lt)] = (w * S.t[j].rows + rowi[j]) | sign;
        }
    }
}

__global__ void __launch_bounds__(ACC_BLOCK_G1, 1) k_accumulate_multi_g1(const uint32_t* __restrict__ entries,
                                                                         const uint32_t* __restrict__ offsets,
                                                                         const uint32_t* __restrict__ seg_base,
                                                                         uint32_t K, const uint32_t* __restrict__ d_M,
                                                                         const uint32_t* __restrict__ d_L,
                                                                         const MsmSegDev* __restrict__ segs,
                                                                         uint32_t nsegs, uint4* __restrict__ partials,
                                                                         unsigned long long* __restrict__ work) {
    const uint32_t M = *d_M, L = *d_L;
    if ((size_t)blockIdx.x * blockDim.x * L >= M) return;   // the whole block has no entries
    accumulate_chunks<Fq, true, true>(entries, offsets, seg_base, K, M, L, nullptr, 0, 0, partials, work, segs,
                                      nsegs);
}

__global__ void __launch_bounds__(ACC_BLOCK_G2, ACC_G2_MIN_BLOCKS) k_accumulate_multi_g2(const uint32_t* __restrict__ entries,
                                                                     const uint32_t* __restrict__ offsets,
                                                                     const uint32_t* __restrict__ seg_base,
                                                                     uint32_t K, const uint32_t* __restrict__ d_M,
                                                                     const uint32_t* __restrict__ d_L,
                                                                     const MsmSegDev* __restrict__ segs,
                                                                     uint32_t nsegs, uint4* __restrict__ partials,
                                                                     unsigned long long* __restrict__ work) {
    accumulate_chunks<Fq2, false, true>(entries, offsets, seg_base, K, *d_M, *d_L, nullptr, 0, 0, partials, work,
                                        segs, nsegs);
}

// The bucket reduction of one segment of a space (msm_reduce_plan with one set).
struct MsmReduceDev {
    uint32_t key_start, B, seg, nb, hb;
    uint32_t block_start;   // its first k_reduce_pieces_multi block
    uint32_t out_block;     // its first point in the blocks' output
    uint32_t out_set;       // its first point in the sets' output
};

// k_reduce_pieces for many segments: block b works on block b - block_start
// of the segment that owns it, with that segment's B and seg.
template <class F, int LB>
__global__ void __launch_bounds__(1 << LB, REDUCE_MIN_BLOCKS) k_reduce_pieces_multi(const uint4* __restrict__ buckets,
                                                                 const MsmReduceDev* __restrict__ segs,
                                                                 uint32_t nsegs, uint4* __restrict__ out) {
    constexpr uint32_t N = 1u << LB;
    extern __shared__ uint4 smem[];
    uint4* s_run = smem;
    uint4* s_tot = smem + N * 4 * Codec<F>::U4;
    uint32_t lo = 0, hi = nsegs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (segs[mid].block_start <= blockIdx.x) lo = mid; else hi = mid;
    }
    const MsmReduceDev sd = segs[lo];
    const uint32_t t = threadIdx.x, jb = blockIdx.x - sd.block_start;
    const uint32_t p = jb * N + t, seg = sd.seg, B = sd.B;
    const bool weighted = seg > 1;
    constexpr bool TOT_SHARED = sizeof(F) > sizeof(g16d::Fq);
    Xyzz<F> run = Xyzz<F>::identity(), tot = Xyzz<F>::identity();
    if (TOT_SHARED && weighted) st_xyzz<F>(s_tot, t, tot);
    if ((size_t)p * seg < B) {
        const size_t g0 = (size_t)sd.key_start + (size_t)p * seg;
#pragma unroll 1
        for (int i = (int)seg - 1; i >= 0; i--) {
            run = xyzz_add<F, REDUCE_INL<F>>(run, ld_xyzz<F>(buckets, g0 + i));
            if (weighted) {
                if constexpr (TOT_SHARED) st_xyzz<F>(s_tot, t, xyzz_add<F, REDUCE_INL<F>>(ld_xyzz<F>(s_tot, t), run));
                else tot = xyzz_add<F, REDUCE_INL<F>>(tot, run);
            }
        }
    }
    st_xyzz<F>(s_run, t, run);
    if (!TOT_SHARED && weighted) st_xyzz<F>(s_tot, t, tot);
    const uint32_t lg = t ? 31 - __clz(t) : 0;
#pragma unroll 1
    for (uint32_t k = 1; k <= (uint32_t)LB; k++) {
        __syncthreads();
        const uint32_t h = N >> k;
        if (t < h) {
            run = xyzz_add<F, REDUCE_INL<F>>(run, ld_xyzz<F>(s_run, t + h));
            st_xyzz<F>(s_run, t, run);
        } else if (t < 2 * h) {
            if (weighted) {
                tot = xyzz_add<F, REDUCE_INL<F>>(ld_xyzz<F>(s_tot, t - h), ld_xyzz<F>(s_tot, t));
                st_xyzz<F>(s_tot, t - h, tot);
            }
        } else {
            const uint32_t hs = 1u << lg, s2 = 1u << (k - (LB - lg) - 1), o = t - hs;
            if ((o & (2 * s2 - 1)) == 0 && o + s2 < hs) {
                run = xyzz_add<F, REDUCE_INL<F>>(run, ld_xyzz<F>(s_run, t + s2));
                st_xyzz<F>(s_run, t, run);
            }
        }
    }
    const size_t o0 = (size_t)sd.out_block + (size_t)jb * (LB + 2);
    if (t == 0) {
        if (!weighted) st_xyzz<F>(out, o0, run);
        st_xyzz<F>(out, o0 + LB + 1, run);
    } else if ((t & (t - 1)) == 0) {
        st_xyzz<F>(out, o0 + 1 + lg, run);
        if (t == 1 && weighted) st_xyzz<F>(out, o0, tot);
    }
}

// k_reduce_sets for many segments: blockIdx.y picks the segment, blockIdx.x
// the term (T, G_0 .. G_(LB-1), Gb_0 .. Gb_(hb-1)); terms past the segment's
// own hb leave at once.
template <class F, int LB>
__global__ void __launch_bounds__(128) k_reduce_sets_multi(const uint4* __restrict__ in,
                                                           const MsmReduceDev* __restrict__ segs,
                                                           uint4* __restrict__ out) {
    extern __shared__ uint4 smem[];
    const MsmReduceDev sd = segs[blockIdx.y];
    const uint32_t o = blockIdx.x;
    if (o >= (uint32_t)LB + 1 + sd.hb) return;   // uniform across the block
    const size_t base = sd.out_block;
    Xyzz<F> acc = Xyzz<F>::identity();
    for (uint32_t j = threadIdx.x; j < sd.nb; j += blockDim.x) {
        if (o <= (uint32_t)LB) acc = xyzz_add<F, false>(acc, ld_xyzz<F>(in, base + (size_t)j * (LB + 2) + o));
        else if ((j >> (o - LB - 1)) & 1u)
            acc = xyzz_add<F, false>(acc, ld_xyzz<F>(in, base + (size_t)j * (LB + 2) + LB + 1));
    }
    acc = block_sum(acc, smem);
    if (threadIdx.x == 0) st_xyzz<F>(out, (size_t)sd.out_set + o, acc);
}

// Window-shifted base table: out[w n + i] = 2^(c w) P_i (affine).  Built once
// per prepared key in two steps, so that the normalisations share inversions.
//
// Step 1, one thread per point: window 0 is P_i itself (written affine), and
// the XYZZ multiples 2^(c w) P_i for w >= 1 (c doublings each) go to tmp at
// (w - 1) n + i; a point at infinity (or below skip) gives zeros / identity.
template <class F>
__global__ void __launch_bounds__(128) k_window_xyzz(const uint4* __restrict__ in, uint32_t n, uint32_t skip, int c,
                                                     int W, uint4* __restrict__ out, uint4* __restrict__ tmp) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Affine<F> p;
    bool inf = i < skip;
    if (!inf) {
        p = ld_affine<F>(in, i - skip);
        inf = p.is_inf();
    }
    if (inf) {
        st_affine<F>(out, i, F::zero(), F::zero());
        for (int w = 1; w < W; w++) st_xyzz<F>(tmp, (size_t)(w - 1) * n + i, Xyzz<F>::identity());
        return;
    }
    st_affine<F>(out, i, p.x, p.y);
    Xyzz<F> acc;
    acc.x = p.x;
    acc.y = p.y;
    acc.zz = F::one();
    acc.zzz = F::one();
    for (int w = 1; w < W; w++) {
        for (int j = 0; j < c; j++) acc = xyzz_dbl<F, false>(acc);
        st_xyzz<F>(tmp, (size_t)(w - 1) * n + i, acc);
    }
}

// Step 2, Montgomery's batch inversion over runs of NORM_RUN consecutive
// entries: one inversion per run instead of one per entry.  With
// d_j = ZZ_j ZZZ_j, x = X ZZZ / d and y = Y ZZ / d.  The output slots hold the
// running products (x) and d_j (y) between the forward and the backward pass;
// an identity entry (ZZ = 0) takes d = 1 and is written as zeros.
constexpr uint32_t NORM_RUN = 32;

template <class F>
__global__ void __launch_bounds__(128) k_window_normalize(const uint4* __restrict__ tmp, size_t count,
                                                          uint4* __restrict__ out) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t a = t * NORM_RUN;
    if (a >= count) return;
    size_t b = a + NORM_RUN < count ? a + NORM_RUN : count;
    F acc = F::one();
    for (size_t j = a; j < b; j++) {
        Xyzz<F> q = ld_xyzz<F>(tmp, j);
        F d = q.zz.is_zero() ? F::one() : fmul<false>(q.zz, q.zzz);
        acc = fmul<false>(acc, d);
        st_affine<F>(out, j, acc, d);
    }
    F inv_acc = inv(acc);   // 1 / (d_a ... d_(b-1))
    for (size_t j = b; j-- > a;) {
        Affine<F> slot = ld_affine_rw<F>(out, j);   // (running product through j, d_j)
        F before = j > a ? ld_affine_rw<F>(out, j - 1).x : F::one();
        F inv_d = fmul<false>(inv_acc, before);   // 1 / d_j
        inv_acc = fmul<false>(inv_acc, slot.y);   // 1 / (d_a ... d_(j-1))
        Xyzz<F> q = ld_xyzz<F>(tmp, j);
        if (q.zz.is_zero()) {
            st_affine<F>(out, j, F::zero(), F::zero());
        } else {
            F x, y;
            fmul2<false>(q.x, q.zzz, q.y, q.zz, x, y);
            fmul2<false>(x, inv_d, y, inv_d, x, y);
            st_affine<F>(out, j, x, y);
        }
    }
}

// Fixed-base multiplication for key generation: P_i = k_i G with 8-bit windows,
// table[w * 256 + d] = d 2^(8 w) G (affine; d = 0 unused), k_i Montgomery Fr.
// The XYZZ result goes to tmp for k_window_normalize.
template <class F>
__global__ void __launch_bounds__(128) k_fixed_base(const uint4* __restrict__ table, const uint4* __restrict__ scalars,
                                                    size_t n, uint4* __restrict__ tmp) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr k;
    uint4 a = __ldg(scalars + 2 * i), b = __ldg(scalars + 2 * i + 1);
    k.v[0] = a.x; k.v[1] = a.y; k.v[2] = a.z; k.v[3] = a.w;
    k.v[4] = b.x; k.v[5] = b.y; k.v[6] = b.z; k.v[7] = b.w;
    k = from_mont(k);
    Xyzz<F> acc = Xyzz<F>::identity();
    for (int w = 0; w < 32; w++) {
        uint32_t d = (k.v[w >> 2] >> (8 * (w & 3))) & 255u;
        if (d) {
            Affine<F> p = ld_affine<F>(table, (size_t)w * 256 + d);
            acc = xyzz_add_affine<F, !std::is_same<F, Fq2>::value>(acc, p.x, p.y);
        }
    }
    st_xyzz<F>(tmp, i, acc);
}

}  // namespace g16d

namespace g16 {

using namespace g16d;

void MsmSort::release() {
    cudaFree(d_scalars_std);
    cudaFree(d_counts);
    cudaFree(d_offsets);
    cudaFree(d_cursor);
    cudaFree(d_seg_base);
    cudaFree(d_fat_list);
    cudaFree(d_scan_tmp);
    cudaFree(d_entries);
    cudaFree(d_total);
    *this = MsmSort();
}

void MsmAccum::release() {
    cudaFree(d_work);
    cudaFree(d_buckets);
    cudaFree(d_partials);
    cudaFree(d_segments);
    cudaFree(d_windows);
    *this = MsmAccum();
}

int msm_shared_window_bits(size_t m) {
    int best = 8;
    double best_cost = 1e300;
    for (int c = 8; c <= 22; c++) {
        double cost = (double)m * msm_windows(c) + 3.0 * (double)(1u << (c - 1));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

template <class F>
static cudaError_t window_table(const void* d_in, size_t n, uint32_t skip, int c, void* d_out, cudaStream_t st,
                                size_t xyzz_bytes) {
    const int W = msm_windows(c);
    const size_t count = n * (size_t)(W - 1);
    void* tmp = nullptr;
    G16_CUDA(g16::dev_malloc(&tmp, (count ? count : 1) * xyzz_bytes));
    cudaError_t e = cudaSuccess;
    {
        TimedLaunch tl("msm_window_table", st);
        k_window_xyzz<F><<<blocks_for(n, 128), 128, 0, st>>>((const uint4*)d_in, (uint32_t)n, skip, c, W,
                                                            (uint4*)d_out, (uint4*)tmp);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess && count) {
        TimedLaunch tl("msm_window_table", st);
        uint4* out1 = (uint4*)((uint8_t*)d_out + n * (xyzz_bytes / 2));   // window 1 onwards
        k_window_normalize<F><<<blocks_for((count + NORM_RUN - 1) / NORM_RUN, 128), 128, 0, st>>>(
            (const uint4*)tmp, count, out1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    return e;
}

template <class F>
static cudaError_t fixed_base(const void* d_table, const void* d_scalars, size_t n, void* d_out, cudaStream_t st,
                              size_t xyzz_bytes) {
    if (!n) return cudaSuccess;
    void* tmp = nullptr;
    G16_CUDA(g16::dev_malloc(&tmp, n * xyzz_bytes));
    cudaError_t e;
    {
        TimedLaunch tl("fixed_base", st);
        k_fixed_base<F><<<blocks_for(n, 128), 128, 0, st>>>((const uint4*)d_table, (const uint4*)d_scalars, n,
                                                            (uint4*)tmp);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) {
        TimedLaunch tl("fixed_base", st);
        k_window_normalize<F><<<blocks_for((n + NORM_RUN - 1) / NORM_RUN, 128), 128, 0, st>>>((const uint4*)tmp, n,
                                                                                            (uint4*)d_out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    return e;
}

cudaError_t fixed_base_g1(const void* d_table, const void* d_scalars, size_t n, void* d_out, cudaStream_t st) {
    return fixed_base<g16d::Fq>(d_table, d_scalars, n, d_out, st, XYZZ_G1_BYTES);
}

cudaError_t fixed_base_g2(const void* d_table, const void* d_scalars, size_t n, void* d_out, cudaStream_t st) {
    return fixed_base<g16d::Fq2>(d_table, d_scalars, n, d_out, st, XYZZ_G2_BYTES);
}

cudaError_t msm_window_table_g1(const void* d_in, size_t n, uint32_t skip, int c, void* d_out, cudaStream_t st) {
    return window_table<g16d::Fq>(d_in, n, skip, c, d_out, st, XYZZ_G1_BYTES);
}

cudaError_t msm_window_table_g2(const void* d_in, size_t n, uint32_t skip, int c, void* d_out, cudaStream_t st) {
    return window_table<g16d::Fq2>(d_in, n, skip, c, d_out, st, XYZZ_G2_BYTES);
}

int msm_window_bits(size_t m) {
    // cost ~ windows * (m + 2 * buckets): bucket reduction runs fully parallel
    // on the device, so buckets weigh less than the reference CPU model's 3
    int best = 8;
    double best_cost = 1e300;
    for (int c = 8; c <= 18; c++) {
        double windows = (255 + c - 1) / c;
        double cost = windows * ((double)m + 2.0 * (double)(1u << (c - 1)));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

// Buffers that are views (fixed) are never reallocated: too small is an error.
static cudaError_t fixed_too_small(size_t need_bytes, size_t cap_bytes) {
    set_error("fixed MSM scratch holds %zu bytes where %zu are needed", cap_bytes, need_bytes);
    return cudaErrorInvalidValue;
}

// Grow-only scratch, reallocated in stream order on st (dev_realloc_async).
template <class T>
static cudaError_t grow(cudaStream_t st, T*& p, size_t& cap, size_t need_elems, bool fixed = false) {
    if (need_elems <= cap && p) return cudaSuccess;
    if (fixed) return fixed_too_small(need_elems * sizeof(T), cap * sizeof(T));
    cap = 0;
    size_t n = need_elems + need_elems / 8 + 64;
    cudaError_t e = g16::dev_realloc_async(&p, n * sizeof(T), st, false);
    if (e != cudaSuccess) {
        cap = 0;
        set_error("cudaMalloc of %zu bytes for MSM scratch failed: %s", n * sizeof(T), cudaGetErrorString(e));
        return e;
    }
    cap = n;
    return cudaSuccess;
}

static cudaError_t grow_bytes(cudaStream_t st, void*& p, size_t& cap, size_t need, bool fixed = false) {
    if (need <= cap && p) return cudaSuccess;
    if (fixed) return fixed_too_small(need, cap);
    cap = 0;
    size_t n = need + need / 8 + 256;
    cudaError_t e = g16::dev_realloc_async(&p, n, st, true);
    if (e != cudaSuccess) {
        cap = 0;
        set_error("cudaMalloc of %zu bytes for MSM scratch failed: %s", n, cudaGetErrorString(e));
        return e;
    }
    cap = n;
    return cudaSuccess;
}

// exclusive scan of in[0..len) into out[0..len] (out[len] = total); total also to *d_total
static cudaError_t scan(const uint32_t* in, uint32_t* out, uint32_t len, uint32_t* tmp, uint32_t* d_total,
                        cudaStream_t st) {
    uint32_t nb = (len + 1023) / 1024;
    if (nb == 0) nb = 1;
    {
        TimedLaunch tl("msm_scan", st);
        k_scan_blocks<<<nb, 256, 0, st>>>(in, out, len, tmp);
    }
    {
        TimedLaunch tl("msm_scan", st);
        k_scan_top<<<1, 1024, 0, st>>>(tmp, nb, d_total);
    }
    {
        TimedLaunch tl("msm_scan", st);
        k_scan_add<<<blocks_for(len ? len : 1, 256), 256, 0, st>>>(out, len, tmp, d_total);
    }
    return cudaGetLastError();
}

cudaError_t msm_sort(MsmSort& s, const void* d_scalars, size_t n, bool montgomery, int c, cudaStream_t st,
                     bool shared_windows, bool constant_work) {
    if (c == 0) c = msm_window_bits(n);
    if (c < 4 || c > 24) {
        set_error("MSM window of %d bits outside [4, 24]", c);
        return cudaErrorInvalidValue;
    }
    s.c = c;
    s.W = (255 + c - 1) / c;
    s.B = 1u << (c - 1);
    s.shared = shared_windows;
    s.K = shared_windows ? s.B : (uint32_t)s.W * s.B;
    s.constant_work = constant_work;
    s.Ks = s.K + (constant_work ? 1u : 0u);
    s.n = n;
    if ((shared_windows ? n * (size_t)s.W : n) >= 0x80000000ull) {
        set_error("MSM of %zu points x %d windows exceeds the 2^31 entry-index limit", n, s.W);
        return cudaErrorInvalidValue;
    }
    // the smallest chunk the accumulate may use (buffers are sized for it);
    // the one it does use is chosen on the device from the entry count (k_nseg)
    s.chunk = 16;
    const uint32_t kw = shared_windows ? 0u : s.B, ew = shared_windows ? (uint32_t)n : 0u;
    const uint32_t sink = constant_work ? s.K : NO_KEY;
    size_t nn = n ? n : 1;
    G16_CUDA(grow(st, s.d_scalars_std, s.cap_scalars, nn * 8, s.fixed));
    size_t kk = (size_t)s.Ks + 1;
    if (s.fixed && (kk > s.cap_k || !s.d_counts || !s.d_offsets || !s.d_cursor || !s.d_seg_base || !s.d_fat_list))
        G16_CUDA(fixed_too_small(kk * sizeof(uint32_t), s.cap_k * sizeof(uint32_t)));
    if (kk > s.cap_k || !s.d_counts) {
        size_t cap = 0;
        G16_CUDA(grow(st, s.d_counts, cap, kk));
        cap = 0;
        G16_CUDA(grow(st, s.d_offsets, cap, kk));
        cap = 0;
        G16_CUDA(grow(st, s.d_cursor, cap, kk));
        cap = 0;
        G16_CUDA(grow(st, s.d_seg_base, cap, kk));
        cap = 0;
        G16_CUDA(grow(st, s.d_fat_list, cap, kk));
        s.cap_k = cap;
    }
    G16_CUDA(grow(st, s.d_scan_tmp, s.cap_tmp, kk / 1024 + 2, s.fixed));
    G16_CUDA(grow(st, s.d_entries, s.cap_entries, nn * s.W, s.fixed));
    if (!s.d_total) {
        if (s.fixed) G16_CUDA(fixed_too_small(4 * sizeof(uint32_t), 0));
        G16_CUDA(g16::dev_realloc_async(&s.d_total, 4 * sizeof(uint32_t), st, false));
    }

    G16_CUDA(cudaMemsetAsync(s.d_counts, 0, kk * sizeof(uint32_t), st));
    G16_CUDA(cudaMemsetAsync(s.d_total, 0, 4 * sizeof(uint32_t), st));
    if (n) {
        timer().add_bytes("msm_digits", 64.0 * n);   // scalars in, standard-form copy out
        TimedLaunch tl("msm_digits", st);
        k_digits_count<<<blocks_for(n, 256), 256, 0, st>>>((const uint4*)d_scalars, montgomery ? 1 : 0, (uint32_t)n,
                                                          c, s.W, kw, sink, (uint4*)s.d_scalars_std, s.d_counts);
    }
    G16_CUDA(cudaGetLastError());
    G16_CUDA(scan(s.d_counts, s.d_offsets, s.Ks, s.d_scan_tmp, s.d_total, st));
    {
        TimedLaunch tl("msm_copy", st);
        k_copy_u32<<<blocks_for(s.Ks, 256), 256, 0, st>>>(s.d_cursor, s.d_offsets, s.Ks);
    }
    if (n) {
        TimedLaunch tl("msm_scatter", st);
        k_scatter<<<blocks_for(n, 256), 256, 0, st>>>((const uint4*)s.d_scalars_std, (uint32_t)n, c, s.W, kw, ew,
                                                     sink, s.d_cursor, s.d_entries);
    }
    G16_CUDA(cudaGetLastError());
    // per-bucket segment counts -> segment base (into counts, then scanned)
    {
        TimedLaunch tl("msm_nseg", st);
        k_nseg<<<blocks_for(s.Ks, 256), 256, 0, st>>>(s.d_offsets, s.Ks, s.K, s.chunk, accumulate_wave(),
                                                       s.d_counts, s.d_fat_list, s.d_total + 2, s.d_total);
    }
    G16_CUDA(scan(s.d_counts, s.d_seg_base, s.Ks, s.d_scan_tmp, s.d_total + 1, st));
    return cudaSuccess;
}

cudaError_t msm_sort_sets(MsmSort* sorts, const MsmLiveSets& sets, const void* d_scalars, size_t n, bool montgomery,
                          int c, cudaStream_t st, bool constant_work, bool shared) {
    if (sets.count < 1 || sets.count > MSM_MAX_SETS) {
        set_error("%d live sets (1 to %d)", sets.count, MSM_MAX_SETS);
        return cudaErrorInvalidValue;
    }
    if (c < 4 || c > 24) {
        set_error("MSM window of %d bits outside [4, 24]", c);
        return cudaErrorInvalidValue;
    }
    const int W = (255 + c - 1) / c;
    if (n >= 0x80000000ull) {
        set_error("MSM of %zu scalars exceeds the 2^31 index limit", n);
        return cudaErrorInvalidValue;
    }
    LiveSetArgs a = {};
    for (int j = 0; j < sets.count; j++) {
        MsmSort& s = sorts[j];
        s.c = c;
        s.W = W;
        s.B = 1u << (c - 1);
        s.shared = shared;
        s.K = shared ? s.B : (uint32_t)W * s.B;
        s.constant_work = constant_work;
        s.Ks = s.K + (constant_work ? 1u : 0u);
        s.n = sets.rows[j];
        s.chunk = 16;
        if ((size_t)sets.rows[j] * (size_t)W >= 0x80000000ull || sets.rows[j] > n) {
            set_error("live set of %u rows x %d windows exceeds the 2^31 entry-index limit", sets.rows[j], W);
            return cudaErrorInvalidValue;
        }
        const size_t kk = (size_t)s.Ks + 1;
        if (kk > s.cap_k || !s.d_counts) {
            size_t cap = 0;
            G16_CUDA(grow(st, s.d_counts, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_offsets, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_cursor, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_seg_base, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_fat_list, cap, kk));
            s.cap_k = cap;
        }
        G16_CUDA(grow(st, s.d_scan_tmp, s.cap_tmp, kk / 1024 + 2));
        G16_CUDA(grow(st, s.d_entries, s.cap_entries, (size_t)(sets.rows[j] ? sets.rows[j] : 1) * W));
        if (!s.d_total) G16_CUDA(g16::dev_realloc_async(&s.d_total, 4 * sizeof(uint32_t), st, false));
        G16_CUDA(cudaMemsetAsync(s.d_counts, 0, kk * sizeof(uint32_t), st));
        G16_CUDA(cudaMemsetAsync(s.d_total, 0, 4 * sizeof(uint32_t), st));
        a.rank[j] = sets.d_rank[j];
        a.counts[j] = s.d_counts;
        a.cursor[j] = s.d_cursor;
        a.entries[j] = s.d_entries;
        a.rows[j] = shared ? sets.rows[j] : 0u;
    }
    a.key_stride = shared ? 0u : (1u << (c - 1));
    // the standard-form copy of the scalars, shared by the sets, lives in the first
    MsmSort& s0 = sorts[0];
    G16_CUDA(grow(st, s0.d_scalars_std, s0.cap_scalars, (n ? n : 1) * 8));
    const uint32_t sink = constant_work ? sorts[0].K : NO_KEY;
    if (n) {
        timer().add_bytes("msm_digits", 64.0 * n);   // scalars in, standard-form copy out
        TimedLaunch tl("msm_digits", st);
        k_digits_count_sets<<<blocks_for(n, 256), 256, 0, st>>>((const uint4*)d_scalars, montgomery ? 1 : 0,
                                                               (uint32_t)n, c, W, sink, sets.count, a,
                                                               (uint4*)s0.d_scalars_std);
    }
    G16_CUDA(cudaGetLastError());
    for (int j = 0; j < sets.count; j++) {
        MsmSort& s = sorts[j];
        G16_CUDA(scan(s.d_counts, s.d_offsets, s.Ks, s.d_scan_tmp, s.d_total, st));
        TimedLaunch tl("msm_copy", st);
        k_copy_u32<<<blocks_for(s.Ks, 256), 256, 0, st>>>(s.d_cursor, s.d_offsets, s.Ks);
    }
    if (n) {
        TimedLaunch tl("msm_scatter", st);
        k_scatter_sets<<<blocks_for(n, 256), 256, 0, st>>>((const uint4*)s0.d_scalars_std, (uint32_t)n, c, W, sink,
                                                          sets.count, a);
    }
    G16_CUDA(cudaGetLastError());
    for (int j = 0; j < sets.count; j++) {
        MsmSort& s = sorts[j];
        {
            TimedLaunch tl("msm_nseg", st);
            k_nseg<<<blocks_for(s.Ks, 256), 256, 0, st>>>(s.d_offsets, s.Ks, s.K, s.chunk, accumulate_wave(),
                                                           s.d_counts, s.d_fat_list, s.d_total + 2, s.d_total);
        }
        G16_CUDA(scan(s.d_counts, s.d_seg_base, s.Ks, s.d_scan_tmp, s.d_total + 1, st));
    }
    return cudaSuccess;
}

// The pieces kernels keep two points per thread in shared memory: above 48 KB a
// block needs the opt-in limit (blocks of 2^8 threads).
static void reduce_attrs() {
    static const bool done = [] {
        const int g1 = 2 * (1 << MSM_REDUCE_LB_G1) * (int)XYZZ_G1_BYTES;
        const int g2 = 2 * (1 << MSM_REDUCE_LB_G2) * (int)XYZZ_G2_BYTES;
        cudaFuncSetAttribute(k_reduce_pieces<g16d::Fq, MSM_REDUCE_LB_G1>, cudaFuncAttributeMaxDynamicSharedMemorySize, g1);
        cudaFuncSetAttribute(k_reduce_pieces_multi<g16d::Fq, MSM_REDUCE_LB_G1>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, g1);
        cudaFuncSetAttribute(k_reduce_pieces<g16d::Fq2, MSM_REDUCE_LB_G2>, cudaFuncAttributeMaxDynamicSharedMemorySize, g2);
        cudaFuncSetAttribute(k_reduce_pieces_multi<g16d::Fq2, MSM_REDUCE_LB_G2>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, g2);
        return true;
    }();
    (void)done;
}

template <class F>
static cudaError_t accumulate(const MsmSort& s, MsmAccum& acc, const void* d_bases, uint32_t base_offset,
                              uint32_t n_bases, cudaStream_t st, size_t xyzz_bytes, const char* tag) {
    size_t max_entries = (s.n ? s.n : 1) * (size_t)s.W;
    size_t chunks = (max_entries + s.chunk - 1) / s.chunk;
    size_t max_partials = (size_t)s.Ks + chunks + 1;
    G16_CUDA(grow_bytes(st, acc.d_partials, acc.cap_partials, max_partials * xyzz_bytes, acc.fixed));
    const uint32_t Wr = s.shared ? 1u : (uint32_t)s.W;   // bucket sets to reduce
    constexpr bool G2 = !std::is_same<F, g16d::Fq>::value;
    constexpr int LB = G2 ? MSM_REDUCE_LB_G2 : MSM_REDUCE_LB_G1;   // pieces per reduction block: 2^LB
    reduce_attrs();
    const MsmReducePlan plan =
        msm_reduce_plan(Wr, s.B, G2, s.reduce_pieces ? s.reduce_pieces : msm_reduce_pieces(s.shared));
    acc.plan = plan;
    G16_CUDA(grow_bytes(st, acc.d_buckets, acc.cap_buckets, (size_t)s.K * xyzz_bytes, acc.fixed));
    if (!plan.direct)
        G16_CUDA(grow_bytes(st, acc.d_segments, acc.cap_segments, plan.block_points() * xyzz_bytes, acc.fixed));
    G16_CUDA(grow_bytes(st, acc.d_windows, acc.cap_windows, plan.result_points() * xyzz_bytes, acc.fixed));
    if (!acc.d_work) {
        if (acc.fixed) G16_CUDA(fixed_too_small(sizeof(unsigned long long), 0));
        G16_CUDA(g16::dev_realloc_async(&acc.d_work, sizeof(unsigned long long), st, false));
    }
    G16_CUDA(cudaMemsetAsync(acc.d_work, 0, sizeof(unsigned long long), st));
    uint4* partials = (uint4*)acc.d_partials;
    {
        TimedLaunch tl(tag, st);
        if (std::is_same<F, g16d::Fq>::value)
            k_accumulate_g1<<<blocks_for(chunks, ACC_BLOCK_G1), ACC_BLOCK_G1, 0, st>>>(
                s.d_entries, s.d_offsets, s.d_seg_base, s.Ks, s.d_total, s.d_total + 3, (const uint4*)d_bases,
                base_offset, n_bases, partials, acc.d_work);
        else
            k_accumulate_g2<<<blocks_for(chunks, ACC_BLOCK_G2), ACC_BLOCK_G2, 0, st>>>(
                s.d_entries, s.d_offsets, s.d_seg_base, s.Ks, s.d_total, s.d_total + 3, (const uint4*)d_bases,
                base_offset, n_bases, partials, acc.d_work);
    }
    G16_CUDA(cudaGetLastError());
    {
        TimedLaunch tl("msm_fat_merge", st);
        k_fat_merge_jobs<F><<<2 * device_sms(), 128, 128 * xyzz_bytes, st>>>(partials, s.d_offsets, s.d_seg_base,
                                                                          s.d_fat_list,
                                                                s.d_total + 2, s.d_total + 3);
    }
    {
        TimedLaunch tl("msm_fat_merge", st);
        k_fat_merge_final<F><<<device_sms(), 64, 64 * xyzz_bytes, st>>>(partials, s.d_offsets, s.d_seg_base,
                                                                        s.d_fat_list,
                                                               s.d_total + 2, s.d_total + 3);
    }
    G16_CUDA(cudaGetLastError());
    {
        TimedLaunch tl("msm_bucket_sums", st);
        k_bucket_sums<F><<<blocks_for(s.K, BUCKET_SUMS_BLOCK), BUCKET_SUMS_BLOCK, 0, st>>>(partials, s.d_offsets, s.d_seg_base, s.K, s.d_total + 3,
                                                                (uint4*)acc.d_buckets);
    }
    {
        TimedLaunch tl("msm_reduce", st);
        uint4* blocks = (uint4*)(plan.direct ? acc.d_windows : acc.d_segments);
        k_reduce_pieces<F, LB><<<dim3(plan.nb, Wr), 1u << LB, 2 * ((size_t)1 << LB) * xyzz_bytes, st>>>(
            (const uint4*)acc.d_buckets, s.B, plan.seg, blocks);
    }
    if (!plan.direct) {
        TimedLaunch tl("msm_reduce", st);
        const unsigned threads = plan.nb < 128 ? plan.nb : 128;
        k_reduce_sets<F, LB><<<dim3(LB + 1 + plan.hb, Wr), threads, threads * xyzz_bytes, st>>>(
            (const uint4*)acc.d_segments, plan.nb, (uint4*)acc.d_windows);
    }
    G16_CUDA(cudaGetLastError());
    return cudaSuccess;
}

cudaError_t msm_accumulate_g1(const MsmSort& s, MsmAccum& acc, const void* d_bases, uint32_t base_offset,
                              uint32_t n_bases, cudaStream_t st) {
    return accumulate<g16d::Fq>(s, acc, d_bases, base_offset, n_bases, st, XYZZ_G1_BYTES, "msm_accumulate_g1");
}

cudaError_t msm_accumulate_g2(const MsmSort& s, MsmAccum& acc, const void* d_bases, uint32_t base_offset,
                              uint32_t n_bases, cudaStream_t st) {
    return accumulate<g16d::Fq2>(s, acc, d_bases, base_offset, n_bases, st, XYZZ_G2_BYTES, "msm_accumulate_g2");
}

// ---- batched MSMs ----
void MsmSpace::release() {
    sort.release();
    acc.release();
    cudaFree(d_segdev);
    cudaFree(d_reduce);
    d_segdev = d_reduce = nullptr;
    cap_segdev = cap_reduce = 0;
}

void MsmSources::release() {
    cudaFree(d_desc);
    cudaFree(d_blk);
    cudaFree(d_std);
    d_desc = nullptr;
    d_blk = nullptr;
    d_std = nullptr;
    cap_desc = cap_blk = cap_std = 0;
}

// Upload a descriptor table into a device buffer that only grows (cap in bytes).
template <class T>
static cudaError_t upload_vec(void*& d, size_t& cap, const std::vector<T>& v, cudaStream_t st) {
    G16_CUDA(grow_bytes(st, d, cap, (v.empty() ? 1 : v.size()) * sizeof(T)));
    if (!v.empty()) G16_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return cudaSuccess;
}

cudaError_t msm_batch_setup(MsmSources& so, MsmSpace* const* spaces, int nspaces, cudaStream_t st) {
    // entries each space can receive: every live row of every target, once per window
    for (int i = 0; i < nspaces; i++) spaces[i]->max_entries = 0;
    for (auto& src : so.srcs) {
        if (src.c < 4 || src.c > 24 || src.ntargets < 0 || src.ntargets > MSM_MAX_TARGETS) {
            set_error("batched MSM source with window %d bits and %d targets", src.c, src.ntargets);
            return cudaErrorInvalidValue;
        }
        const uint32_t W = (uint32_t)msm_windows(src.c);
        for (int j = 0; j < src.ntargets; j++) {
            const MsmSourceTgt& t = src.t[j];
            if (t.space < 0 || t.space >= nspaces || t.seg < 0 || (size_t)t.seg >= spaces[t.space]->segs.size() ||
                spaces[t.space]->segs[t.seg].B != (1u << (src.c - 1)) || (uint64_t)t.rows * W >= 0x80000000ull) {
                set_error("batched MSM target does not match its segment");
                return cudaErrorInvalidValue;
            }
            spaces[t.space]->max_entries += (size_t)(t.d_rank ? t.rows : src.n) * W;
        }
    }
    for (int i = 0; i < nspaces; i++) {
        MsmSpace& sp = *spaces[i];
        const size_t pb = sp.g2 ? XYZZ_G2_BYTES : XYZZ_G1_BYTES;
        uint32_t piece_len = 0;
        if (const char* e = std::getenv("G16_BATCH_PIECE_LEN")) piece_len = (uint32_t)std::max(0, std::atoi(e));   // tuning knob: 1, 2, 4, ..., 32
        std::vector<uint32_t> seg_B;
        for (auto& g : sp.segs) seg_B.push_back(g.B);
        const MsmSpaceReduceLayout L = msm_space_reduce_layout(seg_B, sp.g2, sp.pieces_target, device_sms(), piece_len);
        std::vector<MsmSegDev> segdev;
        std::vector<MsmReduceDev> red;
        for (size_t j = 0; j < sp.segs.size(); j++) {
            MsmSpaceSeg& g = sp.segs[j];
            g.key_start = L.key_start[j];
            g.plan = L.plans[j];
            g.block_start = L.block_start[j];
            g.out_block = L.out_block[j];
            g.out_set = L.out_set[j];
            segdev.push_back({(const uint4*)g.table, g.key_start, g.n_bases});
            red.push_back({g.key_start, g.B, g.plan.seg, g.plan.nb, g.plan.hb, g.block_start, g.out_block, g.out_set});
        }
        sp.max_hb = L.max_hb;
        const uint64_t K = L.K, blocks = L.blocks, out_block = L.block_points, out_set = L.result_points;
        if (K >= 0x80000000ull || sp.max_entries >= 0x80000000ull) {
            set_error("batched MSM space of %llu buckets and %zu entries exceeds 32-bit indices",
                      (unsigned long long)K, sp.max_entries);
            return cudaErrorInvalidValue;
        }
        sp.K = (uint32_t)K;
        sp.blocks = (uint32_t)blocks;
        sp.result_points = (uint32_t)out_set;
        MsmSort& s = sp.sort;
        s.K = s.Ks = sp.K;
        s.B = 0;
        s.shared = true;
        s.chunk = 16;
        s.n = sp.max_entries;   // accumulate sizes its partials by entries, W = 1 below
        s.W = 1;
        const size_t kk = (size_t)sp.K + 1;
        if (kk > s.cap_k || !s.d_counts) {
            size_t cap = 0;
            G16_CUDA(grow(st, s.d_counts, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_offsets, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_cursor, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_seg_base, cap, kk));
            cap = 0;
            G16_CUDA(grow(st, s.d_fat_list, cap, kk));
            s.cap_k = cap;
        }
        G16_CUDA(grow(st, s.d_scan_tmp, s.cap_tmp, kk / 1024 + 2));
        G16_CUDA(grow(st, s.d_entries, s.cap_entries, sp.max_entries ? sp.max_entries : 1));
        if (!s.d_total) G16_CUDA(g16::dev_realloc_async(&s.d_total, 4 * sizeof(uint32_t), st, false));
        MsmAccum& a = sp.acc;
        const size_t chunks = (sp.max_entries + s.chunk - 1) / s.chunk;
        G16_CUDA(grow_bytes(st, a.d_partials, a.cap_partials, ((size_t)sp.K + chunks + 1) * pb));
        G16_CUDA(grow_bytes(st, a.d_buckets, a.cap_buckets, ((size_t)sp.K + 1) * pb));
        G16_CUDA(grow_bytes(st, a.d_segments, a.cap_segments, (out_block + 1) * pb));
        G16_CUDA(grow_bytes(st, a.d_windows, a.cap_windows, (out_set + 1) * pb));
        if (!a.d_work) G16_CUDA(g16::dev_realloc_async(&a.d_work, sizeof(unsigned long long), st, false));
        G16_CUDA(upload_vec(sp.d_segdev, sp.cap_segdev, segdev, st));
        G16_CUDA(upload_vec(sp.d_reduce, sp.cap_reduce, red, st));
    }
    // sources: one block of 256 scalars never straddles two sources
    std::vector<MsmSourceDev> desc;
    std::vector<uint32_t> blk;
    size_t std_elems = 0;
    for (auto& src : so.srcs) std_elems += src.n;
    G16_CUDA(grow_bytes(st, so.d_std, so.cap_std, (std_elems ? std_elems : 1) * 32));
    uint64_t blocks = 0, off = 0;
    for (auto& src : so.srcs) {
        MsmSourceDev d = {};
        d.scalars = (const uint4*)src.d_scalars;
        d.std_out = (uint4*)((uint8_t*)so.d_std + off * 32);
        d.n = src.n;
        d.c = (uint32_t)src.c;
        d.W = (uint32_t)msm_windows(src.c);
        d.ntargets = (uint32_t)src.ntargets;
        for (int j = 0; j < src.ntargets; j++) {
            MsmSpace& sp = *spaces[src.t[j].space];
            d.t[j] = {sp.sort.d_counts, sp.sort.d_cursor, sp.sort.d_entries, src.t[j].d_rank,
                      sp.segs[src.t[j].seg].key_start, src.t[j].d_rank ? src.t[j].rows : src.n};
        }
        desc.push_back(d);
        blk.push_back((uint32_t)blocks);
        blocks += (src.n + 255) / 256;
        off += src.n;
    }
    if (blocks >= 0x80000000ull) {
        set_error("batched MSM sources of %llu blocks", (unsigned long long)blocks);
        return cudaErrorInvalidValue;
    }
    so.total_blocks = (uint32_t)blocks;
    G16_CUDA(upload_vec(so.d_desc, so.cap_desc, desc, st));
    void* dblk = so.d_blk;
    G16_CUDA(upload_vec(dblk, so.cap_blk, blk, st));
    so.d_blk = (uint32_t*)dblk;
    G16_CUDA(cudaStreamSynchronize(st));
    return cudaSuccess;
}

cudaError_t msm_batch_sort(MsmSources& so, MsmSpace* const* spaces, int nspaces, cudaStream_t st) {
    for (int i = 0; i < nspaces; i++) {
        MsmSort& s = spaces[i]->sort;
        G16_CUDA(cudaMemsetAsync(s.d_counts, 0, ((size_t)s.K + 1) * sizeof(uint32_t), st));
        G16_CUDA(cudaMemsetAsync(s.d_total, 0, 4 * sizeof(uint32_t), st));
    }
    const uint32_t nsrc = (uint32_t)so.srcs.size();
    if (so.total_blocks) {
        TimedLaunch tl("msm_digits", st);
        k_digits_multi<<<so.total_blocks, 256, 0, st>>>((const MsmSourceDev*)so.d_desc, so.d_blk, nsrc);
    }
    G16_CUDA(cudaGetLastError());
    for (int i = 0; i < nspaces; i++) {
        MsmSort& s = spaces[i]->sort;
        G16_CUDA(scan(s.d_counts, s.d_offsets, s.K, s.d_scan_tmp, s.d_total, st));
        TimedLaunch tl("msm_copy", st);
        k_copy_u32<<<blocks_for(s.K ? s.K : 1, 256), 256, 0, st>>>(s.d_cursor, s.d_offsets, s.K);
    }
    if (so.total_blocks) {
        TimedLaunch tl("msm_scatter", st);
        k_scatter_multi<<<so.total_blocks, 256, 0, st>>>((const MsmSourceDev*)so.d_desc, so.d_blk, nsrc);
    }
    G16_CUDA(cudaGetLastError());
    for (int i = 0; i < nspaces; i++) {
        MsmSort& s = spaces[i]->sort;
        {
            TimedLaunch tl("msm_nseg", st);
            k_nseg<<<blocks_for(s.K ? s.K : 1, 256), 256, 0, st>>>(s.d_offsets, s.K, s.K, s.chunk, accumulate_wave(),
                                                                   s.d_counts, s.d_fat_list, s.d_total + 2,
                                                                   s.d_total);
        }
        G16_CUDA(scan(s.d_counts, s.d_seg_base, s.K, s.d_scan_tmp, s.d_total + 1, st));
    }
    return cudaSuccess;
}

template <class F, int LB>
static cudaError_t space_accumulate(MsmSpace& sp, cudaStream_t st, size_t xyzz_bytes, const char* tag) {
    MsmSort& s = sp.sort;
    MsmAccum& a = sp.acc;
    const size_t chunks = (sp.max_entries + s.chunk - 1) / s.chunk;
    G16_CUDA(cudaMemsetAsync(a.d_work, 0, sizeof(unsigned long long), st));
    uint4* partials = (uint4*)a.d_partials;
    const uint32_t nsegs = (uint32_t)sp.segs.size();
    // the blocks' output was laid out from the plans: they must use this LB
    for (const auto& g : sp.segs)
        if (g.plan.lb != (uint32_t)LB) {
            set_error("batched MSM reduction planned with 2^%u pieces per block, launched with 2^%d", g.plan.lb, LB);
            return cudaErrorInvalidValue;
        }
    if (chunks) {
        TimedLaunch tl(tag, st);
        if (std::is_same<F, g16d::Fq>::value)
            k_accumulate_multi_g1<<<blocks_for(chunks, ACC_BLOCK_G1), ACC_BLOCK_G1, 0, st>>>(
                s.d_entries, s.d_offsets, s.d_seg_base, s.K, s.d_total, s.d_total + 3, (const MsmSegDev*)sp.d_segdev,
                nsegs, partials, a.d_work);
        else
            k_accumulate_multi_g2<<<blocks_for(chunks, ACC_BLOCK_G2), ACC_BLOCK_G2, 0, st>>>(
                s.d_entries, s.d_offsets, s.d_seg_base, s.K, s.d_total, s.d_total + 3, (const MsmSegDev*)sp.d_segdev,
                nsegs, partials, a.d_work);
    }
    G16_CUDA(cudaGetLastError());
    const uint32_t sms = device_sms();
    {
        TimedLaunch tl("msm_fat_merge", st);
        k_fat_merge_jobs<F><<<2 * sms, 128, 128 * xyzz_bytes, st>>>(partials, s.d_offsets, s.d_seg_base, s.d_fat_list,
                                                                    s.d_total + 2, s.d_total + 3);
    }
    {
        TimedLaunch tl("msm_fat_merge", st);
        k_fat_merge_final<F><<<sms, 64, 64 * xyzz_bytes, st>>>(partials, s.d_offsets, s.d_seg_base, s.d_fat_list,
                                                              s.d_total + 2, s.d_total + 3);
    }
    G16_CUDA(cudaGetLastError());
    if (s.K) {
        TimedLaunch tl("msm_bucket_sums", st);
        k_bucket_sums<F><<<blocks_for(s.K, BUCKET_SUMS_BLOCK), BUCKET_SUMS_BLOCK, 0, st>>>(partials, s.d_offsets, s.d_seg_base, s.K, s.d_total + 3,
                                                                (uint4*)a.d_buckets);
    }
    if (sp.blocks) {
        TimedLaunch tl("msm_reduce", st);
        k_reduce_pieces_multi<F, LB><<<sp.blocks, 1u << LB, 2 * ((size_t)1 << LB) * xyzz_bytes, st>>>(
            (const uint4*)a.d_buckets, (const MsmReduceDev*)sp.d_reduce, nsegs, (uint4*)a.d_segments);
    }
    if (nsegs) {
        TimedLaunch tl("msm_reduce_sets", st);
        k_reduce_sets_multi<F, LB><<<dim3(LB + 1 + sp.max_hb, nsegs), 128, 128 * xyzz_bytes, st>>>(
            (const uint4*)a.d_segments, (const MsmReduceDev*)sp.d_reduce, (uint4*)a.d_windows);
    }
    G16_CUDA(cudaGetLastError());
    return cudaSuccess;
}

cudaError_t msm_space_accumulate(MsmSpace& sp, cudaStream_t st) {
    reduce_attrs();
    if (sp.g2) return space_accumulate<g16d::Fq2, MSM_REDUCE_LB_G2>(sp, st, XYZZ_G2_BYTES, "msm_accumulate_g2");
    return space_accumulate<g16d::Fq, MSM_REDUCE_LB_G1>(sp, st, XYZZ_G1_BYTES, "msm_accumulate_g1");
}

// ---- host: window sums -> Horner ----
static Fq fq_at(const uint8_t* p) {
    uint64_t v[4];
    std::memcpy(v, p, 32);
    return Fq::raw(v);
}

template <class F>
static F read_coord(const uint8_t* p);
template <>
Fq read_coord<Fq>(const uint8_t* p) { return fq_at(p); }
template <>
Fq2 read_coord<Fq2>(const uint8_t* p) { return {fq_at(p), fq_at(p + 32)}; }

// XYZZ (x = X / ZZ, y = Y / ZZZ) -> Jacobian (x = X' / Z^2, y = Y' / Z^3)
// without an inversion: Z = ZZ ZZZ, X' = X ZZ ZZZ^2, Y' = Y ZZ^3 ZZZ^2.
template <class F>
static Jac<F> xyzz_to_jac(const uint8_t* p) {
    const size_t cs = sizeof(F) == sizeof(Fq) ? 32 : 64;   // coordinate bytes
    F X = read_coord<F>(p), Y = read_coord<F>(p + cs), zz = read_coord<F>(p + 2 * cs), zzz = read_coord<F>(p + 3 * cs);
    if (zz.is_zero()) return Jac<F>::identity();
    F zzz2 = zzz.sqr();
    Jac<F> r;
    r.z = zz * zzz;
    r.x = X * zz * zzz2;
    r.y = Y * zz.sqr() * zz * zzz2;
    return r;
}

// One set's sum_b (b + 1) S_b from the reduction's points (msm_reduce_plan).
template <class F>
static Jac<F> set_sum(const uint8_t* p, const MsmReducePlan& pl) {
    const size_t pb = 4 * (sizeof(F) == sizeof(Fq) ? 32 : 64);
    auto at = [&](size_t i) { return xyzz_to_jac<F>(p + i * pb); };
    Jac<F> T = Jac<F>::identity();
    std::vector<Jac<F>> G(pl.lb, Jac<F>::identity()), Gb(pl.hb, Jac<F>::identity());
    if (pl.direct) {
        for (uint32_t j = 0; j < pl.nb; j++) {
            const size_t o = (size_t)j * pl.block_terms();
            T = T + at(o);
            for (uint32_t i = 0; i < pl.lb; i++) G[i] = G[i] + at(o + 1 + i);
            if (pl.hb) {
                Jac<F> R = at(o + pl.lb + 1);
                for (uint32_t i = 0; i < pl.hb; i++)
                    if ((j >> i) & 1u) Gb[i] = Gb[i] + R;
            }
        }
    } else {
        T = at(0);
        for (uint32_t i = 0; i < pl.lb; i++) G[i] = at(1 + i);
        for (uint32_t i = 0; i < pl.hb; i++) Gb[i] = at(pl.lb + 1 + i);
    }
    Jac<F> acc = Jac<F>::identity();
    for (int i = (int)pl.hb - 1; i >= 0; i--) acc = acc.dbl() + Gb[i];
    for (int j = (int)pl.lb - 1; j >= 0; j--) acc = acc.dbl() + G[j];
    for (uint32_t s = pl.seg; s > 1; s >>= 1) acc = acc.dbl();
    return acc + T;
}

template <class F>
static Jac<F> combine(const uint8_t* result, const MsmReducePlan& pl, int c) {
    const size_t set_bytes = (size_t)pl.set_terms() * 4 * (sizeof(F) == sizeof(Fq) ? 32 : 64);
    const int W = (int)pl.sets;
    if (W == 0) return Jac<F>::identity();
    Jac<F> acc = set_sum<F>(result + (size_t)(W - 1) * set_bytes, pl);
    for (int i = W - 2; i >= 0; i--) {
        for (int j = 0; j < c; j++) acc = acc.dbl();
        acc = acc + set_sum<F>(result + (size_t)i * set_bytes, pl);
    }
    return acc;
}

G1J msm_combine_g1(const uint8_t* result_xyzz, const MsmReducePlan& plan, int c) {
    return combine<Fq>(result_xyzz, plan, c);
}
G2J msm_combine_g2(const uint8_t* result_xyzz, const MsmReducePlan& plan, int c) {
    return combine<Fq2>(result_xyzz, plan, c);
}

}  // namespace g16

namespace g16 {

G1J msm_space_combine_g1(const uint8_t* results, const MsmSpace& sp, size_t s) {
    const MsmSpaceSeg& g = sp.segs[s];
    return msm_combine_g1(results + (size_t)g.out_set * XYZZ_G1_BYTES, g.plan, 1);
}

G2J msm_space_combine_g2(const uint8_t* results, const MsmSpace& sp, size_t s) {
    const MsmSpaceSeg& g = sp.segs[s];
    return msm_combine_g2(results + (size_t)g.out_set * XYZZ_G2_BYTES, g.plan, 1);
}

}  // namespace g16
