// Radix-2 Fr NTT kernels (see ntt.cuh).
#include "common.cuh"
#include "field.cuh"
#include "host_bn254.hpp"
#include "ntt.cuh"
#include <vector>

namespace g16d {

struct Vec3 {
    uint4* p[3];
};

__device__ __forceinline__ Fr ld_s(const uint4* sm, uint32_t e) {
    uint4 a = sm[2 * e], b = sm[2 * e + 1];
    Fr r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}
__device__ __forceinline__ void st_s(uint4* sm, uint32_t e, const Fr& x) {
    sm[2 * e] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    sm[2 * e + 1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}
__device__ __forceinline__ Fr ld_g(const uint4* g, size_t i) {
    uint4 a = __ldg(g + 2 * i), b = __ldg(g + 2 * i + 1);
    Fr r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}
__device__ __forceinline__ Fr ld_rw(const uint4* g, size_t i) {
    uint4 a = g[2 * i], b = g[2 * i + 1];
    Fr r;
    r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w;
    r.v[4] = b.x; r.v[5] = b.y; r.v[6] = b.z; r.v[7] = b.w;
    return r;
}
__device__ __forceinline__ void st_g(uint4* g, size_t i, const Fr& x) {
    g[2 * i] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    g[2 * i + 1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
}

// The butterflies, the coset multiply and the join use mul, the CIOS product
// on 32x32->64-bit multiply-adds (field.cuh), which measured faster than the
// PTX carry-chain form mul_cc; the table builders below keep mul_cc, so both
// forms stay under the parity tests.

// One radix-2 stage on a shared-memory tile.  The tile holds elements
// i = hi*2^(s_lo+k) + mid*2^s_lo + (lo0 + l) at smem slot mid*L + l; stage
// s = s_lo + j pairs mid values differing in bit j.  The butterfly's
// position inside its 2^(s+1) block is (mid mod 2^j)*2^s_lo + lo0 + l and
// its twiddle omega_{2^(s+1)}^pos = tw[pos << (log_n - s - 1)].
template <bool DIF>
__device__ __forceinline__ void run_stage(uint4* sm, uint32_t j, uint32_t s_lo, uint32_t log_L, uint32_t lo0,
                                          uint32_t log_n, uint32_t half_tile, const uint4* __restrict__ tw) {
    const uint32_t L = 1u << log_L;
    const uint32_t s = s_lo + j;
    const uint32_t jmask = (1u << j) - 1u;
    for (uint32_t q = threadIdx.x; q < half_tile; q += blockDim.x) {
        uint32_t l = q & (L - 1u);
        uint32_t mq = q >> log_L;
        uint32_t mid_a = ((mq >> j) << (j + 1)) | (mq & jmask);
        uint32_t ea = (mid_a << log_L) | l;
        uint32_t eb = ea + (1u << (j + log_L));
        uint32_t pos = ((mid_a & jmask) << s_lo) | (lo0 + l);
        Fr a = ld_s(sm, ea), b = ld_s(sm, eb);
        if (DIF) {
            Fr d = sub(a, b);
            a = add(a, b);
            b = pos ? mul(d, ld_g(tw, (size_t)pos << (log_n - s - 1))) : d;
        } else {
            Fr t = pos ? mul(b, ld_g(tw, (size_t)pos << (log_n - s - 1))) : b;
            b = sub(a, t);
            a = add(a, t);
        }
        st_s(sm, ea, a);
        st_s(sm, eb, b);
    }
}

// Stages [s_lo, s_lo + k) of 2^log_n, one tile of (2^k)*L elements per block
// (block bx of the pass).  Optional epilogues: multiply by *scale, or write
// h = join_a * join_b - x to join_out instead of storing x.
template <bool DIF>
__device__ __forceinline__ void ntt_pass_tile(uint4* sm, uint4* data, uint32_t bx, uint32_t log_n, uint32_t s_lo,
                                              uint32_t k, uint32_t log_L, const uint4* __restrict__ tw,
                                              const uint4* __restrict__ scale, const uint4* __restrict__ join_a,
                                              const uint4* __restrict__ join_b, uint4* __restrict__ join_out) {
    const uint32_t L = 1u << log_L;
    const uint32_t tile = (1u << k) << log_L;
    const uint32_t bph = s_lo - log_L;
    const size_t hi = bx >> bph;
    const uint32_t lo0 = (bx & ((1u << bph) - 1u)) << log_L;
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        uint32_t mid = e >> log_L, l = e & (L - 1u);
        size_t gi = (hi << (s_lo + k)) | ((size_t)mid << s_lo) | (lo0 + l);
        sm[2 * e] = data[2 * gi];
        sm[2 * e + 1] = data[2 * gi + 1];
    }
    __syncthreads();
    for (uint32_t jj = 0; jj < k; jj++) {
        uint32_t j = DIF ? k - 1 - jj : jj;
        run_stage<DIF>(sm, j, s_lo, log_L, lo0, log_n, tile / 2, tw);
        __syncthreads();
    }
    Fr sc;
    if (scale) sc = ld_g(scale, 0);
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        uint32_t mid = e >> log_L, l = e & (L - 1u);
        size_t gi = (hi << (s_lo + k)) | ((size_t)mid << s_lo) | (lo0 + l);
        Fr x = ld_s(sm, e);
        if (scale) x = mul(x, sc);
        if (join_out) {
            Fr h = sub(mul(ld_rw(join_a, gi), ld_rw(join_b, gi)), x);
            st_g(join_out, gi, h);
        } else {
            st_g(data, gi, x);
        }
    }
}

// blockIdx.y selects the vector
template <bool DIF>
__global__ void __launch_bounds__(256) k_ntt_pass(Vec3 vecs, uint32_t log_n, uint32_t s_lo, uint32_t k,
                                                  uint32_t log_L, const uint4* __restrict__ tw,
                                                  const uint4* __restrict__ scale, const uint4* __restrict__ join_a,
                                                  const uint4* __restrict__ join_b, uint4* __restrict__ join_out) {
    extern __shared__ uint4 sm[];
    ntt_pass_tile<DIF>(sm, vecs.p[blockIdx.y], blockIdx.x, log_n, s_lo, k, log_L, tw, scale, join_a, join_b,
                       join_out);
}

// The fused middle of iNTT -> coset -> NTT: DIF stages [0, k) with inverse
// twiddles, a[p] *= coset[p], DIT stages [0, k) with forward twiddles, on
// contiguous tiles of 2^k.  Optional h = join_a * join_b - x epilogue for a
// transform that has no outer passes.
__device__ __forceinline__ void ntt_mid_tile(uint4* sm, uint4* data, uint32_t bx, uint32_t log_n, uint32_t k,
                                             const uint4* __restrict__ tw, const uint4* __restrict__ tw_inv,
                                             const uint4* __restrict__ coset, const uint4* __restrict__ join_a,
                                             const uint4* __restrict__ join_b, uint4* __restrict__ join_out) {
    const uint32_t tile = 1u << k;
    const size_t base = (size_t)bx << k;
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        sm[2 * e] = data[2 * (base + e)];
        sm[2 * e + 1] = data[2 * (base + e) + 1];
    }
    __syncthreads();
    for (int j = (int)k - 1; j >= 0; j--) {
        run_stage<true>(sm, (uint32_t)j, 0, 0, 0, log_n, tile / 2, tw_inv);
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) st_s(sm, e, mul(ld_s(sm, e), ld_g(coset, base + e)));
    __syncthreads();
    for (uint32_t j = 0; j < k; j++) {
        run_stage<false>(sm, j, 0, 0, 0, log_n, tile / 2, tw);
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        Fr x = ld_s(sm, e);
        if (join_out) {
            st_g(join_out, base + e, sub(mul(ld_rw(join_a, base + e), ld_rw(join_b, base + e)), x));
        } else {
            st_g(data, base + e, x);
        }
    }
}

// DIF stages [0, k) with inverse twiddles on contiguous tiles of 2^k, then
// each position p multiplied by table[p] and stored: the last step of an
// inverse transform to bit-reversed order with a per-position scale (gnark's
// H coefficients: table = shift^-bitrev(p) / n).
__global__ void __launch_bounds__(256) k_ntt_dif_scale(uint4* data, uint32_t log_n, uint32_t k,
                                                       const uint4* __restrict__ tw_inv,
                                                       const uint4* __restrict__ table) {
    extern __shared__ uint4 sm[];
    const uint32_t tile = 1u << k;
    const size_t base = (size_t)blockIdx.x << k;
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) {
        sm[2 * e] = data[2 * (base + e)];
        sm[2 * e + 1] = data[2 * (base + e) + 1];
    }
    __syncthreads();
    for (int j = (int)k - 1; j >= 0; j--) {
        run_stage<true>(sm, (uint32_t)j, 0, 0, 0, log_n, tile / 2, tw_inv);
        __syncthreads();
    }
    for (uint32_t e = threadIdx.x; e < tile; e += blockDim.x) st_g(data, base + e, mul(ld_s(sm, e), ld_g(table, base + e)));
}

__global__ void __launch_bounds__(256) k_ntt_mid(Vec3 vecs, uint32_t log_n, uint32_t k, const uint4* __restrict__ tw,
                                                 const uint4* __restrict__ tw_inv, const uint4* __restrict__ coset,
                                                 const uint4* __restrict__ join_a, const uint4* __restrict__ join_b,
                                                 uint4* __restrict__ join_out) {
    extern __shared__ uint4 sm[];
    ntt_mid_tile(sm, vecs.p[blockIdx.y], blockIdx.x, log_n, k, tw, tw_inv, coset, join_a, join_b, join_out);
}

// ---- many transforms per launch (batched proving) ----
// A job is one vector's pass (or fused middle) of one transform; the blocks
// of a launch are the jobs' tiles back to back, block_start being a job's
// first block.
struct NttJob {
    uint4* data;
    const uint4* tw;        // pass: the pass's twiddles; middle: forward twiddles
    const uint4* tw_inv;    // middle: inverse twiddles
    const uint4* coset;     // middle: shift^bitrev(p) / n
    const uint4* join_a;    // join epilogue h = a * b - x, or null
    const uint4* join_b;
    uint4* join_out;
    uint32_t log_n, s_lo, k, log_L, block_start, pad;
};

__device__ __forceinline__ uint32_t job_of(const NttJob* __restrict__ jobs, uint32_t njobs, uint32_t b) {
    uint32_t lo = 0, hi = njobs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].block_start <= b) lo = mid; else hi = mid;
    }
    return lo;
}

template <bool DIF>
__global__ void __launch_bounds__(256) k_ntt_pass_multi(const NttJob* __restrict__ jobs, uint32_t njobs) {
    extern __shared__ uint4 sm[];
    const NttJob& j = jobs[job_of(jobs, njobs, blockIdx.x)];
    ntt_pass_tile<DIF>(sm, j.data, blockIdx.x - j.block_start, j.log_n, j.s_lo, j.k, j.log_L, j.tw, nullptr, j.join_a,
                       j.join_b, j.join_out);
}

__global__ void __launch_bounds__(256) k_ntt_mid_multi(const NttJob* __restrict__ jobs, uint32_t njobs) {
    extern __shared__ uint4 sm[];
    const NttJob& j = jobs[job_of(jobs, njobs, blockIdx.x)];
    ntt_mid_tile(sm, j.data, blockIdx.x - j.block_start, j.log_n, j.k, j.tw, j.tw_inv, j.coset, j.join_a, j.join_b,
                 j.join_out);
}

__device__ __forceinline__ Fr fr_pow_u64(Fr b, uint64_t e) {
    Fr acc = Fr::one();
    while (e) {
        if (e & 1) acc = mul_cc(acc, b);
        b = mul_cc(b, b);
        e >>= 1;
    }
    return acc;
}

// out[i or bitrev(i)] = scale * base^i for i < count, 16 per thread
__global__ void k_powers(uint4* out, Fr base, Fr scale, uint64_t count, uint32_t bitrev_log) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t i0 = t * 16;
    if (i0 >= count) return;
    Fr p = mul_cc(scale, fr_pow_u64(base, i0));
    for (uint64_t i = i0; i < i0 + 16 && i < count; i++) {
        size_t dst = bitrev_log ? (size_t)(__brevll(i) >> (64 - bitrev_log)) : (size_t)i;
        st_g(out, dst, p);
        p = mul_cc(p, base);
    }
}

// a[i] *= shift^i, 16 per thread
__global__ void k_distribute(uint4* a, Fr shift, uint64_t n) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t i0 = t * 16;
    if (i0 >= n) return;
    Fr p = fr_pow_u64(shift, i0);
    for (uint64_t i = i0; i < i0 + 16 && i < n; i++) {
        st_g(a, i, mul_cc(ld_rw(a, i), p));
        p = mul_cc(p, shift);
    }
}

__global__ void k_bitrev(uint4* a, uint32_t log_n, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t j = __brevll(i) >> (64 - log_n);
    if (j > i) {
        Fr x = ld_rw(a, i), y = ld_rw(a, j);
        st_g(a, i, y);
        st_g(a, j, x);
    }
}

__global__ void k_join(const uint4* a, const uint4* b, const uint4* c, uint4* h, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    st_g(h, i, sub(mul_cc(ld_rw(a, i), ld_rw(b, i)), ld_rw(c, i)));
}

}  // namespace g16d

namespace g16 {

using namespace g16d;

void NttTables::release() {
    cudaFree(d_tw);
    cudaFree(d_tw_inv);
    cudaFree(d_coset);
    cudaFree(d_coset_inv);
    d_tw = d_tw_inv = d_coset = d_coset_inv = nullptr;
    log_n = -1;
}

static g16d::Fr to_dev(const g16::Fr& x) {
    g16d::Fr r;
    std::memcpy(r.v, x.x.v, 32);
    return r;
}

cudaError_t ntt_tables(NttTables& t, int log_n, cudaStream_t st) {
    if (t.log_n == log_n) return cudaSuccess;
    if (log_n < 1 || log_n > 27) {
        set_error("NTT size 2^%d outside [2^1, 2^27]", log_n);
        return cudaErrorInvalidValue;
    }
    host_init();
    t.release();
    size_t n = (size_t)1 << log_n;
    G16_CUDA(g16::dev_malloc(&t.d_tw, (n / 2) * 32));
    G16_CUDA(g16::dev_malloc(&t.d_tw_inv, (n / 2) * 32));
    G16_CUDA(g16::dev_malloc(&t.d_coset, n * 32 + 32));   // + one slot holding 1/n for the scale epilogue
    g16::Fr w = domain_root(log_n), wi = w.inv();
    g16::Fr ninv = g16::Fr::from_u64(n).inv();
    g16::Fr shift = domain_root(log_n + 1);
    std::memcpy(t.n_inv, ninv.x.v, 32);
    std::memcpy(t.shift, shift.x.v, 32);
    g16d::Fr d_one;
    std::memcpy(d_one.v, g16::Fr::one().x.v, 32);
    {
        TimedLaunch tl("ntt_tables", st);
        k_powers<<<blocks_for((n / 2 + 15) / 16, 128), 128, 0, st>>>((uint4*)t.d_tw, to_dev(w), d_one, n / 2, 0);
    }
    {
        TimedLaunch tl("ntt_tables", st);
        k_powers<<<blocks_for((n / 2 + 15) / 16, 128), 128, 0, st>>>((uint4*)t.d_tw_inv, to_dev(wi), d_one, n / 2,
                                                                      0);
    }
    {
        TimedLaunch tl("ntt_tables", st);
        k_powers<<<blocks_for((n + 15) / 16, 128), 128, 0, st>>>((uint4*)t.d_coset, to_dev(shift), to_dev(ninv), n,
                                                                  (uint32_t)log_n);
    }
    G16_CUDA(cudaMemcpyAsync((uint8_t*)t.d_coset + n * 32, ninv.x.v, 32, cudaMemcpyHostToDevice, st));
    G16_CUDA(cudaGetLastError());
    G16_CUDA(cudaStreamSynchronize(st));
    t.log_n = log_n;
    return cudaSuccess;
}

using Pass = NttPass;
static uint32_t inner_k(const NttTiling& tl, uint32_t log_n) { return ntt_inner_k(tl, log_n); }
static std::vector<Pass> outer_passes(const NttTiling& tl, uint32_t log_n, uint32_t k0) {
    return ntt_outer_passes(tl, log_n, k0);
}

static bool attrs_done = false;
static void set_attrs() {
    if (attrs_done) return;
    size_t smem = ((size_t)1 << NTT_MAX_TILE_LOG) * 32;
    cudaFuncSetAttribute(k_ntt_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_ntt_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_ntt_mid, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_ntt_pass_multi<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_ntt_pass_multi<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_ntt_mid_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_ntt_dif_scale, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attrs_done = true;
}

static cudaError_t launch_pass(bool dif, Vec3 v, int nv, uint32_t log_n, const Pass& p, const void* tw,
                               const void* scale, const void* ja, const void* jb, void* jo, cudaStream_t st) {
    uint32_t tile = (1u << p.k) << p.log_L;
    size_t n = (size_t)1 << log_n;
    dim3 grid((unsigned)(n / tile), nv);
    unsigned threads = tile / 2 < 256 ? tile / 2 : 256;
    size_t smem = (size_t)tile * 32;
    const char* name = dif ? "ntt_pass_dif" : "ntt_pass_dit";
    // work: one Fr product per butterfly, plus the scale / join epilogue;
    // bytes: each vector read and written once, the join also reads A and B
    timer().add_units(name, (double)nv * (double)(n / 2) * p.k + (scale ? (double)nv * n : 0.0) + (jo ? (double)n : 0.0));
    timer().add_bytes(name, 64.0 * nv * n + (jo ? 64.0 * n : 0.0));
    TimedLaunch tl(name, st);
    if (dif)
        k_ntt_pass<true><<<grid, threads, smem, st>>>(v, log_n, p.s_lo, p.k, p.log_L, (const uint4*)tw,
                                                       (const uint4*)scale, (const uint4*)ja, (const uint4*)jb,
                                                       (uint4*)jo);
    else
        k_ntt_pass<false><<<grid, threads, smem, st>>>(v, log_n, p.s_lo, p.k, p.log_L, (const uint4*)tw,
                                                        (const uint4*)scale, (const uint4*)ja, (const uint4*)jb,
                                                        (uint4*)jo);
    return cudaGetLastError();
}

static cudaError_t launch_mid(Vec3 v, int nv, const NttTables& t, const void* ja, const void* jb, void* jo,
                              cudaStream_t st) {
    uint32_t log_n = (uint32_t)t.log_n;
    uint32_t k0 = inner_k(t.tiling, log_n);
    uint32_t tile = 1u << k0;
    size_t n = (size_t)1 << log_n;
    dim3 grid((unsigned)(n / tile), nv);
    unsigned threads = tile / 2 < 256 ? tile / 2 : 256;
    timer().add_units("ntt_mid_fused", (double)nv * ((double)n * k0 + n) + (jo ? (double)n : 0.0));
    timer().add_bytes("ntt_mid_fused", 64.0 * nv * n + (jo ? 64.0 * n : 0.0));
    TimedLaunch tl("ntt_mid_fused", st);
    k_ntt_mid<<<grid, threads, (size_t)tile * 32, st>>>(v, log_n, k0, (const uint4*)t.d_tw, (const uint4*)t.d_tw_inv,
                                                         (const uint4*)t.d_coset, (const uint4*)ja, (const uint4*)jb,
                                                         (uint4*)jo);
    return cudaGetLastError();
}

cudaError_t ntt_h_pipeline(const NttTables& t, void* a, void* b, void* c, void* h, cudaStream_t st) {
    set_attrs();
    uint32_t log_n = (uint32_t)t.log_n;
    uint32_t k0 = inner_k(t.tiling, log_n);
    auto outer = outer_passes(t.tiling, log_n, k0);
    Vec3 abc = {{(uint4*)a, (uint4*)b, (uint4*)c}};
    // inverse, DIF, top stages first
    for (size_t i = outer.size(); i-- > 0;)
        G16_CUDA(launch_pass(true, abc, 3, log_n, outer[i], t.d_tw_inv, nullptr, nullptr, nullptr, nullptr, st));
    if (outer.empty()) {
        G16_CUDA(launch_mid(abc, 2, t, nullptr, nullptr, nullptr, st));
        Vec3 cc = {{(uint4*)c, nullptr, nullptr}};
        return launch_mid(cc, 1, t, a, b, h, st);
    }
    G16_CUDA(launch_mid(abc, 3, t, nullptr, nullptr, nullptr, st));
    for (size_t i = 0; i + 1 < outer.size(); i++)
        G16_CUDA(launch_pass(false, abc, 3, log_n, outer[i], t.d_tw, nullptr, nullptr, nullptr, nullptr, st));
    G16_CUDA(launch_pass(false, abc, 2, log_n, outer.back(), t.d_tw, nullptr, nullptr, nullptr, nullptr, st));
    Vec3 cc = {{(uint4*)c, nullptr, nullptr}};
    return launch_pass(false, cc, 1, log_n, outer.back(), t.d_tw, nullptr, a, b, h, st);
}

cudaError_t ntt_intt_coset_ntt(const NttTables& t, void* a, cudaStream_t st) {
    set_attrs();
    uint32_t log_n = (uint32_t)t.log_n;
    uint32_t k0 = inner_k(t.tiling, log_n);
    auto outer = outer_passes(t.tiling, log_n, k0);
    Vec3 v = {{(uint4*)a, nullptr, nullptr}};
    for (size_t i = outer.size(); i-- > 0;)
        G16_CUDA(launch_pass(true, v, 1, log_n, outer[i], t.d_tw_inv, nullptr, nullptr, nullptr, nullptr, st));
    G16_CUDA(launch_mid(v, 1, t, nullptr, nullptr, nullptr, st));
    for (auto& p : outer)
        G16_CUDA(launch_pass(false, v, 1, log_n, p, t.d_tw, nullptr, nullptr, nullptr, nullptr, st));
    return cudaSuccess;
}

static cudaError_t dit_natural(const NttTables& t, void* a, const void* tw, const void* scale, cudaStream_t st) {
    set_attrs();
    uint32_t log_n = (uint32_t)t.log_n;
    size_t n = (size_t)1 << log_n;
    {
        TimedLaunch tl("ntt_bitrev", st);
        k_bitrev<<<blocks_for(n, 256), 256, 0, st>>>((uint4*)a, log_n, n);
    }
    G16_CUDA(cudaGetLastError());
    uint32_t k0 = inner_k(t.tiling, log_n);
    auto outer = outer_passes(t.tiling, log_n, k0);
    Vec3 v = {{(uint4*)a, nullptr, nullptr}};
    Pass inner = {0, k0, 0};
    G16_CUDA(launch_pass(false, v, 1, log_n, inner, tw, outer.empty() ? scale : nullptr, nullptr, nullptr, nullptr,
                         st));
    for (size_t i = 0; i < outer.size(); i++)
        G16_CUDA(launch_pass(false, v, 1, log_n, outer[i], tw, i + 1 == outer.size() ? scale : nullptr, nullptr,
                             nullptr, nullptr, st));
    return cudaSuccess;
}

cudaError_t ntt_gnark_table(NttTables& t, cudaStream_t st) {
    if (t.d_coset_inv) return cudaSuccess;
    if (t.log_n < 1) {
        set_error("gnark table before the domain tables");
        return cudaErrorInvalidValue;
    }
    const size_t n = (size_t)1 << t.log_n;
    G16_CUDA(g16::dev_malloc(&t.d_coset_inv, n * 32));
    const g16::Fr shift_inv = g16::Fr::raw(t.shift).inv(), ninv = g16::Fr::raw(t.n_inv);
    {
        TimedLaunch tl("ntt_tables", st);
        k_powers<<<blocks_for((n + 15) / 16, 128), 128, 0, st>>>((uint4*)t.d_coset_inv, to_dev(shift_inv), to_dev(ninv),
                                                                  n, (uint32_t)t.log_n);
    }
    G16_CUDA(cudaGetLastError());
    return cudaStreamSynchronize(st);
}

cudaError_t ntt_to_gnark_coefficients(const NttTables& t, void* h, cudaStream_t st) {
    if (!t.d_coset_inv) {
        set_error("gnark coefficients without the inverse coset table");
        return cudaErrorInvalidValue;
    }
    set_attrs();
    const uint32_t log_n = (uint32_t)t.log_n;
    const uint32_t k0 = inner_k(t.tiling, log_n);
    auto outer = outer_passes(t.tiling, log_n, k0);
    Vec3 v = {{(uint4*)h, nullptr, nullptr}};
    for (size_t i = outer.size(); i-- > 0;)   // inverse, DIF, top stages first
        G16_CUDA(launch_pass(true, v, 1, log_n, outer[i], t.d_tw_inv, nullptr, nullptr, nullptr, nullptr, st));
    const uint32_t tile = 1u << k0;
    const size_t n = (size_t)1 << log_n;
    const unsigned threads = tile / 2 < 256 ? tile / 2 : 256;
    timer().add_units("ntt_pass_dif", (double)(n / 2) * k0 + (double)n);
    timer().add_bytes("ntt_pass_dif", 64.0 * n);
    TimedLaunch tl("ntt_pass_dif", st);
    k_ntt_dif_scale<<<(unsigned)(n / tile), threads, (size_t)tile * 32, st>>>((uint4*)h, log_n, k0,
                                                                            (const uint4*)t.d_tw_inv,
                                                                            (const uint4*)t.d_coset_inv);
    return cudaGetLastError();
}

cudaError_t ntt_forward(const NttTables& t, void* a, cudaStream_t st) { return dit_natural(t, a, t.d_tw, nullptr, st); }

cudaError_t ntt_inverse(const NttTables& t, void* a, cudaStream_t st) {
    size_t n = (size_t)1 << t.log_n;
    return dit_natural(t, a, t.d_tw_inv, (const uint8_t*)t.d_coset + n * 32, st);
}

cudaError_t ntt_distribute_powers(void* a, size_t n, const uint64_t* shift_mont, cudaStream_t st) {
    g16d::Fr s;
    std::memcpy(s.v, shift_mont, 32);
    TimedLaunch tl("ntt_distribute", st);
    k_distribute<<<blocks_for((n + 15) / 16, 128), 128, 0, st>>>((uint4*)a, s, n);
    return cudaGetLastError();
}

}  // namespace g16

namespace g16 {

using g16d::NttJob;

void NttBatch::release() {
    cudaFree(d_jobs);
    d_jobs = nullptr;
    cap_jobs = 0;
    phases.clear();
}

// The batch's launches.  Every transform runs iNTT -> coset -> NTT on its A,
// B and C and writes H = A B - C: its inverse outer passes (top stages first),
// the fused middle, its forward outer passes.  The transforms are aligned so
// that their middles share one launch: inverse phase m runs outer pass
// Dmax - 1 - m of every transform that has that many, forward phase m runs
// outer pass m.  C's last pass, which reads the finished A and B for the join,
// runs after every other phase, in one launch per kind of pass.
cudaError_t ntt_batch_setup(NttBatch& nb, const std::vector<NttBatchItem>& items, cudaStream_t st) {
    set_attrs();
    nb.phases.clear();
    std::vector<uint32_t> logs;
    std::vector<NttTiling> tilings;
    for (auto& it : items) {
        if (!it.t || it.t->log_n < 1) {
            set_error("batched NTT item without tables");
            return cudaErrorInvalidValue;
        }
        logs.push_back((uint32_t)it.t->log_n);
        tilings.push_back(it.t->tiling);
    }
    std::vector<NttJob> all;
    auto add_phase = [&](int kind, std::vector<NttJob>& jobs) {
        if (jobs.empty()) return;
        NttPhase ph;
        ph.kind = kind;
        ph.first = (uint32_t)all.size();
        ph.njobs = (uint32_t)jobs.size();
        uint32_t blocks = 0;
        size_t smem = 0;
        for (auto& j : jobs) {
            j.block_start = blocks;
            const uint32_t tile = kind == 2 ? (1u << j.k) : ((1u << j.k) << j.log_L);
            blocks += (uint32_t)(((size_t)1 << j.log_n) / tile);
            smem = std::max(smem, (size_t)tile * 32);
            ph.products += kind == 2 ? ((double)((size_t)1 << j.log_n) * (j.k + 1)) : ((double)((size_t)1 << j.log_n) / 2 * j.k);
            ph.bytes += 64.0 * (double)((size_t)1 << j.log_n) * (j.join_out ? 2 : 1);
        }
        ph.blocks = blocks;
        ph.smem = smem;
        all.insert(all.end(), jobs.begin(), jobs.end());
        nb.phases.push_back(ph);
    };
    auto pass_job = [&](size_t i, int v, const Pass& p, bool dif, bool join) {
        const NttBatchItem& it = items[i];
        NttJob j = {};
        j.data = (uint4*)(v == 0 ? it.a : v == 1 ? it.b : it.c);
        j.tw = (const uint4*)(dif ? it.t->d_tw_inv : it.t->d_tw);
        if (join) {
            j.join_a = (const uint4*)it.a;
            j.join_b = (const uint4*)it.b;
            j.join_out = (uint4*)it.h;
        }
        j.log_n = logs[i];
        j.s_lo = p.s_lo;
        j.k = p.k;
        j.log_L = p.log_L;
        return j;
    };
    auto mid_job = [&](size_t i, int v, uint32_t k0, bool join) {
        const NttBatchItem& it = items[i];
        NttJob j = {};
        j.data = (uint4*)(v == 0 ? it.a : v == 1 ? it.b : it.c);
        j.tw = (const uint4*)it.t->d_tw;
        j.tw_inv = (const uint4*)it.t->d_tw_inv;
        j.coset = (const uint4*)it.t->d_coset;
        if (join) {
            j.join_a = (const uint4*)it.a;
            j.join_b = (const uint4*)it.b;
            j.join_out = (uint4*)it.h;
        }
        j.log_n = logs[i];
        j.k = k0;
        return j;
    };
    for (const NttPhasePlan& ph : ntt_batch_plan(logs, tilings)) {
        std::vector<NttJob> jobs;
        for (const NttJobPlan& jp : ph.jobs)
            jobs.push_back(jp.kind == 2 ? mid_job(jp.item, jp.vec, jp.pass.k, jp.join)
                                        : pass_job(jp.item, jp.vec, jp.pass, jp.kind == 0, jp.join));
        add_phase(ph.kind, jobs);
    }
    const size_t need = (all.empty() ? 1 : all.size()) * sizeof(NttJob);
    if (need > nb.cap_jobs) {   // the job table only grows, in stream order (dev_realloc_async)
        nb.cap_jobs = 0;
        G16_CUDA(g16::dev_realloc_async(&nb.d_jobs, need + need / 2, st, false));
        nb.cap_jobs = need + need / 2;
    }
    if (!all.empty()) G16_CUDA(cudaMemcpyAsync(nb.d_jobs, all.data(), all.size() * sizeof(NttJob), cudaMemcpyHostToDevice, st));
    G16_CUDA(cudaStreamSynchronize(st));
    return cudaSuccess;
}

cudaError_t ntt_batch_run(const NttBatch& nb, cudaStream_t st) {
    for (const NttPhase& ph : nb.phases) {
        const NttJob* jobs = (const NttJob*)nb.d_jobs + ph.first;
        const char* name = ph.kind == 0 ? "ntt_pass_dif" : ph.kind == 1 ? "ntt_pass_dit" : "ntt_mid_fused";
        timer().add_units(name, ph.products);
        timer().add_bytes(name, ph.bytes);
        TimedLaunch tl(name, st);
        if (ph.kind == 0) k_ntt_pass_multi<true><<<ph.blocks, 256, ph.smem, st>>>(jobs, ph.njobs);
        else if (ph.kind == 1) k_ntt_pass_multi<false><<<ph.blocks, 256, ph.smem, st>>>(jobs, ph.njobs);
        else k_ntt_mid_multi<<<ph.blocks, 256, ph.smem, st>>>(jobs, ph.njobs);
        G16_CUDA(cudaGetLastError());
    }
    return cudaSuccess;
}

}  // namespace g16
