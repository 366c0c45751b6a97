// Radix-2 Fr NTT on sm_100a (host interface).
//
// Replaces the reference's CUDA stages 1-3 (crates/cuda/src/kernels/ntt.cu:
// g16_ntt_head / g16_ntt_tail) and the CPU CpuNtt API
// (crates/ntt/src/lib.rs:415-584).  Values are fixed by the mathematics (a
// DFT over omega_n = TWO_ADIC_ROOT^(2^(28 - log n)), crates/field/src/lib.rs:46-84),
// so outputs are bit-identical to the CPU's whatever the pass structure.
//
// Structure: a transform of 2^log_n is cut into shared-memory passes.  The
// inner pass covers stages [0, k0) on contiguous tiles of 2^k0 elements; the
// outer passes cover the remaining stages on tiles gathered with stride
// 2^s_lo (L consecutive columns per tile for 128-byte segments).  The
// prover's iNTT -> coset -> NTT chain runs DIF (natural -> bit-reversed) for
// the inverse and DIT (bit-reversed -> natural) for the forward, so the two
// inner passes and the coset multiply in between fuse into one kernel and no
// bit-reversal pass exists; the forward's last pass of C also fuses
// H = A*B - C (crates/groth16/src/cpu.rs:230-246, no division by Z).
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

namespace g16 {

// Tiling of the shared-memory passes: the inner pass works on contiguous
// tiles of 2^tile_log elements, each outer pass on tiles of 2^k * 2^outer_log_l
// elements with k <= tile_log - outer_log_l (2^outer_log_l consecutive
// columns per tile row).  The values are the same for every tiling; only the
// number of passes over HBM and the shared-memory footprint change.
struct NttTiling {
    uint32_t tile_log = 11;      // 2048 elements, 64 KiB of shared memory
    uint32_t outer_log_l = 2;    // 4 columns = 128-byte rows
};
constexpr uint32_t NTT_MAX_TILE_LOG = 12;   // 128 KiB of shared memory

// Is the tiling one the kernels accept?
inline bool ntt_tiling_valid(const NttTiling& t) {
    return t.tile_log >= 2 && t.tile_log <= NTT_MAX_TILE_LOG && t.outer_log_l < t.tile_log && t.outer_log_l <= 4;
}

// The passes of a transform of 2^log_n under a tiling (host arithmetic only, so
// that the kernels' indexing can be checked against it on the CPU): the inner
// pass covers stages [0, k0) on contiguous tiles of 2^k0; each outer pass covers
// stages [s_lo, s_lo + k) on tiles of 2^k rows of 2^log_L consecutive columns.
struct NttPass {
    uint32_t s_lo, k, log_L;
};

// the inner pass's stage count
inline uint32_t ntt_inner_k(const NttTiling& tl, uint32_t log_n) { return log_n < tl.tile_log ? log_n : tl.tile_log; }

// outer passes covering stages [k0, log_n) in increasing s_lo, as even as the
// tile's row count 2^(tile_log - outer_log_l) allows
inline std::vector<NttPass> ntt_outer_passes(const NttTiling& tl, uint32_t log_n, uint32_t k0) {
    std::vector<NttPass> v;
    uint32_t rem = log_n - k0;
    if (!rem) return v;
    uint32_t kmax = tl.tile_log - tl.outer_log_l;
    uint32_t np = (rem + kmax - 1) / kmax;
    uint32_t s = k0;
    for (uint32_t i = 0; i < np; i++) {
        uint32_t k = rem / np + (i < rem % np ? 1 : 0);
        uint32_t ll = tl.outer_log_l < s ? tl.outer_log_l : s;
        v.push_back({s, k, ll});
        s += k;
    }
    return v;
}

struct NttTables {
    int log_n = -1;
    NttTiling tiling;
    void* d_tw = nullptr;       // omega^i, i < n/2 (Montgomery Fr)
    void* d_tw_inv = nullptr;   // omega^-i, i < n/2
    void* d_coset = nullptr;    // shift^bitrev(p) / n, p < n (the proving coset shift omega_2n)
    void* d_coset_inv = nullptr;   // shift^-bitrev(p) / n, for gnark keys only (ntt_gnark_table)
    uint64_t n_inv[4];          // 1/n, Montgomery
    uint64_t shift[4];          // omega_2n, Montgomery
    void release();
};

// Build (or keep) the tables for 2^log_n on the device, log_n in [1, 27].
cudaError_t ntt_tables(NttTables& t, int log_n, cudaStream_t st);

// The prover's stages 1-4 on device vectors of n = 2^log_n: A, B, C each go
// iNTT -> * shift^i/n -> NTT (natural order in and out, in place) and
// h = A*B - C is written to h (may alias none of A, B, C).
cudaError_t ntt_h_pipeline(const NttTables& t, void* a, void* b, void* c, void* h, cudaStream_t st);

// For a gnark key: the table shift^-bitrev(p) / n (built once), and H's values
// on the odd coset -> H's coefficients, times -2, in bit-reversed order: the
// inverse transform to bit-reversed order, then position p times
// shift^-bitrev(p) / n (intt_to_bitrev + coset_scale_bitrev,
// crates/groth16/src/cpu.rs:265-286).  In place on 2^log_n Fr.
cudaError_t ntt_gnark_table(NttTables& t, cudaStream_t st);
cudaError_t ntt_to_gnark_coefficients(const NttTables& t, void* h, cudaStream_t st);

// One vector through the same chain (the reference's intt_coset_ntt).
cudaError_t ntt_intt_coset_ntt(const NttTables& t, void* a, cudaStream_t st);

// Standalone transforms, natural order in and out.
cudaError_t ntt_forward(const NttTables& t, void* a, cudaStream_t st);
cudaError_t ntt_inverse(const NttTables& t, void* a, cudaStream_t st);   // includes the 1/n scale
// a[i] *= shift^i (crates/ntt/src/lib.rs:582), shift Montgomery
cudaError_t ntt_distribute_powers(void* a, size_t n, const uint64_t* shift_mont, cudaStream_t st);

// ---- many prover chains per launch (batched proving) ----
// ntt_h_pipeline for many proofs of any sizes and tilings: every launch
// covers one step of every chain (ntt_batch_setup lays the steps out).
// The launches of a batch of H pipelines (ntt_batch_setup) before they are
// bound to device vectors.  A job is item `item`'s vector `vec` (0 A, 1 B, 2 C)
// in an outer pass (kind 0: inverse DIF with inverse twiddles, 1: forward DIT)
// or in the fused middle (kind 2; pass.k = the inner stage count); `join`:
// its epilogue writes h = A B - C instead of the vector.  The jobs of a phase
// run in one launch, side by side.  Phases: the inverse outer passes
// right-aligned (an item with fewer passes joins later), the middles (of A and
// B only for an item without outer passes), the forward outer passes
// left-aligned (an item's last one for A and B only), then C's last step with
// the join: the middles of items without outer passes, then the last forward
// passes.  Host arithmetic only, so that the order can be checked on the CPU.
struct NttJobPlan {
    uint32_t item;
    int vec, kind;
    NttPass pass;
    bool join;
};
struct NttPhasePlan {
    int kind;
    std::vector<NttJobPlan> jobs;
};

inline std::vector<NttPhasePlan> ntt_batch_plan(const std::vector<uint32_t>& log_n, const std::vector<NttTiling>& tiling) {
    const size_t n = log_n.size();
    std::vector<uint32_t> k0(n);
    std::vector<std::vector<NttPass>> outer(n);
    size_t dmax = 0;
    for (size_t i = 0; i < n; i++) {
        k0[i] = ntt_inner_k(tiling[i], log_n[i]);
        outer[i] = ntt_outer_passes(tiling[i], log_n[i], k0[i]);
        if (outer[i].size() > dmax) dmax = outer[i].size();
    }
    std::vector<NttPhasePlan> phases;
    auto add = [&](int kind, std::vector<NttJobPlan>& jobs) {
        if (!jobs.empty()) phases.push_back({kind, jobs});
    };
    for (size_t m = 0; m < dmax; m++) {   // inverse outer passes, right-aligned
        std::vector<NttJobPlan> jobs;
        const size_t q = dmax - 1 - m;
        for (uint32_t i = 0; i < n; i++)
            if (outer[i].size() > q)
                for (int v = 0; v < 3; v++) jobs.push_back({i, v, 0, outer[i][q], false});
        add(0, jobs);
    }
    {
        std::vector<NttJobPlan> jobs;
        for (uint32_t i = 0; i < n; i++)
            for (int v = 0; v < (outer[i].empty() ? 2 : 3); v++) jobs.push_back({i, v, 2, {0, k0[i], 0}, false});
        add(2, jobs);
    }
    for (size_t m = 0; m < dmax; m++) {   // forward outer passes, left-aligned
        std::vector<NttJobPlan> jobs;
        for (uint32_t i = 0; i < n; i++) {
            const size_t np = outer[i].size();
            if (m >= np) continue;
            for (int v = 0; v < (m + 1 == np ? 2 : 3); v++) jobs.push_back({i, v, 1, outer[i][m], false});
        }
        add(1, jobs);
    }
    {   // C's last step with the join
        std::vector<NttJobPlan> mids, passes;
        for (uint32_t i = 0; i < n; i++) {
            if (outer[i].empty()) mids.push_back({i, 2, 2, {0, k0[i], 0}, true});
            else passes.push_back({i, 2, 1, outer[i].back(), true});
        }
        add(2, mids);
        add(1, passes);
    }
    return phases;
}

struct NttBatchItem {
    const NttTables* t;     // the proof's domain tables and tiling
    void *a, *b, *c, *h;    // device vectors of 2^t->log_n Fr; h = A B - C out
};
struct NttPhase {
    int kind = 0;           // 0 inverse outer pass, 1 forward outer pass, 2 fused middle
    uint32_t first = 0, njobs = 0, blocks = 0;
    size_t smem = 0;
    double products = 0, bytes = 0;   // algorithmic work, for the kernel timer
};
struct NttBatch {
    std::vector<NttPhase> phases;
    void* d_jobs = nullptr;
    size_t cap_jobs = 0;    // bytes; the job table only grows
    void release();
};
// Lays out and uploads the launches for the items (synchronises st).
cudaError_t ntt_batch_setup(NttBatch& nb, const std::vector<NttBatchItem>& items, cudaStream_t st);
// Enqueues them (no host synchronisation).
cudaError_t ntt_batch_run(const NttBatch& nb, cudaStream_t st);

}  // namespace g16
