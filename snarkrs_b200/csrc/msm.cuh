// Pippenger MSM engine for BN254 G1 / G2 on sm_100a (host interface).
//
// Replaces the reference's CUDA MSM (crates/cuda/src/msm.rs + kernels/msm.cu:
// count / scan / scatter / segmented accumulate / merge / reduce, host
// Horner at msm.rs:3976-4010) and implements the MsmBackend contract of
// crates/msm/src/lib.rs:52-82: sum_i k_i P_i, scalars in standard or
// Montgomery form, infinity bases and zero scalars contribute nothing.
//
// Pipeline, all on one stream, no host synchronisation until the window
// sums are read back:
//   1. digits: signed c-bit digits over 255 bits (carry-free recoding, the
//      same digit set as crates/msm/src/lib.rs:319-333), per-(window,bucket)
//      histogram with warp-aggregated atomics;
//   2. exclusive scan -> bucket offsets; scatter of (point index | sign) into
//      bucket order: a counting sort of (window, bucket, point) keys;
//   3. accumulate: the sorted list is cut into chunks whose length the
//      device picks from the entry count, one thread per chunk adds its
//      points into XYZZ partial bucket sums, so a fat bucket (a repeated
//      witness value) is spread over many threads;
//   4. fat buckets (more than a few partials, e.g. every scalar equal to 1)
//      are folded by blocks in two tree stages; then one thread per bucket
//      sums its partials into S_b;
//   5. the reduction sum_b (b+1) S_b: threads fold pieces of seg buckets by
//      running sums, blocks split the pieces' weights over their bits in
//      shared memory (msm_reduce_plan), a second kernel sums the blocks' bit
//      terms per set; no step has a long dependent chain, since a dependent
//      XYZZ addition costs microseconds of latency;
//   6. host: each set's sum from its bit terms, then Horner over the W
//      window sums (c doublings between windows).
// One sort serves every base vector that shares the scalars: the prover
// sorts the witness once and accumulates A, B1, L (G1) and B2 (G2) from it.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "host_bn254.hpp"

namespace g16 {

// Bucket reduction plan for `sets` bucket sets of B buckets each (B a power of
// two).  A set's sum is sum_b (b + 1) S_b.  Its buckets are cut into pieces of
// seg buckets (one thread's running sums), 2^lb pieces per block (lb =
// MSM_REDUCE_LB_G1 or _G2 below; a block keeps two arrays of 2^lb points in
// shared memory), nb = 2^hb blocks per set.  Each block leaves lb + 2 points, T, G_0 .. G_(lb-1)
// and its run total R; with more than two blocks in all, a second kernel sums
// them per set into lb + 1 + hb points, T, G_0 .. G_(lb-1), Gb_0 .. Gb_(hb-1),
// and the host forms
//   set sum = T + seg (sum_j 2^j G_j + 2^lb sum_i 2^i Gb_i).
// seg grows (up to 32) until the pieces over all sets number at most the
// target.  Fewer, longer pieces keep the reduction's footprint small where it
// runs beside other MSMs' accumulations, whose 512-thread blocks need a whole
// SM: the prover's window-shifted MSMs (one bucket set) aim at 8192 pieces,
// measured best for the 2^21-constraint prove (45.7 proofs/s against 44.1
// with 32768) and equal at 2^17.  A standalone MSM (one set per window) has
// the GPU to itself and aims at 32768, shortening the chains; so does the
// prover's H MSM (MsmSort::reduce_pieces), whose reduction runs last, when the
// witness MSMs' accumulations are mostly done.
constexpr uint64_t MSM_REDUCE_PIECES = 8192;
constexpr uint64_t MSM_REDUCE_PIECES_ALONE = 32768;
constexpr uint32_t MSM_REDUCE_MAX_SEG = 32;
constexpr uint64_t msm_reduce_pieces(bool shared_windows) {
    return shared_windows ? MSM_REDUCE_PIECES : MSM_REDUCE_PIECES_ALONE;
}

// Pieces per reduction block, 2^LB: one block of 2^LB threads halves its pieces'
// run sums LB times.  The pieces kernels hold ~250 registers a thread, so 2^8
// threads is the largest block an SM takes, and a block of 2^8 fills one SM's
// register file.  The reduction's chains are latency-bound and run beside the
// other MSMs' accumulations, whose 512-thread blocks each need a whole SM:
// 8192 pieces as 32 blocks of 2^8 hold 32 SMs, as 64 blocks of 2^7 (or 128 of
// 2^6, G2) up to 64 (128).  Measured on the 2^21-constraint prove: 2^8 for both
// groups 53.55-53.61 proofs/s against 53.04-53.20 with 2^7 (G1) and 2^6 (G2),
// the batched workload 1179-1221 against 1135-1156, although the reduction's
// own serialized time grows from 2.95 to 3.54 ms per proof.
#ifndef G16_REDUCE_LB_G1
#define G16_REDUCE_LB_G1 8
#endif
#ifndef G16_REDUCE_LB_G2
#define G16_REDUCE_LB_G2 8
#endif
constexpr uint32_t MSM_REDUCE_LB_G1 = G16_REDUCE_LB_G1;
constexpr uint32_t MSM_REDUCE_LB_G2 = G16_REDUCE_LB_G2;

struct MsmReducePlan {
    uint32_t sets = 0, B = 0, seg = 1, lb = MSM_REDUCE_LB_G1, nb = 1, hb = 0;
    bool direct = true;   // the host reads the blocks' own points
    constexpr uint32_t block_terms() const { return lb + 2; }
    constexpr uint32_t set_terms() const { return direct ? nb * (lb + 2) : lb + 1 + hb; }
    constexpr size_t block_points() const { return (size_t)sets * nb * (lb + 2); }
    constexpr size_t result_points() const { return (size_t)sets * set_terms(); }
};

constexpr MsmReducePlan msm_reduce_plan(uint32_t sets, uint32_t B, bool g2, uint64_t pieces_target) {
    MsmReducePlan r;
    r.sets = sets;
    r.B = B;
    r.lb = g2 ? MSM_REDUCE_LB_G2 : MSM_REDUCE_LB_G1;
    r.seg = 1;
    while (r.seg < MSM_REDUCE_MAX_SEG && r.seg < B && (uint64_t)sets * B / r.seg > pieces_target) r.seg *= 2;
    const uint32_t pieces = B / r.seg;
    r.nb = (pieces >> r.lb) ? (pieces >> r.lb) : 1;
    r.hb = 0;
    while ((1u << r.hb) < r.nb) r.hb++;
    r.direct = (uint64_t)sets * r.nb <= 2;
    return r;
}

// The bucket-reduction layout of a batched MSM space (msm_batch_setup): its
// segments' buckets back to back (key_start), and per segment a plan with one
// bucket set, its first k_reduce_pieces_multi block, its first block-output
// point (each block writes plan.block_terms() points) and its first result
// point (plan.set_terms(), summed on the device).  One piece length for the
// space: its pieces about fill the SMs' resident reduction threads (two
// blocks of 2^lb, at most 256 threads, per SM), runs of at most 32 buckets;
// piece_len_override (a power of two up to 32) replaces it, and
// pieces_target (non-zero) replaces the per-segment target.  Host arithmetic
// only, so that the kernels' indexing can be checked against it on the CPU.
struct MsmSpaceReduceLayout {
    std::vector<MsmReducePlan> plans;
    std::vector<uint32_t> key_start, block_start, out_block, out_set;
    uint64_t K = 0, blocks = 0, block_points = 0, result_points = 0;
    uint32_t max_hb = 0, piece_len = 1;
};

inline MsmSpaceReduceLayout msm_space_reduce_layout(const std::vector<uint32_t>& seg_B, bool g2, uint64_t pieces_target,
                                                    uint32_t sms, uint32_t piece_len_override) {
    MsmSpaceReduceLayout L;
    const uint32_t lb = g2 ? MSM_REDUCE_LB_G2 : MSM_REDUCE_LB_G1;
    uint64_t K = 0;
    for (uint32_t B : seg_B) K += B;
    const uint64_t resident = (2ull << lb) < 256 ? (2ull << lb) : 256;
    const uint64_t fill = (uint64_t)sms * resident;
    while (L.piece_len < MSM_REDUCE_MAX_SEG && K / L.piece_len > fill) L.piece_len *= 2;
    if (piece_len_override >= 1 && piece_len_override <= MSM_REDUCE_MAX_SEG && !(piece_len_override & (piece_len_override - 1)))
        L.piece_len = piece_len_override;
    for (uint32_t B : seg_B) {
        const uint64_t target = pieces_target ? pieces_target : (B / L.piece_len ? B / L.piece_len : 1);
        MsmReducePlan pl = msm_reduce_plan(1, B, g2, target);
        pl.direct = false;   // every segment's block terms are summed on the device
        L.key_start.push_back((uint32_t)L.K);
        L.block_start.push_back((uint32_t)L.blocks);
        L.out_block.push_back((uint32_t)L.block_points);
        L.out_set.push_back((uint32_t)L.result_points);
        L.K += B;
        L.blocks += pl.nb;
        L.block_points += (uint64_t)pl.nb * pl.block_terms();
        L.result_points += pl.set_terms();
        if (pl.hb > L.max_hb) L.max_hb = pl.hb;
        L.plans.push_back(pl);
    }
    return L;
}

struct MsmSort {
    // parameters
    int c = 0, W = 0;
    uint32_t B = 0;        // buckets per window, 2^(c-1)
    uint32_t K = 0;        // W * B, or B when the windows share one bucket set
    uint32_t Ks = 0;       // buckets sorted into: K, or K + 1 with the constant-work sink bucket
    bool shared = false;   // entries index window-shifted bases (w * n + i), one bucket set
    bool constant_work = false;   // zero digits are sorted into the sink bucket K
    uint64_t reduce_pieces = 0;   // bucket-reduction piece target; 0: msm_reduce_pieces(shared)
    size_t n = 0;          // scalars sorted
    uint32_t chunk = 16;   // smallest accumulate chunk (buffers are sized for it)
    // device buffers (capacities in elements)
    uint32_t* d_scalars_std = nullptr;  size_t cap_scalars = 0;   // 8 u32 per scalar
    uint32_t* d_counts = nullptr;       size_t cap_k = 0;         // K + 1
    uint32_t* d_offsets = nullptr;                                // K + 1
    uint32_t* d_cursor = nullptr;                                 // K
    uint32_t* d_seg_base = nullptr;                               // K + 1
    uint32_t* d_fat_list = nullptr;                               // buckets with many partials
    uint32_t* d_scan_tmp = nullptr;     size_t cap_tmp = 0;
    uint32_t* d_entries = nullptr;      size_t cap_entries = 0;
    uint32_t* d_total = nullptr;                                  // [0] = M, [1] = S, [2] = fat buckets, [3] = L
    // the buffers are views into memory the struct does not own (the
    // allocation-free entry point's fixed scratch): a buffer too small for a
    // call is an error, never a cudaFree and cudaMalloc
    bool fixed = false;
    void release();
};

struct MsmAccum {
    void* d_partials = nullptr;    size_t cap_partials = 0;   // bytes
    void* d_buckets = nullptr;     size_t cap_buckets = 0;    // bytes, one XYZZ sum per bucket
    void* d_segments = nullptr;    size_t cap_segments = 0;   // bytes, the reduction blocks' points
    void* d_windows = nullptr;     size_t cap_windows = 0;    // bytes
    unsigned long long* d_work = nullptr;                      // mixed additions performed
    MsmReducePlan plan;                                        // shape of d_windows
    bool fixed = false;                                        // views, as MsmSort::fixed
    size_t result_bytes(size_t xyzz_bytes) const { return plan.result_points() * xyzz_bytes; }
    void release();
};

// Window width for m scalars that reach the buckets.  The reference CPU model
// (crates/msm/src/lib.rs:160-172) with the GPU's cheaper bucket reduction.
int msm_window_bits(size_t m);

// Sort n device-resident scalars (32 bytes each; montgomery != 0 converts
// from Montgomery form first).  c = 0 picks msm_window_bits(n).
// shared_windows: the bases are the window-shifted table 2^(c w) P_i laid out
// at w * n + i (msm_window_table); all windows then fall into one bucket set
// and the result needs no Horner step.
// constant_work (the reference's Work::Constant, crates/msm/src/lib.rs:206-220):
// every window of every scalar becomes an entry, zero digits included, which
// go to a sink bucket K that no reduction reads; the entry count, the
// accumulate launch and its additions then follow the key, not the witness.
cudaError_t msm_sort(MsmSort& s, const void* d_scalars, size_t n, bool montgomery, int c, cudaStream_t st,
                     bool shared_windows = false, bool constant_work = false);

// One scalar vector sorted for several MSMs over window-shifted tables whose
// bases differ in which are at infinity (the prover's witness MSMs: A; B1 and
// B2; L).  Set j keeps scalar i when d_rank[j][i] != MSM_DEAD, and its entries
// name row d_rank[j][i] of the set's own table of rows[j] bases (infinity
// bases compacted out): entry w * rows[j] + d_rank[j][i].  The digits are
// computed once and each lands in every set its scalar is live in, so a base
// at infinity costs no accumulate step (the reference's prescan and key_live:
// crates/msm/src/lib.rs:534-563, crates/cuda/src/msm.rs:1308).  sorts[j] gets
// set j's sort, as msm_sort(shared_windows = true) would give for it.  With
// shared = false the sets read plain (compacted) bases instead: one bucket set
// per window and entry d_rank[j][i], as msm_sort(shared_windows = false).
constexpr uint32_t MSM_DEAD = 0xffffffffu;
constexpr int MSM_MAX_SETS = 3;
struct MsmLiveSets {
    int count = 0;
    const uint32_t* d_rank[MSM_MAX_SETS] = {nullptr, nullptr, nullptr};
    uint32_t rows[MSM_MAX_SETS] = {0, 0, 0};
};
cudaError_t msm_sort_sets(MsmSort* sorts, const MsmLiveSets& sets, const void* d_scalars, size_t n, bool montgomery,
                          int c, cudaStream_t st, bool constant_work = false, bool shared = true);

// Window count for c-bit signed digits over 255 bits.
inline int msm_windows(int c) { return (255 + c - 1) / c; }
// Window width for window-shifted bases: the cost is ~m * ceil(255/c) mixed
// additions plus a single bucket reduction over 2^(c-1) buckets.
int msm_shared_window_bits(size_t m);

// Build the window-shifted base table: out[w * n + i] = 2^(c w) P_i, affine,
// for i < n, where P_i = in[i - skip] for i >= skip and infinity below skip.
// Fixed-base multiplication (key generation): out[i] = k_i G (affine, packed;
// the point at infinity for k_i = 0), k_i Montgomery Fr on the device, with
// table[w * 256 + d] = d 2^(8 w) G packed affine (32 x 256 entries).
cudaError_t fixed_base_g1(const void* d_table, const void* d_scalars, size_t n, void* d_out, cudaStream_t st);
cudaError_t fixed_base_g2(const void* d_table, const void* d_scalars, size_t n, void* d_out, cudaStream_t st);

cudaError_t msm_window_table_g1(const void* d_in, size_t n, uint32_t skip, int c, void* d_out, cudaStream_t st);
cudaError_t msm_window_table_g2(const void* d_in, size_t n, uint32_t skip, int c, void* d_out, cudaStream_t st);

// Accumulate bases against a sorted scalar set and reduce to W window sums
// (XYZZ, device, in acc.d_windows).  Entry i uses base i - base_offset; entries
// below base_offset or at/after base_offset + n_bases are skipped.
cudaError_t msm_accumulate_g1(const MsmSort& s, MsmAccum& acc, const void* d_bases, uint32_t base_offset,
                              uint32_t n_bases, cudaStream_t st);
cudaError_t msm_accumulate_g2(const MsmSort& s, MsmAccum& acc, const void* d_bases, uint32_t base_offset,
                              uint32_t n_bases, cudaStream_t st);

// Host side: the reduction's points (acc.d_windows as copied back, laid out by
// plan) -> each set's sum -> Horner over the sets with c doublings between
// them -> Jacobian.
G1J msm_combine_g1(const uint8_t* result_xyzz, const MsmReducePlan& plan, int c);
G2J msm_combine_g2(const uint8_t* result_xyzz, const MsmReducePlan& plan, int c);

constexpr size_t XYZZ_G1_BYTES = 128;
constexpr size_t XYZZ_G2_BYTES = 256;

// The prover reads each of its five MSM results (the reduction's points) back
// into a pinned host slot of this many bytes: one bucket set with window tables;
// with a compact key one set per window, W (lb + 1 + hb) points.
constexpr size_t MSM_RESULT_SLOT_BYTES = 32 * 256;
constexpr size_t MSM_RESULT_SLOT_COMPACT_BYTES = 128 * 1024;

// ---- batched MSMs (many MSMs in one launch per step) ----
// A space holds the buckets of many MSMs of one group (segments) back to back;
// sources are device scalar vectors (Montgomery Fr), each sorted into up to
// MSM_MAX_TARGETS segments of any spaces in one digits pass and one scatter
// pass.  One accumulate launch per space then adds every entry of every
// segment, each against its own window-shifted table, and one reduction pass
// reduces every segment's bucket set.  Batched proving uses three spaces: the
// witnesses' G1 MSMs (A, B1, L of every proof), their G2 MSMs (B2) and the H
// MSMs.
constexpr int MSM_MAX_TARGETS = 4;

struct MsmSpaceSeg {
    uint32_t B = 0;                  // buckets, 2^(c-1) for the source's window bits c
    const void* table = nullptr;     // window-shifted bases (msm_window_table), rows x W entries
    uint32_t n_bases = 0;            // entries of the table
    // laid out by msm_batch_setup
    uint32_t key_start = 0;          // first bucket in the space
    MsmReducePlan plan;              // one set of B buckets; the sets kernel always runs
    uint32_t block_start = 0, out_block = 0, out_set = 0;
};

struct MsmSpace {
    bool g2 = false;
    // reduction pieces per segment; 0: every segment's buckets run in pieces of
    // one length, chosen from the space's bucket count so that the pieces of
    // all segments about fill the device
    uint64_t pieces_target = 0;
    std::vector<MsmSpaceSeg> segs;
    // laid out by msm_batch_setup
    uint32_t K = 0;                  // buckets over all segments
    uint32_t blocks = 0;             // reduction blocks over all segments
    uint32_t max_hb = 0;
    uint32_t result_points = 0;      // points of acc.d_windows the host reads
    size_t max_entries = 0;
    MsmSort sort;                    // sort buffers over the whole space
    MsmAccum acc;                    // partials, bucket sums, blocks' points (d_segments), results (d_windows)
    void* d_segdev = nullptr;        // accumulate descriptors
    void* d_reduce = nullptr;        // reduction descriptors
    size_t cap_segdev = 0, cap_reduce = 0;
    void release();
};

struct MsmSourceTgt {
    int space = 0, seg = 0;          // index into the spaces passed to msm_batch_setup, and segment
    const uint32_t* d_rank = nullptr;   // scalar -> table row, MSM_DEAD for a base at infinity; nullptr: identity
    uint32_t rows = 0;               // table rows of the segment
};

struct MsmSourceSpec {
    const void* d_scalars = nullptr; // Montgomery Fr on the device
    uint32_t n = 0;
    int c = 0;                       // window bits (its segments have B = 2^(c-1))
    int ntargets = 0;
    MsmSourceTgt t[MSM_MAX_TARGETS];
};

struct MsmSources {
    std::vector<MsmSourceSpec> srcs;
    uint32_t total_blocks = 0;
    void* d_desc = nullptr;
    uint32_t* d_blk = nullptr;
    void* d_std = nullptr;           // standard-form copies of the scalars
    size_t cap_desc = 0, cap_blk = 0, cap_std = 0;   // bytes; the buffers only grow
    void release();
};

// Lays out every space's segments (keys, reduction plans), grows the spaces'
// buffers to the entries the sources can produce, and uploads the descriptors;
// buffers are kept across calls (only grown), so a new layout of a similar
// batch allocates nothing.  Synchronises st.
cudaError_t msm_batch_setup(MsmSources& so, MsmSpace* const* spaces, int nspaces, cudaStream_t st);
// Sorts every source into its segments (no host synchronisation).
cudaError_t msm_batch_sort(MsmSources& so, MsmSpace* const* spaces, int nspaces, cudaStream_t st);
// Accumulates and reduces every segment of one space: results in
// sp.acc.d_windows, sp.result_points points (no host synchronisation).
cudaError_t msm_space_accumulate(MsmSpace& sp, cudaStream_t st);
// Host: segment s's sum from the space's results as read back.
G1J msm_space_combine_g1(const uint8_t* results, const MsmSpace& sp, size_t s);
G2J msm_space_combine_g2(const uint8_t* results, const MsmSpace& sp, size_t s);

// kernel-time accounting hook (events around each kernel class), optional
struct KernelTimer;
void msm_set_timer(KernelTimer* t);

}  // namespace g16
