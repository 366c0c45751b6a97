// Internal: the prover's handle types and helpers shared by prover.cu (single
// proofs, the C ABI) and batch.cu (batched proving).  Not part of the C ABI.
#pragma once
#include <atomic>
#include <condition_variable>
#include <memory>
#include <mutex>
#include <vector>
#include <cuda_runtime.h>
#include "common.cuh"
#include "g16b200.h"
#include "host_bn254.hpp"
#include "msm.cuh"
#include "ntt.cuh"

namespace g16 {
struct BatchPool;   // batched proving (batch.cu)
}

struct g16_backend {
    int ordinal = 0;
    uint64_t vram_limit = 0;
    std::atomic<uint64_t> vram_used{0};
    std::atomic<bool> constant_work{false};   // Work::Constant for every MSM of this backend
    cudaStream_t stream = nullptr;
    std::mutex mu;   // primitives share the scratch below
    g16::MsmSort sort;
    g16::MsmAccum acc;
    void* d_in = nullptr;
    size_t cap_in = 0;
    void* d_in2 = nullptr;
    size_t cap_in2 = 0;
    std::vector<std::unique_ptr<g16::NttTables>> ntt;   // by log_n
    uint8_t* h_pinned = nullptr;                   // window sums readback
    size_t cap_pinned = 0;
    unsigned long long* h_work = nullptr;
    std::mutex batch_mu;                           // guards batch
    g16::BatchPool* batch = nullptr;               // the batched-proving engines, built on first use
    std::atomic<uint64_t> batch_submissions{0}, batch_layouts{0}, batch_replays{0}, batch_grown{0}, batch_engines{0};
    std::atomic<int> fault{0};                     // sticky status that put this backend out of use (injected)
    std::atomic<int> inject{0};                    // fault for the next device entry point (g16_backend_inject_fault)
};

namespace g16 {

// The device state of one proof in flight.  A prepared circuit keeps a pool of
// these, so several proofs of the same circuit overlap on the GPU, each on its
// own five streams (the main one and one per witness MSM) with its own scratch.
struct Workspace {
    void* d_w = nullptr;       // witness, n_vars Fr
    void* d_abc = nullptr;     // A | B | C, n Fr each
    void* d_hpoly = nullptr;   // H, n Fr
    MsmSort sort_w[3], sort_h;  // witness sorts: the A, B (B1 and B2) and L live sets
    MsmAccum acc[5];           // A, B2, B1, L, H
    uint8_t* h_win = nullptr;  // pinned readback of the MSM results
    unsigned long long* h_work = nullptr;
    cudaStream_t stream = nullptr;             // gather -> NTT -> H MSM, and the join
    cudaStream_t side[4] = {nullptr, nullptr, nullptr, nullptr};   // witness MSMs A, B1, L, B2, one each
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_sort = nullptr;
    cudaEvent_t ev_side[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaGraphExec_t graph = nullptr;   // stages 0-9 captured once, replayed per proof
    uint64_t graph_kernels = 0;
    bool graph_constant_work = false;  // the mode the graph was captured in
    uint64_t proofs = 0;
    uint64_t bytes = 0;                // fixed device buffers
    size_t win_slot = 0;               // bytes of h_win per MSM

    cudaError_t init(uint32_t n_vars, uint32_t n, size_t slot) {
        win_slot = slot;
        cudaError_t e = g16::dev_malloc(&d_w, 32ull * n_vars);
        if (e == cudaSuccess) e = g16::dev_malloc(&d_abc, 32ull * n * 3);
        if (e == cudaSuccess) e = g16::dev_malloc(&d_hpoly, 32ull * n);
        if (e == cudaSuccess) e = cudaMallocHost((void**)&h_win, 5 * slot);
        if (e == cudaSuccess) e = cudaMallocHost((void**)&h_work, 16 * sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
        for (auto& x : side)
            if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking);
        for (auto& x : ev)
            if (e == cudaSuccess) e = cudaEventCreate(&x);
        for (cudaEvent_t* x : {&ev_fork, &ev_sort, &ev_side[0], &ev_side[1], &ev_side[2], &ev_side[3]})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(x, cudaEventDisableTiming);
        bytes = 32ull * n_vars + 32ull * n * 4;
        return e;
    }
    void release() {
        for (cudaStream_t s : {stream, side[0], side[1], side[2], side[3]})
            if (s) cudaStreamSynchronize(s);
        if (graph) cudaGraphExecDestroy(graph);
        cudaFree(d_w);
        cudaFree(d_abc);
        cudaFree(d_hpoly);
        for (auto& x : sort_w) x.release();
        sort_h.release();
        for (auto& a : acc) a.release();
        if (h_win) cudaFreeHost(h_win);
        if (h_work) cudaFreeHost(h_work);
        for (auto& x : ev)
            if (x) cudaEventDestroy(x);
        for (cudaEvent_t x : {ev_fork, ev_sort, ev_side[0], ev_side[1], ev_side[2], ev_side[3]})
            if (x) cudaEventDestroy(x);
        for (cudaStream_t s : {side[0], side[1], side[2], side[3], stream})
            if (s) cudaStreamDestroy(s);
        *this = Workspace();
    }
};

}  // namespace g16

struct g16_circuit {
    g16_backend* be = nullptr;
    uint32_t n_vars = 0, n_public = 0, n = 0;
    int log_n = 0;
    // resident key
    uint32_t *d_rp[2] = {nullptr, nullptr}, *d_sig[2] = {nullptr, nullptr}, *d_vid[2] = {nullptr, nullptr};
    void* d_values = nullptr;
    // the witness MSMs' bases with the points at infinity compacted out: A over
    // the A live set, B1 and B2 over the B set, L over the L set (live_sets)
    void *d_a = nullptr, *d_b1 = nullptr, *d_b2 = nullptr, *d_l = nullptr, *d_h = nullptr;
    uint32_t* d_rank[3] = {nullptr, nullptr, nullptr};   // wire -> row in the set's bases, or g16::MSM_DEAD
    uint32_t rows[3] = {0, 0, 0};                        // live wires of the A, B and L sets
    // window-shifted base tables 2^(c w) P_i at w * rows + i (msm_window_table);
    // all null when the key is held compact
    void *t_a = nullptr, *t_b1 = nullptr, *t_b2 = nullptr, *t_l = nullptr, *t_h = nullptr;
    int c_w = 0, c_h = 0;   // window bits of the witness and H MSMs
    // true: the MSMs read the window-shifted tables, all windows in one bucket
    // set; false (compact key, about a tenth of the memory): they read the plain
    // bases with one bucket set per window and a Horner step on the host
    bool tables = true;
    // a gnark key: no constraint matrices (proves only from A.w and B.w rows),
    // H taken as gnark's bit-reversed coefficients over h_count = n - 1 bases
    bool rows_only = false;
    uint32_t h_count = 0;   // H MSM length: n, or n - 1 for a gnark key
    g16::NttTables ntt;
    g16::G1A alpha1, beta1, delta1;
    g16::G2A beta2, delta2, gamma2;
    std::vector<g16::G1A> ic;               // verifying key: constant wire, then the public inputs
    // workspaces: one per proof in flight
    std::mutex mu;
    std::condition_variable cv;
    std::vector<std::unique_ptr<g16::Workspace>> pool;
    std::vector<g16::Workspace*> idle;
    uint32_t max_workspaces = 8;
    uint64_t ws_estimate = 0;          // device bytes of one workspace, scratch included
    bool serial = false;               // every stage on one stream (profiling)
    bool graphs = true;                // replay proofs as captured CUDA graphs
    bool tuning = false;               // g16_autotune / g16_tuning_set running: no new proofs start
    uint32_t batch_users = 0;          // batched submissions reading this circuit's tables (no tuning meanwhile)
    g16_tuning tuned = {0, 0, 0, 0, 0.0, 0.0};
    g16_stage_timings t = {0, 0, 0, 0, 0, 0};
    uint64_t readback_bytes = 0;       // device-to-host bytes of the last proof
    uint64_t device_bytes = 0;
    std::vector<void*> allocs;
};


namespace g16 {

// Error helpers: set the thread's last error text and return the status.
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
// G16_FAULT_* classes of a cudaError_t value (g16_cuda_error_class).
int error_class(int code);
// G16_OK, or the refusal of a device put out of use by a sticky fault; also
// delivers an injected fault.  First call of every entry point using b's device.
int device_usable(g16_backend* b);
// The sticky status that took device `ordinal` out of use in this process, or 0.
int device_fault(int ordinal);

// The key-only products of stage 11 (BlinderTerms::new, crates/groth16/src/prove.rs:335-346).
struct BlinderTerms {
    G1J d1r, d1s, d1rs;
    G2J d2s;
};
BlinderTerms blinder_terms(const g16_circuit* c, const Fr& r, const Fr& s);

// The five MSM outputs of one proof.
struct MsmJac {
    G1J a, b1, l, h;
    G2J b2;
};
// Stage 11: pi_A, pi_B, pi_C and the affine proof (assemble_from_terms, prove.rs:391-430).
void assemble(const g16_circuit* c, const MsmJac& m, const BlinderTerms& t, const Fr& r, const Fr& s, g16_proof* out);
// WitnessLength / ConstantWire checks (prove.rs:272-283); w_host may be null.
int check_witness(const g16_circuit* c, size_t n, const uint8_t* w_host);

// Batched proving over one launch per stage (batch.cu); G16_OK, or a status
// with the error set.  G16_ERR_DEVICE_MEMORY before any launch means the batch
// does not fit and the caller may prove it another way.
int prove_batch_engine(g16_backend* b, size_t count, g16_circuit* const* circuits, const uint8_t* const* witnesses,
                       const size_t* lens, const uint8_t* r, const uint8_t* s, g16_proof* out, double* done_ms);
// Sizes every engine of the backend (creating them up to their limit) for a
// batch of these circuits without proving it, taking each engine in turn when idle.
int reserve_batch_engines(g16_backend* b, g16_circuit* const* circuits, size_t count);
// Drops the batched-proving engine's state that refers to circuit c (before c is freed).
void batch_forget(g16_backend* b, const g16_circuit* c);
// Frees the batched-proving engine of a backend.
void batch_free(g16_backend* b);

}  // namespace g16
