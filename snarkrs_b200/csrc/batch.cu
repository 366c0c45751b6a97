// Batched proving: many proofs of any mix of prepared circuits, each stage of
// every proof in one launch.
//
// The reference proves one request per call (crates/groth16/src/prove.rs).
// Here a submission of jobs becomes one pass over the device: one gather
// launch for every job's rows, one launch per step of every job's
// iNTT -> coset -> NTT chain (ntt_batch_*), one sort of every witness into the
// G1 and G2 MSM spaces, one accumulate launch per space covering the A, B1 and
// L MSMs of every job (and one for every B2), one sort and one accumulate for
// every H MSM, and one bucket-reduction pass per space (msm_batch_*).  Each job
// keeps its circuit's own window sizes (tuning) and NTT tiling.  From the
// second submission of the same jobs' circuits on, the whole sequence over its
// three streams is captured once as a CUDA graph and replayed.  The host
// computes the key-only blinder products while the device runs, then
// assembles the proofs on a thread pool.  Results are bit-identical to single
// proofs.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <thread>
#include "common.cuh"
#include "gather.cuh"
#include "prover.hpp"

namespace g16d {

// One job's stage 0: rows of its circuit's CSR, witness and A | B | C.
struct GatherJob {
    const uint32_t* rp[2];
    const uint32_t* sig[2];
    const uint32_t* vid[2];
    const uint4* values;
    const uint4* w;
    uint4* abc;
    uint32_t n, block_start;
};

__global__ void __launch_bounds__(256) k_gather_multi(const GatherJob* __restrict__ jobs, uint32_t njobs) {
    uint32_t lo = 0, hi = njobs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].block_start <= blockIdx.x) lo = mid; else hi = mid;
    }
    const GatherJob& j = jobs[lo];
    const uint32_t row = (blockIdx.x - j.block_start) * 256 + threadIdx.x;
    if (row >= j.n) return;
    gather_row(row, j.rp[0], j.sig[0], j.vid[0], j.rp[1], j.sig[1], j.vid[1], j.values, j.w, j.abc,
               j.abc + 2 * (size_t)j.n, j.abc + 4 * (size_t)j.n);
}

}  // namespace g16d

namespace g16 {

#define CK_BATCH(call)                                               \
    do {                                                             \
        cudaError_t e__ = (call);                                    \
        if (e__ != cudaSuccess) return cuda_fail(e__, #call);        \
    } while (0)

// The state a job's plan depends on: its circuit, window sizes, tiling and tables.
struct BatchKey {
    const g16_circuit* c;
    int cw, ch;
    uint32_t tile, outer;
    const void *ta, *tb1, *tb2, *tl, *th;
    bool operator==(const BatchKey& o) const {
        return c == o.c && cw == o.cw && ch == o.ch && tile == o.tile && outer == o.outer && ta == o.ta &&
               tb1 == o.tb1 && tb2 == o.tb2 && tl == o.tl && th == o.th;
    }
};

static BatchKey key_of(const g16_circuit* c) {
    return {c, c->c_w, c->c_h, c->ntt.tiling.tile_log, c->ntt.tiling.outer_log_l, c->t_a, c->t_b1, c->t_b2, c->t_l,
            c->t_h};
}

// One batched submission's device state.  The buffers are kept across
// submissions and only grow, so a submission of a new mix of circuits (a new
// layout) allocates nothing once the engine has seen one as large; the layout
// itself (offsets, descriptors) is rebuilt when the mix changes, and the CUDA
// graph is kept for the layout it was captured for.
struct BatchEngine {
    std::vector<BatchKey> key;              // the layout built; empty: none
    uint64_t accounted = 0;                 // device bytes counted against the backend's budget
    void* d_arena = nullptr;
    size_t cap_arena = 0;
    std::vector<size_t> off_w, off_abc, off_h;
    MsmSpace g1, g2, hs;
    MsmSources src_w, src_h;
    NttBatch ntt;
    void* d_gather = nullptr;
    size_t cap_gather = 0;
    uint32_t gather_blocks = 0, gather_jobs = 0;
    uint8_t* h_res = nullptr;               // pinned: G1, G2 and H results, back to back
    size_t cap_res = 0;
    uint8_t* h_stage = nullptr;             // pinned: the jobs' witnesses, laid out as the arena's first region
    size_t cap_stage = 0;
    size_t w_bytes = 0;                     // bytes of that region
    size_t res_g1 = 0, res_g2 = 0, res_h = 0;
    cudaStream_t st[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_sorted = nullptr, ev_g1 = nullptr, ev_g2 = nullptr;
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_kernels = 0;
    int runs = 0;                           // submissions on the current layout

    // forget the layout (and its graph); the buffers stay
    void drop_layout() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_kernels = 0;
        runs = 0;
        key.clear();
        off_w.clear();
        off_abc.clear();
        off_h.clear();
        g1.segs.clear();
        g2.segs.clear();
        hs.segs.clear();
        src_w.srcs.clear();
        src_h.srcs.clear();
    }

    void release() {
        for (cudaStream_t s : st)
            if (s) cudaStreamSynchronize(s);
        drop_layout();
        g1.release();
        g2.release();
        hs.release();
        src_w.release();
        src_h.release();
        ntt.release();
        cudaFree(d_gather);
        cudaFree(d_arena);
        if (h_res) cudaFreeHost(h_res);
        if (h_stage) cudaFreeHost(h_stage);
        for (cudaEvent_t e : {ev_fork, ev_sorted, ev_g1, ev_g2})
            if (e) cudaEventDestroy(e);
        for (cudaStream_t s : st)
            if (s) cudaStreamDestroy(s);
        *this = BatchEngine();
    }
};

// The backend's engines: several submissions may run at once, each on its own
// engine and streams, so that one's host work (staging, assembly) overlaps
// another's device work.
struct BatchPool {
    std::vector<std::unique_ptr<BatchEngine>> all;
    std::vector<BatchEngine*> idle;
    std::condition_variable cv;
};

namespace {

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Device bytes a plan for these jobs takes, for the budget check before any allocation.
uint64_t plan_estimate(g16_circuit* const* cs, size_t count) {
    uint64_t b = 0;
    for (size_t j = 0; j < count; j++) {
        const g16_circuit* c = cs[j];
        const uint64_t Ww = (uint64_t)msm_windows(c->c_w), Wh = (uint64_t)msm_windows(c->c_h);
        const uint64_t Kw = 1ull << (c->c_w - 1), Kh = 1ull << (c->c_h - 1);
        const uint64_t ew = (uint64_t)(c->rows[0] + 2 * c->rows[1] + c->rows[2]) * Ww, eh = (uint64_t)c->n * Wh;
        b += 32ull * c->n_vars + 128ull * c->n + 32ull * (c->n_vars + c->n) + 2048;
        b += (ew + eh) * 4 + (4 * Kw + Kh) * 24;                                 // entries, sort buffers
        b += (3 * Kw * 2 + (ew - c->rows[1] * Ww) / 16) * XYZZ_G1_BYTES;          // G1 partials, buckets
        b += (Kw * 2 + c->rows[1] * Ww / 16) * XYZZ_G2_BYTES;
        b += (Kh * 2 + eh / 16) * XYZZ_G1_BYTES;
    }
    return b + (8ull << 20);
}

// device buffer that only grows, reallocated in stream order on st (the engine
// is idle when it grows; dev_realloc_async)
cudaError_t grow_dev(cudaStream_t st, void*& p, size_t& cap, size_t need) {
    if (p && need <= cap) return cudaSuccess;
    cap = 0;
    const size_t n = need + need / 4 + 256;
    cudaError_t e = g16::dev_realloc_async(&p, n, st, true);
    if (e == cudaSuccess) cap = n;
    return e;
}

// pinned host buffer that only grows; a page-locked allocation serialises the
// device's streams, so it grows to twice what it needs
cudaError_t grow_pinned(uint8_t*& p, size_t& cap, size_t need) {
    if (p && need <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t n = 2 * need + 256;
    cudaError_t e = cudaMallocHost((void**)&p, n);
    if (e == cudaSuccess) cap = n;
    if (e == cudaSuccess && value_fill_byte() >= 0) std::memset(p, value_fill_byte(), n);
    return e;
}

int build(BatchEngine& E, g16_circuit* const* cs, size_t count) {
    E.drop_layout();
    if (!E.st[0]) {
        for (cudaStream_t* s : {&E.st[0], &E.st[1], &E.st[2]})
            CK_BATCH(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&E.ev_fork, &E.ev_sorted, &E.ev_g1, &E.ev_g2})
            CK_BATCH(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    // arena: every job's witness (one region, filled by one copy from the pinned
    // staging buffer), then every job's A | B | C, then every job's H
    size_t off = 0;
    for (size_t j = 0; j < count; j++) {
        E.off_w.push_back(off);
        off = align256(off + 32ull * cs[j]->n_vars);
    }
    E.w_bytes = off;
    for (size_t j = 0; j < count; j++) {
        E.off_abc.push_back(off);
        off = align256(off + 96ull * cs[j]->n);
    }
    for (size_t j = 0; j < count; j++) {
        E.off_h.push_back(off);
        off = align256(off + 32ull * cs[j]->n);
    }
    CK_BATCH(grow_dev(E.st[0], E.d_arena, E.cap_arena, off));
    CK_BATCH(grow_pinned(E.h_stage, E.cap_stage, E.w_bytes));
    uint8_t* arena = (uint8_t*)E.d_arena;
    // MSM spaces: G1 (A, B1, L of every job), G2 (B2), H
    E.g1.g2 = false;
    E.g2.g2 = true;
    E.hs.g2 = false;
    // reduction pieces: one length per space, from its bucket count (msm_batch_setup)
    E.g1.pieces_target = E.g2.pieces_target = E.hs.pieces_target = 0;
    for (size_t j = 0; j < count; j++) {
        const g16_circuit* c = cs[j];
        const uint32_t Bw = 1u << (c->c_w - 1), Bh = 1u << (c->c_h - 1);
        const uint32_t Ww = (uint32_t)msm_windows(c->c_w), Wh = (uint32_t)msm_windows(c->c_h);
        MsmSpaceSeg s;
        s.B = Bw;
        s.table = c->t_a;
        s.n_bases = c->rows[0] * Ww;
        E.g1.segs.push_back(s);
        s.table = c->t_b1;
        s.n_bases = c->rows[1] * Ww;
        E.g1.segs.push_back(s);
        s.table = c->t_l;
        s.n_bases = c->rows[2] * Ww;
        E.g1.segs.push_back(s);
        s.table = c->t_b2;
        s.n_bases = c->rows[1] * Ww;
        E.g2.segs.push_back(s);
        s.B = Bh;
        s.table = c->t_h;
        s.n_bases = c->n * Wh;
        E.hs.segs.push_back(s);
        MsmSourceSpec w;
        w.d_scalars = arena + E.off_w[j];
        w.n = c->n_vars;
        w.c = c->c_w;
        w.ntargets = 4;
        w.t[0] = {0, (int)(3 * j), c->d_rank[0], c->rows[0]};
        w.t[1] = {0, (int)(3 * j + 1), c->d_rank[1], c->rows[1]};
        w.t[2] = {0, (int)(3 * j + 2), c->d_rank[2], c->rows[2]};
        w.t[3] = {1, (int)j, c->d_rank[1], c->rows[1]};
        E.src_w.srcs.push_back(w);
        MsmSourceSpec h;
        h.d_scalars = arena + E.off_h[j];
        h.n = c->n;
        h.c = c->c_h;
        h.ntargets = 1;
        h.t[0] = {0, (int)j, nullptr, c->n};
        E.src_h.srcs.push_back(h);
    }
    MsmSpace* wsp[2] = {&E.g1, &E.g2};
    MsmSpace* hsp[1] = {&E.hs};
    CK_BATCH(msm_batch_setup(E.src_w, wsp, 2, E.st[0]));
    CK_BATCH(msm_batch_setup(E.src_h, hsp, 1, E.st[0]));
    // the NTT chains and the gather
    std::vector<NttBatchItem> items;
    std::vector<g16d::GatherJob> gj;
    uint32_t blocks = 0;
    for (size_t j = 0; j < count; j++) {
        const g16_circuit* c = cs[j];
        uint8_t* abc = arena + E.off_abc[j];
        const size_t vb = 32ull * c->n;
        items.push_back({&c->ntt, abc, abc + vb, abc + 2 * vb, arena + E.off_h[j]});
        g16d::GatherJob g = {};
        for (int m = 0; m < 2; m++) {
            g.rp[m] = c->d_rp[m];
            g.sig[m] = c->d_sig[m];
            g.vid[m] = c->d_vid[m];
        }
        g.values = (const uint4*)c->d_values;
        g.w = (const uint4*)(arena + E.off_w[j]);
        g.abc = (uint4*)abc;
        g.n = c->n;
        g.block_start = blocks;
        blocks += (c->n + 255) / 256;
        gj.push_back(g);
    }
    CK_BATCH(ntt_batch_setup(E.ntt, items, E.st[0]));
    CK_BATCH(grow_dev(E.st[0], E.d_gather, E.cap_gather, gj.size() * sizeof(g16d::GatherJob)));
    // on st[0] and waited for: a plain cudaMemcpy from pageable memory may return
    // before its DMA lands, on the legacy stream, which orders nothing against
    // the engine's non-blocking streams (the gather would read the previous
    // layout's jobs)
    CK_BATCH(cudaMemcpyAsync(E.d_gather, gj.data(), gj.size() * sizeof(g16d::GatherJob), cudaMemcpyHostToDevice,
                             E.st[0]));
    CK_BATCH(cudaStreamSynchronize(E.st[0]));
    E.gather_blocks = blocks;
    E.gather_jobs = (uint32_t)gj.size();
    E.res_g1 = (size_t)E.g1.result_points * XYZZ_G1_BYTES;
    E.res_g2 = (size_t)E.g2.result_points * XYZZ_G2_BYTES;
    E.res_h = (size_t)E.hs.result_points * XYZZ_G1_BYTES;
    CK_BATCH(grow_pinned(E.h_res, E.cap_res, E.res_g1 + E.res_g2 + E.res_h + 64));
    for (size_t j = 0; j < count; j++) E.key.push_back(key_of(cs[j]));
    return G16_OK;
}

// Every stage of every job, over the engine's three streams, joined on st[0].
int enqueue(BatchEngine& E) {
    // with kernel timing on, every step runs on one stream, so that each
    // launch's event span is its own duration
    const bool serial = timer().enabled;
    cudaStream_t s0 = E.st[0], s1 = serial ? s0 : E.st[1], s2 = serial ? s0 : E.st[2];
    MsmSpace* wsp[2] = {&E.g1, &E.g2};
    MsmSpace* hsp[1] = {&E.hs};
    CK_BATCH(cudaEventRecord(E.ev_fork, s0));
    CK_BATCH(cudaStreamWaitEvent(s1, E.ev_fork, 0));
    // the witnesses' MSMs: one sort, then the G1 space on s1 and the G2 space on s2
    CK_BATCH(msm_batch_sort(E.src_w, wsp, 2, s1));
    CK_BATCH(cudaEventRecord(E.ev_sorted, s1));
    CK_BATCH(cudaStreamWaitEvent(s2, E.ev_sorted, 0));
    CK_BATCH(msm_space_accumulate(E.g2, s2));
    CK_BATCH(cudaMemcpyAsync(E.h_res + E.res_g1, E.g2.acc.d_windows, E.res_g2, cudaMemcpyDeviceToHost, s2));
    CK_BATCH(cudaEventRecord(E.ev_g2, s2));
    CK_BATCH(msm_space_accumulate(E.g1, s1));
    CK_BATCH(cudaMemcpyAsync(E.h_res, E.g1.acc.d_windows, E.res_g1, cudaMemcpyDeviceToHost, s1));
    CK_BATCH(cudaEventRecord(E.ev_g1, s1));
    // stage 0, the NTT chains and the H MSMs on s0
    if (E.gather_blocks) {
        TimedLaunch tl("gather", s0);
        g16d::k_gather_multi<<<E.gather_blocks, 256, 0, s0>>>((const g16d::GatherJob*)E.d_gather, E.gather_jobs);
    }
    CK_BATCH(cudaGetLastError());
    CK_BATCH(ntt_batch_run(E.ntt, s0));
    CK_BATCH(msm_batch_sort(E.src_h, hsp, 1, s0));
    CK_BATCH(msm_space_accumulate(E.hs, s0));
    CK_BATCH(cudaMemcpyAsync(E.h_res + E.res_g1 + E.res_g2, E.hs.acc.d_windows, E.res_h, cudaMemcpyDeviceToHost, s0));
    CK_BATCH(cudaStreamWaitEvent(s0, E.ev_g1, 0));
    CK_BATCH(cudaStreamWaitEvent(s0, E.ev_g2, 0));
    return G16_OK;
}

// Runs fn(i) for i < n on up to `threads` host threads.
template <class Fn>
void parallel_for(size_t n, size_t threads, Fn&& fn) {
    threads = std::max<size_t>(1, std::min(threads, n));
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i; (i = next.fetch_add(1)) < n;) fn(i);
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < threads; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
}

size_t host_threads() {
    size_t h = std::thread::hardware_concurrency();
    return std::max<size_t>(1, std::min<size_t>(h ? h : 4, 32));
}

}  // namespace

void batch_forget(g16_backend* b, const g16_circuit* c) {
    std::lock_guard<std::mutex> g(b->batch_mu);
    if (!b->batch) return;
    // engines in use belong to submissions whose circuits are alive; idle ones
    // holding a layout over c forget it
    for (BatchEngine* E : b->batch->idle)
        for (auto& k : E->key)
            if (k.c == c) {
                E->drop_layout();
                break;
            }
}

}  // namespace g16

int g16_batch_stats_get(const g16_backend* b, g16_batch_stats* out) {
    if (!b || !out) return g16::fail(G16_ERR_INVALID_ARGUMENT, "g16_batch_stats_get: null argument");
    out->submissions = b->batch_submissions.load();
    out->layouts = b->batch_layouts.load();
    out->replays = b->batch_replays.load();
    out->grown_bytes = b->batch_grown.load();
    out->engines = b->batch_engines.load();
    return G16_OK;
}

namespace g16 {

void batch_free(g16_backend* b) {
    std::lock_guard<std::mutex> g(b->batch_mu);
    if (!b->batch) return;
    for (auto& E : b->batch->all) {
        b->vram_used -= std::min<uint64_t>(b->vram_used, E->accounted);
        E->release();
    }
    delete b->batch;
    b->batch = nullptr;
}

// Engines a backend keeps (G16_BATCH_ENGINES, 1-8; default 4).
size_t batch_max_engines() {
    size_t n = 4;
    if (const char* e = std::getenv("G16_BATCH_ENGINES")) n = (size_t)std::max(1, std::min(8, std::atoi(e)));
    return n;
}

// While it lives, no circuit of the batch is retuned (g16_autotune waits for
// batch_users to drop to zero): the batch reads their tables.
struct BatchUsers {
    std::vector<g16_circuit*> cs;
    BatchUsers(g16_circuit* const* c, size_t n) : cs(c, c + n) {
        std::sort(cs.begin(), cs.end());
        cs.erase(std::unique(cs.begin(), cs.end()), cs.end());
        for (g16_circuit* x : cs) {
            std::unique_lock<std::mutex> lk(x->mu);
            x->cv.wait(lk, [&] { return !x->tuning; });
            x->batch_users++;
        }
    }
    ~BatchUsers() {
        for (g16_circuit* x : cs) {
            {
                std::lock_guard<std::mutex> g(x->mu);
                x->batch_users--;
            }
            x->cv.notify_all();
        }
    }
};

// Layout E for the batch, its grow-only buffers counted against the backend's
// device budget; on failure E keeps no layout.
int layout_engine(g16_backend* b, BatchEngine& E, g16_circuit* const* cs, size_t count) {
    const uint64_t need = plan_estimate(cs, count);
    if (need > E.accounted) {   // the engine's buffers grow: check and count the difference
        if (b->vram_used + (need - E.accounted) > b->vram_limit)
            return fail(G16_ERR_DEVICE_MEMORY, "batch of %zu proofs needs about %llu MiB of device memory", count,
                        (unsigned long long)(need >> 20));
        b->vram_used += need - E.accounted;
        E.accounted = need;
    }
    const uint64_t allocs0 = timer().device_alloc_bytes.load();
    int rc = build(E, cs, count);
    if (rc != G16_OK) {
        E.drop_layout();
        return rc;
    }
    b->batch_layouts++;
    b->batch_grown += timer().device_alloc_bytes.load() - allocs0;
    return G16_OK;
}

int reserve_batch_engines(g16_backend* b, g16_circuit* const* cs, size_t count) {
    if (!count) return G16_OK;
    const size_t max_engines = batch_max_engines();
    // one engine at a time, each as soon as it is idle, so that batches running
    // meanwhile keep the others; as in prove_batch_engine, the engine is taken
    // before the circuits' retuning guard (g16_autotune waits for batch users, a
    // batch holding an engine waits for tuning to end)
    std::vector<BatchEngine*> sized;
    for (;;) {
        BatchEngine* eng = nullptr;
        {
            std::unique_lock<std::mutex> lk(b->batch_mu);
            if (!b->batch) b->batch = new BatchPool();
            BatchPool& P = *b->batch;
            while (P.all.size() < max_engines) {
                P.all.push_back(std::make_unique<BatchEngine>());
                P.idle.push_back(P.all.back().get());
                b->batch_engines++;
            }
            if (sized.size() >= P.all.size()) break;
            auto fresh = [&] {
                for (size_t i = 0; i < P.idle.size(); i++)
                    if (std::find(sized.begin(), sized.end(), P.idle[i]) == sized.end()) return (long)i;
                return -1L;
            };
            P.cv.wait(lk, [&] { return fresh() >= 0; });
            const long i = fresh();
            eng = P.idle[(size_t)i];
            P.idle.erase(P.idle.begin() + i);
        }
        struct GiveBack {
            g16_backend* b;
            BatchEngine* e;
            ~GiveBack() {
                {
                    std::lock_guard<std::mutex> g(b->batch_mu);
                    b->batch->idle.push_back(e);
                }
                b->batch->cv.notify_all();
            }
        } give_back{b, eng};
        BatchUsers users(cs, count);
        int rc = layout_engine(b, *eng, cs, count);
        if (rc != G16_OK) return rc;
        eng->drop_layout();   // sized; the next batch lays itself out
        sized.push_back(eng);
    }
    return G16_OK;
}

int prove_batch_engine(g16_backend* b, size_t count, g16_circuit* const* cs, const uint8_t* const* witnesses,
                       const size_t* lens, const uint8_t* r, const uint8_t* s, g16_proof* out, double* done_ms) {
    const auto t_start = std::chrono::steady_clock::now();
    if (!count) return G16_OK;
    // the blinders first: nothing below may return before the device work it
    // enqueued has finished
    std::vector<Fr> rr(count), ss(count);
    for (size_t j = 0; j < count; j++) {
        uint64_t a[4], c[4];
        std::memcpy(a, r + 32 * j, 32);
        std::memcpy(c, s + 32 * j, 32);
        if (!Fr::canonical(a) || !Fr::canonical(c)) return fail(G16_ERR_INVALID_ARGUMENT, "job %zu: r or s not below r", j);
        rr[j] = Fr::raw(a);
        ss[j] = Fr::raw(c);
    }
    // an idle engine, preferably one whose layout (and graph) is this mix's
    std::vector<BatchKey> want;
    for (size_t j = 0; j < count; j++) want.push_back(key_of(cs[j]));
    BatchEngine* eng = nullptr;
    const size_t max_engines = batch_max_engines();
    {
        std::unique_lock<std::mutex> lk(b->batch_mu);
        if (!b->batch) b->batch = new BatchPool();
        BatchPool& P = *b->batch;
        P.cv.wait(lk, [&] { return !P.idle.empty() || P.all.size() < max_engines; });
        for (size_t i = 0; i < P.idle.size() && !eng; i++)
            if (P.idle[i]->key == want) {
                eng = P.idle[i];
                P.idle.erase(P.idle.begin() + (long)i);
            }
        if (!eng && !P.idle.empty()) {
            eng = P.idle.back();
            P.idle.pop_back();
        }
        if (!eng) {
            P.all.push_back(std::make_unique<BatchEngine>());
            eng = P.all.back().get();
            b->batch_engines++;
        }
    }
    struct GiveBack {
        g16_backend* b;
        BatchEngine* e;
        ~GiveBack() {
            {
                std::lock_guard<std::mutex> g(b->batch_mu);
                b->batch->idle.push_back(e);
            }
            b->batch->cv.notify_all();
        }
    } give_back{b, eng};
    BatchUsers users(cs, count);
    BatchEngine& E = *eng;
    if (!(E.key == want)) {
        int rc = layout_engine(b, E, cs, count);
        if (rc != G16_OK) return rc;
    }
    // witnesses in: gathered into pinned memory by host threads, then one copy
    const size_t threads = host_threads();
    parallel_for(count, threads, [&](size_t j) { std::memcpy(E.h_stage + E.off_w[j], witnesses[j], 32 * lens[j]); });
    CK_BATCH(cudaMemcpyAsync(E.d_arena, E.h_stage, E.w_bytes, cudaMemcpyHostToDevice, E.st[0]));
    // the key-only blinder products on the host while the device runs
    std::vector<BlinderTerms> terms(count);
    std::thread blinders([&] { parallel_for(count, threads, [&](size_t j) { terms[j] = blinder_terms(cs[j], rr[j], ss[j]); }); });
    int rc = G16_OK;
    const bool use_graph = !timer().enabled && E.runs > 0;
    if (use_graph && !E.graph) {
        uint64_t k0 = timer().launches.load();
        cudaError_t e = cudaStreamBeginCapture(E.st[0], cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = enqueue(E);
            cudaGraph_t g = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(E.st[0], &g);
            if (rc == G16_OK && e2 != cudaSuccess) rc = cuda_fail(e2, "batch graph capture");
            if (rc == G16_OK) {
                e2 = cudaGraphInstantiate(&E.graph, g, 0);
                if (e2 != cudaSuccess) rc = cuda_fail(e2, "batch graph instantiate");
            }
            if (g) cudaGraphDestroy(g);
            E.graph_kernels = timer().launches.load() - k0;
            timer().launches.fetch_sub(E.graph_kernels);   // counted when replayed
        } else {
            rc = cuda_fail(e, "batch graph capture");
        }
    }
    if (rc == G16_OK) {
        b->batch_submissions++;
        if (use_graph) {
            b->batch_replays++;
            cudaError_t e = cudaGraphLaunch(E.graph, E.st[0]);
            if (e != cudaSuccess) rc = cuda_fail(e, "batch graph launch");
            else timer().launches.fetch_add(E.graph_kernels);
        } else {
            rc = enqueue(E);
        }
    }
    if (rc == G16_OK) {
        cudaError_t e = cudaStreamSynchronize(E.st[0]);
        if (e != cudaSuccess) rc = cuda_fail(e, "batched proving");
    }
    blinders.join();
    if (rc != G16_OK) {
        // a partly enqueued submission may still run on any of the three
        // streams: let it finish before the engine is handed out again, and
        // forget the layout (its graph may be half-built)
        for (cudaStream_t st : E.st)
            if (st) cudaStreamSynchronize(st);
        E.drop_layout();
        return rc;
    }
    timer().collect();
    E.runs++;
    // stage 11 for every job
    const uint8_t *rg1 = E.h_res, *rg2 = E.h_res + E.res_g1, *rh = E.h_res + E.res_g1 + E.res_g2;
    parallel_for(count, threads, [&](size_t j) {
        MsmJac m;
        m.a = msm_space_combine_g1(rg1, E.g1, 3 * j);
        m.b1 = msm_space_combine_g1(rg1, E.g1, 3 * j + 1);
        m.l = msm_space_combine_g1(rg1, E.g1, 3 * j + 2);
        m.b2 = msm_space_combine_g2(rg2, E.g2, j);
        m.h = msm_space_combine_g1(rh, E.hs, j);
        assemble(cs[j], m, terms[j], rr[j], ss[j], out + j);
        if (done_ms)
            done_ms[j] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    });
    return G16_OK;
}

}  // namespace g16
