// Served proving: a request loop with continuous batching.
//
// Requests (a registered key id, a witness, r and s) enter a FIFO queue.
// `lanes` worker threads each take, as soon as they are free, every request
// queued at that moment (in arrival order, up to a work cap) and prove them
// together in one batched submission (g16_prove_batch: each stage of all of
// them in one launch, any mix of circuits and sizes).  Requests that arrive
// while a batch is on the GPU wait for the next free worker, which takes them
// all, and the workers' batches overlap on the device (each on its own
// engine: streams and scratch).  Admission by device memory has two levels:
//   * proving keys are prepared on first use and stay resident in HBM while
//     the sum of resident keys' device bytes fits the key budget; a key that
//     does not fit evicts the least recently used idle keys first;
//   * a batch starts only when its working set fits the backend's
//     device-memory budget (otherwise its proofs run one by one on workspaces,
//     each waiting for room).
// The result of every request is the same as proving it alone.
//
// Built on the public C ABI only (include/g16b200.h).
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>
#include "common.cuh"
#include "g16b200.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t ticket = 0;
    uint32_t key_id = 0;
    std::vector<uint8_t> witness;
    uint8_t r[32], s[32];
    Clock::time_point submitted, started, finished;
    bool done = false;
    int rc = G16_OK;
    std::string err;
    g16_proof proof;
};

struct KeyEntry {
    std::vector<uint8_t> zkey;      // host copy of the .zkey bytes
    g16_circuit* circ = nullptr;    // resident when non-null
    bool preparing = false;
    int in_use = 0;
    uint64_t last_use = 0;
    uint64_t bytes = 0;             // device bytes when last resident
};

}  // namespace

struct g16_server {
    g16_backend* b = nullptr;
    uint64_t budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_keys;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
    std::unordered_map<uint32_t, KeyEntry> keys;
    uint64_t next_ticket = 1, clock = 0, resident_bytes = 0;
    uint64_t submitted = 0, completed = 0, prepared = 0, evicted = 0;
    uint64_t batches = 0, batched = 0, alone = 0;
    std::vector<std::thread> workers;
    bool stop = false;
    size_t max_batch = 64;          // requests per batch
    uint64_t batch_wires = 1u << 21;   // work cap of a batch: witness wires summed
    uint64_t solo_wires = 1u << 19;    // requests of at least this many wires are proved alone (0: none)
};

namespace {

uint64_t live_bytes(g16_server* sv) {
    uint64_t t = 0;
    for (auto& kv : sv->keys)
        if (kv.second.circ) t += g16_circuit_device_bytes(kv.second.circ);
    return t;
}

// The batch engines, sized for a quarter more than the largest batch of this
// key alone that the caps allow (at most max_batch requests and batch_wires
// wires).  Under load the queue grows and so do the batches: an engine that
// first met them then would reallocate its buffers while other requests run,
// which slows the server when it is already behind.  A mix of keys can need
// more than each key's own largest batch (its bucket arrays sum over the jobs,
// about a fifth more for the served mix of 2^14-2^18 constraints), hence the
// quarter.  Best effort: a mix that needs more still grows.
void reserve_engines_for(g16_server* sv, g16_circuit* c, size_t max_batch, uint64_t batch_wires, uint64_t solo_wires) {
    const uint64_t wires = g16_circuit_n_vars(c);
    if (!wires || (solo_wires && wires >= solo_wires)) return;   // proved alone
    const size_t largest = (size_t)std::min<uint64_t>(max_batch, std::max<uint64_t>(1, batch_wires / wires));
    if (largest < 2) return;   // a batch of one is proved alone
    const size_t copies = largest + (largest + 3) / 4;
    std::vector<g16_circuit*> cs(copies, c);
    g16_batch_reserve(sv->b, copies, cs.data());
}

// ensure_resident could only go on by waiting, which a worker already holding
// keys must not do: the request goes back to the queue for a later batch
constexpr int DEFER = -1;

// Make `id` resident.  Called with the lock held; drops it while preparing.
// may_wait: the caller holds no key, so it may wait for other workers' keys
// to go idle (a worker that holds keys and waited could wait on a worker that
// waits on it).
int ensure_resident(g16_server* sv, uint32_t id, std::unique_lock<std::mutex>& lk, std::string& err,
                    bool may_wait) {
    KeyEntry& k = sv->keys[id];
    for (;;) {
        if (k.circ) return G16_OK;
        if (!k.preparing) break;
        if (!may_wait) return DEFER;
        sv->cv_keys.wait(lk);
    }
    k.preparing = true;
    // evict least recently used idle keys until the estimate fits the budget
    uint64_t want = k.bytes ? k.bytes : (uint64_t)k.zkey.size() * 12;
    for (;;) {
        uint64_t live = live_bytes(sv);
        if (live + want <= sv->budget) break;
        KeyEntry* victim = nullptr;
        for (auto& kv : sv->keys) {
            KeyEntry& e = kv.second;
            if (e.circ && e.in_use == 0 && (!victim || e.last_use < victim->last_use)) victim = &e;
        }
        if (!victim) {
            bool any_busy = false;
            for (auto& kv : sv->keys) any_busy |= kv.second.circ && kv.second.in_use > 0;
            if (!any_busy) break;   // nothing to evict and nothing will free: try anyway
            if (!may_wait) {
                k.preparing = false;
                sv->cv_keys.notify_all();
                return DEFER;
            }
            sv->cv_keys.wait(lk);   // wait for a key to go idle
            continue;
        }
        victim->bytes = g16_circuit_device_bytes(victim->circ);
        g16_circuit* c = victim->circ;
        victim->circ = nullptr;
        sv->evicted++;
        lk.unlock();
        g16_circuit_free(c);
        lk.lock();
    }
    std::vector<uint8_t> bytes = k.zkey;   // stable copy while unlocked
    const size_t max_batch = sv->max_batch;
    const uint64_t batch_wires = sv->batch_wires, solo_wires = sv->solo_wires;
    const uint32_t lanes = (uint32_t)sv->workers.size();
    lk.unlock();
    g16_zkey* z = nullptr;
    g16_circuit* c = nullptr;
    int rc = g16_zkey_parse(bytes.data(), bytes.size(), 0, &z);
    if (rc == G16_OK) {
        g16_zkey_view v;
        g16_zkey_view_get(z, &v);
        rc = g16_prepare(sv->b, &v, &c);
        g16_zkey_free(z);
    }
    if (rc == G16_OK) {
        // as many ready workspaces as workers that may prove this key alone at once,
        // and engines sized for its batches: first requests then allocate nothing
        // and replay graphs (best effort)
        g16_circuit_warm(c, lanes);
        reserve_engines_for(sv, c, max_batch, batch_wires, solo_wires);
    }
    if (rc != G16_OK) {
        char buf[512];
        g16_last_error(buf, sizeof buf);
        err = buf;
    }
    lk.lock();
    k.preparing = false;
    if (rc == G16_OK) {
        k.circ = c;
        k.bytes = g16_circuit_device_bytes(c);
        sv->prepared++;
    }
    sv->cv_keys.notify_all();
    return rc;
}

std::string last_error_text() {
    char buf[512];
    g16_last_error(buf, sizeof buf);
    return buf;
}

// Called with the lock held: the request is finished.
void complete(g16_server* sv, Request* q, int rc, const std::string& err) {
    q->rc = rc;
    q->err = err;
    q->done = true;
    std::vector<uint8_t>().swap(q->witness);
    sv->completed++;
}

// Work of a request for the batch cap: its witness length (wires).
uint64_t work_of(const Request* q) { return q->witness.size() / 32; }

// A large request is proved alone: its stages fill the device by themselves,
// and in a batch the small requests beside it would wait for its MSMs (a
// batch's proofs complete together).
bool solo(const g16_server* sv, const Request* q) { return sv->solo_wires && work_of(q) >= sv->solo_wires; }

void worker(g16_server* sv) {
    std::unique_lock<std::mutex> lk(sv->mu);
    for (;;) {
        sv->cv_work.wait(lk, [&] { return sv->stop || !sv->queue.empty(); });
        if (sv->stop && sv->queue.empty()) return;
        // a large request at the head goes alone; otherwise the queued small
        // requests, in arrival order, while the batch's work stays under the
        // cap (the first one always goes), leaving large ones for other workers
        std::vector<Request*> batch;
        uint64_t work = 0;
        if (solo(sv, sv->queue.front())) {
            batch.push_back(sv->queue.front());
            sv->queue.pop_front();
        } else {
            for (auto it = sv->queue.begin(); it != sv->queue.end() && batch.size() < sv->max_batch;) {
                Request* q = *it;
                if (solo(sv, q)) {
                    ++it;
                    continue;
                }
                if (!batch.empty() && work + work_of(q) > sv->batch_wires) break;
                work += work_of(q);
                batch.push_back(q);
                it = sv->queue.erase(it);
            }
        }
        if (!sv->queue.empty()) sv->cv_work.notify_one();   // the rest is another worker's
        // keys resident and pinned for the batch; requests refused up front end here
        std::vector<Request*> run, deferred;
        std::vector<g16_circuit*> circs;
        for (Request* q : batch) {
            std::string err;
            int rc = ensure_resident(sv, q->key_id, lk, err, run.empty());
            if (rc == DEFER) {
                deferred.push_back(q);
                continue;
            }
            KeyEntry& k = sv->keys[q->key_id];
            if (rc == G16_OK && q->witness.size() / 32 != g16_circuit_n_vars(k.circ)) {
                rc = G16_ERR_WITNESS_LENGTH;
                err = "witness has " + std::to_string(q->witness.size() / 32) + " values, the circuit has " +
                      std::to_string(g16_circuit_n_vars(k.circ)) + " wires";
            }
            if (rc != G16_OK) {
                q->started = q->finished = Clock::now();
                complete(sv, q, rc, err);
                continue;
            }
            k.in_use++;
            k.last_use = ++sv->clock;
            run.push_back(q);
            circs.push_back(k.circ);
        }
        // requests whose keys could not be made resident beside this batch's go
        // back to the head of the queue, in order
        for (size_t i = deferred.size(); i-- > 0;) sv->queue.push_front(deferred[i]);
        if (!deferred.empty()) sv->cv_work.notify_one();
        if (!run.empty()) {
            lk.unlock();
            const size_t n = run.size();
            std::vector<const uint8_t*> wits(n);
            std::vector<size_t> lens(n);
            std::vector<uint8_t> rs(32 * n), ss(32 * n);
            std::vector<g16_proof> proofs(n);
            std::vector<double> done(n, 0.0);
            for (size_t i = 0; i < n; i++) {
                wits[i] = run[i]->witness.data();
                lens[i] = run[i]->witness.size() / 32;
                std::memcpy(&rs[32 * i], run[i]->r, 32);
                std::memcpy(&ss[32 * i], run[i]->s, 32);
            }
            const Clock::time_point t0 = Clock::now();
            for (Request* q : run) q->started = t0;
            // one request is plain proving on a workspace of its circuit (max_batch
            // 1 is one-proof-at-a-time serving); more go as one batched submission
            int rc = n == 1 ? g16_prove_with_blinders(circs[0], wits[0], lens[0], run[0]->r, run[0]->s, &proofs[0])
                            : g16_prove_batch_timed(sv->b, n, circs.data(), wits.data(), lens.data(), rs.data(),
                                                    ss.data(), proofs.data(), done.data());
            if (n == 1 && rc == G16_OK) done[0] = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
            std::vector<int> rcs(n, rc);
            std::vector<std::string> errs(n, rc == G16_OK ? std::string() : last_error_text());
            if (rc != G16_OK) {
                // the batch failed as a whole: each request alone gets its own status
                for (size_t i = 0; i < n; i++) {
                    rcs[i] = g16_prove_with_blinders(circs[i], wits[i], lens[i], run[i]->r, run[i]->s, &proofs[i]);
                    errs[i] = rcs[i] == G16_OK ? std::string() : last_error_text();
                    done[i] = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
                }
            }
            lk.lock();
            if (n == 1) {
                sv->alone++;
            } else {
                sv->batches++;
                sv->batched += n;
            }
            for (size_t i = 0; i < n; i++) {
                Request* q = run[i];
                q->finished = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double, std::milli>(done[i]));
                q->proof = proofs[i];
                sv->keys[q->key_id].in_use--;
                complete(sv, q, rcs[i], errs[i]);
            }
            sv->cv_keys.notify_all();
        }
        sv->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

int g16_server_new(g16_backend* b, uint64_t key_budget_bytes, int lanes, g16_server** out) {
    if (!b || !out || lanes < 1 || lanes > 64) {
        g16::set_error("g16_server_new: need a backend and 1..64 lanes");
        return G16_ERR_INVALID_ARGUMENT;
    }
    auto sv = std::make_unique<g16_server>();
    sv->b = b;
    sv->budget = key_budget_bytes ? key_budget_bytes : ~0ull;
    if (const char* e = std::getenv("G16_SERVE_BATCH")) sv->max_batch = (size_t)std::max(1, std::atoi(e));
    if (const char* e = std::getenv("G16_SERVE_BATCH_WIRES")) sv->batch_wires = std::max<uint64_t>(1, std::strtoull(e, nullptr, 10));
    if (const char* e = std::getenv("G16_SERVE_SOLO_WIRES")) sv->solo_wires = std::strtoull(e, nullptr, 10);
    for (int i = 0; i < lanes; i++) sv->workers.emplace_back(worker, sv.get());
    *out = sv.release();
    return G16_OK;
}

int g16_server_set_max_batch(g16_server* sv, size_t max_batch) {
    if (!sv || max_batch < 1) {
        g16::set_error("g16_server_set_max_batch: need a server and at least 1");
        return G16_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> g(sv->mu);
    sv->max_batch = max_batch;
    return G16_OK;
}

int g16_server_register_key(g16_server* sv, uint32_t key_id, const uint8_t* zkey, size_t len) {
    if (!sv || !zkey || !len) {
        g16::set_error("g16_server_register_key: null argument");
        return G16_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> g(sv->mu);
    KeyEntry& k = sv->keys[key_id];
    if (k.circ || k.preparing || k.in_use) {
        g16::set_error("g16_server_register_key: key %u is already registered and in use", key_id);
        return G16_ERR_INVALID_ARGUMENT;
    }
    k.zkey.assign(zkey, zkey + len);
    k.bytes = 0;
    return G16_OK;
}

int g16_server_submit(g16_server* sv, uint32_t key_id, const uint8_t* w_mont, size_t n, const uint8_t* r_mont,
                      const uint8_t* s_mont, uint64_t* ticket) {
    if (!sv || !w_mont || !r_mont || !s_mont || !ticket) {
        g16::set_error("g16_server_submit: null argument");
        return G16_ERR_INVALID_ARGUMENT;
    }
    auto q = std::make_unique<Request>();
    q->key_id = key_id;
    q->witness.assign(w_mont, w_mont + 32 * n);
    std::memcpy(q->r, r_mont, 32);
    std::memcpy(q->s, s_mont, 32);
    std::lock_guard<std::mutex> g(sv->mu);
    if (!sv->keys.count(key_id)) {
        g16::set_error("g16_server_submit: key %u is not registered", key_id);
        return G16_ERR_INVALID_ARGUMENT;
    }
    q->ticket = sv->next_ticket++;
    q->submitted = Clock::now();
    *ticket = q->ticket;
    sv->queue.push_back(q.get());
    sv->requests[q->ticket] = std::move(q);
    sv->submitted++;
    sv->cv_work.notify_one();
    return G16_OK;
}

int g16_server_wait(g16_server* sv, uint64_t ticket, g16_proof* out, double* queue_ms, double* latency_ms) {
    if (!sv || !out) {
        g16::set_error("g16_server_wait: null argument");
        return G16_ERR_INVALID_ARGUMENT;
    }
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->requests.find(ticket);
    if (it == sv->requests.end()) {
        g16::set_error("g16_server_wait: unknown ticket %llu", (unsigned long long)ticket);
        return G16_ERR_INVALID_ARGUMENT;
    }
    Request* q = it->second.get();
    sv->cv_done.wait(lk, [&] { return q->done; });
    using ms = std::chrono::duration<double, std::milli>;
    if (queue_ms) *queue_ms = ms(q->started - q->submitted).count();
    if (latency_ms) *latency_ms = ms(q->finished - q->submitted).count();
    int rc = q->rc;
    if (rc == G16_OK) *out = q->proof;
    else g16::set_error("%s", q->err.c_str());
    sv->requests.erase(it);
    return rc;
}

int g16_server_stats_get(g16_server* sv, g16_server_stats* out) {
    if (!sv || !out) {
        g16::set_error("g16_server_stats_get: null argument");
        return G16_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> g(sv->mu);
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->prepared = sv->prepared;
    out->evicted = sv->evicted;
    out->resident_keys = 0;
    for (auto& kv : sv->keys) out->resident_keys += kv.second.circ ? 1 : 0;
    out->resident_bytes = live_bytes(sv);
    out->queued = sv->queue.size();
    out->batches = sv->batches;
    out->batched = sv->batched;
    out->alone = sv->alone;
    return G16_OK;
}

void g16_server_free(g16_server* sv) {
    if (!sv) return;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    for (auto& t : sv->workers) t.join();
    for (auto& kv : sv->keys)
        if (kv.second.circ) g16_circuit_free(kv.second.circ);
    delete sv;
}

}  // extern "C"
