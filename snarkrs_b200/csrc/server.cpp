// Served proving: a request loop with continuous batching.
//
// Requests (a registered key id, a witness, r and s) enter a FIFO queue.
// `lanes` worker threads each take the next request as soon as they are free,
// so requests that arrive while others are on the GPU are admitted as lanes
// free up and their kernels overlap on the device (each proof runs on its own
// workspace: five streams, its own scratch).  Admission by device memory has
// two levels:
//   * proving keys are prepared on first use and stay resident in HBM while
//     the sum of resident keys' device bytes fits the key budget; a key that
//     does not fit evicts the least recently used idle keys first;
//   * a proof starts only when its circuit can hand out a workspace, which
//     waits while the backend's device-memory budget has no room for one.
// The result of every request is the same as proving it alone.
//
// Built on the public C ABI only (include/g16b200.h).
#include <chrono>
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
    std::vector<std::thread> workers;
    bool stop = false;
};

namespace {

uint64_t live_bytes(g16_server* sv) {
    uint64_t t = 0;
    for (auto& kv : sv->keys)
        if (kv.second.circ) t += g16_circuit_device_bytes(kv.second.circ);
    return t;
}

// Make `id` resident.  Called with the lock held; drops it while preparing.
int ensure_resident(g16_server* sv, uint32_t id, std::unique_lock<std::mutex>& lk, std::string& err) {
    KeyEntry& k = sv->keys[id];
    for (;;) {
        if (k.circ) return G16_OK;
        if (!k.preparing) break;
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

void worker(g16_server* sv) {
    std::unique_lock<std::mutex> lk(sv->mu);
    for (;;) {
        sv->cv_work.wait(lk, [&] { return sv->stop || !sv->queue.empty(); });
        if (sv->stop && sv->queue.empty()) return;
        Request* q = sv->queue.front();
        sv->queue.pop_front();
        std::string err;
        int rc = ensure_resident(sv, q->key_id, lk, err);
        KeyEntry& k = sv->keys[q->key_id];
        if (rc == G16_OK) {
            k.in_use++;
            k.last_use = ++sv->clock;
            g16_circuit* c = k.circ;
            lk.unlock();
            q->started = Clock::now();
            rc = g16_prove_with_blinders(c, q->witness.data(), q->witness.size() / 32, q->r, q->s, &q->proof);
            if (rc != G16_OK) {
                char buf[512];
                g16_last_error(buf, sizeof buf);
                err = buf;
            }
            q->finished = Clock::now();
            lk.lock();
            k.in_use--;
            sv->cv_keys.notify_all();
        } else {
            q->started = q->finished = Clock::now();
        }
        q->rc = rc;
        q->err = err;
        q->done = true;
        std::vector<uint8_t>().swap(q->witness);
        sv->completed++;
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
    for (int i = 0; i < lanes; i++) sv->workers.emplace_back(worker, sv.get());
    *out = sv.release();
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
