// Groth16 prover orchestration and the extern "C" boundary (include/g16b200.h).
//
// Mirrors the reference's CUDA backend split (crates/cuda/src/backend.rs:
// CudaBackend / CudaCircuit; stages.rs: stages 0-4; msm.rs: stages 5-9) and
// the PreparedCircuit contract (crates/groth16/src/lib.rs:371-455):
//   prepare      upload CSR, bases and domain tables once (backend.rs:325-457)
//   stage 0      gather A.w and B.w over the CSR rows, C = A*B (cpu.rs:140-174, 316-341)
//   stages 1-4   iNTT -> coset -> NTT for A, B, C, H = A*B - C (cpu.rs:191-252)
//   stages 5-9   five MSMs: A, B1, L in G1 and B2 in G2 from one sort of the
//                witness, H in G1 (cpu.rs:477-632)
//   stage 11     blinding and assembly on the host (prove.rs:335-430), the
//                four key-only products computed on a side thread while the
//                device runs, as blinded_with does (prove.rs:201-229).
#include <atomic>
#include <cstdarg>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <future>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "common.cuh"
#include "curve.cuh"
#include "field.cuh"
#include "formats.hpp"
#include "gather.cuh"
#include "g16b200.h"
#include "host_bn254.hpp"
#include "msm.cuh"
#include "ntt.cuh"
#include "pairing.hpp"
#include <sys/random.h>

namespace g16 {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

KernelTimer& timer() {
    static KernelTimer t;
    return t;
}

}  // namespace g16

using namespace g16;

// ---------------------------------------------------------------- kernels
namespace g16d {

// Stage 0: one thread per constraint row (gather.cuh).
__global__ void __launch_bounds__(256) k_gather(const uint32_t* __restrict__ rpa, const uint32_t* __restrict__ siga,
                                                const uint32_t* __restrict__ vida, const uint32_t* __restrict__ rpb,
                                                const uint32_t* __restrict__ sigb, const uint32_t* __restrict__ vidb,
                                                const uint4* __restrict__ values, const uint4* __restrict__ w,
                                                uint32_t n, uint4* __restrict__ A, uint4* __restrict__ B,
                                                uint4* __restrict__ C) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    gather_row(row, rpa, siga, vida, rpb, sigb, vidb, values, w, A, B, C);
}

// Stage 0 handed over (h_and_msms_from_rows): C = A * B on the caller's rows,
// zero past them (crates/groth16/src/cpu.rs:409-425).
__global__ void k_rows_c(const uint4* __restrict__ A, const uint4* __restrict__ B, uint4* __restrict__ C,
                         uint32_t n) {
    uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    store32(reinterpret_cast<Fr*>(C) + row,
            mul(load32(reinterpret_cast<const Fr*>(A) + row), load32(reinterpret_cast<const Fr*>(B) + row)));
}

// Throughput probe for the 32-bit multiply-add the field code is built from:
// eight independent chains alternating mad.lo.u32 and mad.hi.u32, so the
// issue rate, not latency, bounds it.  Gives the integer roofline's peak.
__global__ void __launch_bounds__(256) k_imad_peak(uint32_t* out, uint32_t iters, uint32_t seed) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t x0 = t ^ seed, x1 = t + 1, x2 = t + 2, x3 = t + 3, x4 = t + 4, x5 = t + 5, x6 = t + 6, x7 = t + 7;
    uint32_t b = 0x9e3779b9u ^ t, c = 0x7f4a7c15u + seed;
    for (uint32_t i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 4; u++) {
            asm volatile(
                "mad.lo.u32 %0, %0, %8, %9;\n\t"
                "mad.lo.u32 %1, %1, %8, %9;\n\t"
                "mad.lo.u32 %2, %2, %8, %9;\n\t"
                "mad.lo.u32 %3, %3, %8, %9;\n\t"
                "mad.lo.u32 %4, %4, %8, %9;\n\t"
                "mad.lo.u32 %5, %5, %8, %9;\n\t"
                "mad.lo.u32 %6, %6, %8, %9;\n\t"
                "mad.lo.u32 %7, %7, %8, %9;\n\t"
                "mad.hi.u32 %0, %0, %8, %9;\n\t"
                "mad.hi.u32 %1, %1, %8, %9;\n\t"
                "mad.hi.u32 %2, %2, %8, %9;\n\t"
                "mad.hi.u32 %3, %3, %8, %9;\n\t"
                "mad.hi.u32 %4, %4, %8, %9;\n\t"
                "mad.hi.u32 %5, %5, %8, %9;\n\t"
                "mad.hi.u32 %6, %6, %8, %9;\n\t"
                "mad.hi.u32 %7, %7, %8, %9;"
                : "+r"(x0), "+r"(x1), "+r"(x2), "+r"(x3), "+r"(x4), "+r"(x5), "+r"(x6), "+r"(x7)
                : "r"(b), "r"(c));
        }
    }
    out[t] = x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
}

}  // namespace g16d

#include "prover.hpp"

struct g16_hpoly {
    g16_circuit* owner = nullptr;
    void* d_h = nullptr;
    uint32_t n = 0;
};

struct g16_zkey {
    ZkeyHost k;
};

namespace g16 {

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    set_error("%s", buf);
    return code;
}

// Device-fault classes of a CUDA runtime status (the reference's
// is_device_fault and is_sticky, crates/cuda/src/context.rs:134-215, there over
// the driver's CUresult; the runtime documents its cudaError_t twins in the
// same words).
int error_class(int code) {
    switch (code) {
    // kernel exceptions, the watchdog and a contained hardware error: "the
    // process is left in an inconsistent state and any further CUDA work will
    // return the same error"
    case cudaErrorIllegalAddress:
    case cudaErrorAssert:
    case cudaErrorHardwareStackError:
    case cudaErrorIllegalInstruction:
    case cudaErrorMisalignedAddress:
    case cudaErrorInvalidAddressSpace:
    case cudaErrorInvalidPc:
    case cudaErrorLaunchFailure:
    case cudaErrorLaunchTimeout:
    case cudaErrorContained:
        return G16_FAULT_DEVICE | G16_FAULT_STICKY;
    // the device or its daemons failed, the context stays usable
    case cudaErrorMemoryAllocation:
    case cudaErrorDevicesUnavailable:
    case cudaErrorECCUncorrectable:
    case cudaErrorNvlinkUncorrectable:
    case cudaErrorSystemNotReady:
    case cudaErrorMpsConnectionFailed:
    case cudaErrorMpsRpcFailure:
    case cudaErrorMpsServerNotReady:
    case cudaErrorMpsMaxClientsReached:
    case cudaErrorMpsMaxConnectionsReached:
    case cudaErrorMpsClientTerminated:
    case cudaErrorTimeout:
    case cudaErrorExternalDevice:
    case cudaErrorUnknown:
        return G16_FAULT_DEVICE;
    default:
        return 0;
    }
}

// The sticky status that took each device out of use in this process, or 0.
static std::atomic<int> g_device_fault[64];

static const char* const STICKY_TEXT =
    "; a sticky fault: the CUDA context is unusable for the rest of this process, and every later call on this "
    "device is refused; prove on another device or in a new process";

// The status for a failed CUDA call (or an injected one): DEVICE_MEMORY for
// out of memory, else DEVICE; a sticky code also marks the device (when
// mark_device) for the rest of the process.
static int fault_status(int e, const char* what, bool mark_device) {
    const bool sticky = (error_class(e) & G16_FAULT_STICKY) != 0;
    if (sticky && mark_device) {
        int dev = -1;
        if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64) {
            int none = 0;
            g_device_fault[dev].compare_exchange_strong(none, e);
        }
    }
    const char* text = cudaGetErrorString((cudaError_t)e);
    if (e == cudaErrorMemoryAllocation) return fail(G16_ERR_DEVICE_MEMORY, "%s: %s", what, text);
    std::string prev = [] {
        char b[512];
        g16_last_error(b, sizeof b);
        return std::string(b);
    }();
    if (prev.empty()) return fail(G16_ERR_DEVICE, "%s: %s%s", what, text, sticky ? STICKY_TEXT : "");
    return fail(G16_ERR_DEVICE, "%s: %s%s (%s)", what, text, sticky ? STICKY_TEXT : "", prev.c_str());
}

int cuda_fail(cudaError_t e, const char* what) { return fault_status((int)e, what, true); }

int device_fault(int ordinal) { return ordinal >= 0 && ordinal < 64 ? g_device_fault[ordinal].load() : 0; }

// Called first by every entry point that uses b's device: refuses when a
// sticky fault took the device (or this backend) out of use, and delivers a
// pending injected fault.
int device_usable(g16_backend* b) {
    int code = b->fault.load();
    if (!code) code = device_fault(b->ordinal);
    if (code)
        return fail(G16_ERR_DEVICE, "CUDA device %d is out of use after %s%s", b->ordinal,
                    cudaGetErrorString((cudaError_t)code), STICKY_TEXT);
    const int inj = b->inject.exchange(0);
    if (inj) {
        if (error_class(inj) & G16_FAULT_STICKY) {
            int none = 0;
            b->fault.compare_exchange_strong(none, inj);
        }
        set_error("%s", "");
        return fault_status(inj, "injected fault", false);
    }
    return G16_OK;
}

}  // namespace g16

namespace {

#define CK(call, what)                                  \
    do {                                                \
        cudaError_t e__ = (call);                       \
        if (e__ != cudaSuccess) return cuda_fail(e__, what); \
    } while (0)

cudaError_t circuit_alloc(g16_circuit* c, void** p, size_t bytes) {
    cudaError_t e = g16::dev_malloc(p, bytes ? bytes : 32);
    if (e == cudaSuccess) {
        c->allocs.push_back(*p);
        c->device_bytes += bytes;
        c->be->vram_used += bytes;
    }
    return e;
}

// Device bytes of one workspace: witness, A|B|C, H, and the MSM scratch
// (sorted entries, partial sums, bucket sums) at window bits c_w and c_h, for
// live sets of ra (A), rb (B1, B2) and rl (L) wires; tables: one bucket set
// per MSM (window tables), else one per window (compact key).
uint64_t workspace_estimate(uint64_t nv, uint64_t n, int c_w, int c_h, uint64_t ra, uint64_t rb, uint64_t rl,
                            bool tables) {
    const uint64_t Ww = (uint64_t)msm_windows(c_w), Wh = (uint64_t)msm_windows(c_h);
    const uint64_t Kw = (1ull << (c_w - 1)) * (tables ? 1 : Ww), Kh = (1ull << (c_h - 1)) * (tables ? 1 : Wh);
    uint64_t b = nv * 32 + n * 32 * 4;
    b += nv * 32 + (ra + rb + rl) * Ww * 4 + 3 * 24 * (Kw + 1) + n * 32 + n * Wh * 4 + 24 * (Kh + 1);
    b += 128 * (3 * Kw * 2 + (ra + rb + rl) * Ww / 16 + 3) + 256 * (Kw * 2 + rb * Ww / 16 + 1);
    b += 128 * (Kh * 2 + n * Wh / 16 + 1) + (16ull << 20);
    return b;
}

void circuit_free_alloc(g16_circuit* c, void* p, uint64_t bytes) {
    if (!p) return;
    for (size_t i = 0; i < c->allocs.size(); i++)
        if (c->allocs[i] == p) {
            c->allocs.erase(c->allocs.begin() + (long)i);
            break;
        }
    cudaFree(p);
    c->device_bytes -= std::min<uint64_t>(c->device_bytes, bytes);
    c->be->vram_used -= std::min<uint64_t>(c->be->vram_used, bytes);
}

// (Re)build the window-shifted tables of the witness MSMs (A, B1, L, B2) for
// window bits cw, each over its live set's compacted bases; the new tables
// replace the old ones only when all are built.
int build_witness_tables(g16_circuit* c, int cw, cudaStream_t st) {
    if (!c->tables) {   // a compact key: the MSMs read the plain bases at any window width
        c->c_w = cw;
        return G16_OK;
    }
    const uint64_t W = (uint64_t)msm_windows(cw);
    const uint64_t ra = c->rows[0], rb = c->rows[1], rl = c->rows[2];
    if (std::max(ra, std::max(rb, rl)) * W >= 0x80000000ull)
        return fail(G16_ERR_BACKEND, "circuit too large for 31-bit MSM entry indices");
    void *ta = nullptr, *tb1 = nullptr, *tl = nullptr, *tb2 = nullptr;
    cudaError_t e = circuit_alloc(c, &ta, 64 * ra * W);
    if (e == cudaSuccess) e = circuit_alloc(c, &tb1, 64 * rb * W);
    if (e == cudaSuccess) e = circuit_alloc(c, &tl, 64 * rl * W);
    if (e == cudaSuccess) e = circuit_alloc(c, &tb2, 128 * rb * W);
    if (e == cudaSuccess && ra) e = msm_window_table_g1(c->d_a, ra, 0, cw, ta, st);
    if (e == cudaSuccess && rb) e = msm_window_table_g1(c->d_b1, rb, 0, cw, tb1, st);
    if (e == cudaSuccess && rl) e = msm_window_table_g1(c->d_l, rl, 0, cw, tl, st);
    if (e == cudaSuccess && rb) e = msm_window_table_g2(c->d_b2, rb, 0, cw, tb2, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "window tables");
        circuit_free_alloc(c, ta, 64 * ra * W);
        circuit_free_alloc(c, tb1, 64 * rb * W);
        circuit_free_alloc(c, tl, 64 * rl * W);
        circuit_free_alloc(c, tb2, 128 * rb * W);
        return rc;
    }
    if (c->c_w) {
        const uint64_t Wo = (uint64_t)msm_windows(c->c_w);
        circuit_free_alloc(c, c->t_a, 64 * ra * Wo);
        circuit_free_alloc(c, c->t_b1, 64 * rb * Wo);
        circuit_free_alloc(c, c->t_l, 64 * rl * Wo);
        circuit_free_alloc(c, c->t_b2, 128 * rb * Wo);
    }
    c->t_a = ta;
    c->t_b1 = tb1;
    c->t_l = tl;
    c->t_b2 = tb2;
    c->c_w = cw;
    return G16_OK;
}

// The same for the H MSM's table at window bits ch.
int build_h_table(g16_circuit* c, int ch, cudaStream_t st) {
    if (!c->tables) {
        c->c_h = ch;
        return G16_OK;
    }
    const uint64_t n = c->h_count, W = (uint64_t)msm_windows(ch);
    if (n * W >= 0x80000000ull) return fail(G16_ERR_BACKEND, "domain too large for 31-bit MSM entry indices");
    void* th = nullptr;
    cudaError_t e = circuit_alloc(c, &th, 64 * n * W);
    if (e == cudaSuccess) e = msm_window_table_g1(c->d_h, n, 0, ch, th, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "window tables");
        circuit_free_alloc(c, th, 64 * n * W);
        return rc;
    }
    if (c->c_h) circuit_free_alloc(c, c->t_h, 64 * n * (uint64_t)msm_windows(c->c_h));
    c->t_h = th;
    c->c_h = ch;
    return G16_OK;
}

// Host readback slot of one MSM's reduction terms (sizes checked against every
// window width by tests/test_reduce_plan.py).
constexpr size_t WIN_SLOT_COMPACT = MSM_RESULT_SLOT_COMPACT_BYTES;
// Bucket-reduction piece target of the witness MSMs (0: the library default for
// MSMs whose reductions run beside other work); G16_WITNESS_REDUCE_PIECES overrides it.
uint64_t witness_reduce_pieces() {
    static const uint64_t v = [] {
        const char* e = std::getenv("G16_WITNESS_REDUCE_PIECES");
        return e ? std::strtoull(e, nullptr, 10) : 0ull;
    }();
    return v;
}

size_t win_slot(const g16_circuit* c) { return c->tables ? MSM_RESULT_SLOT_BYTES : WIN_SLOT_COMPACT; }

// Take an idle workspace, or build one while the pool is below its cap and the
// backend's device-memory budget has room; otherwise wait for one to come back.
int acquire(g16_circuit* c, Workspace** out) {
    std::unique_lock<std::mutex> lk(c->mu);
    for (;;) {
        if (c->tuning) {
            c->cv.wait(lk);
            continue;
        }
        if (!c->idle.empty()) {
            *out = c->idle.back();
            c->idle.pop_back();
            return G16_OK;
        }
        bool room = c->be->vram_used + c->ws_estimate <= c->be->vram_limit;
        if (c->pool.size() < c->max_workspaces && (room || c->pool.empty())) {
            auto ws = std::make_unique<Workspace>();
            cudaError_t e = ws->init(c->n_vars, c->n, win_slot(c));
            if (e == cudaSuccess) {
                c->device_bytes += c->ws_estimate;
                c->be->vram_used += c->ws_estimate;
                *out = ws.get();
                c->pool.push_back(std::move(ws));
                return G16_OK;
            }
            ws->release();
            cudaGetLastError();
            if (c->pool.empty()) return cuda_fail(e, "workspace allocation");
            c->max_workspaces = (uint32_t)c->pool.size();   // out of memory: stop growing the pool
        }
        c->cv.wait(lk);
    }
}

void release(g16_circuit* c, Workspace* ws) {
    {
        std::lock_guard<std::mutex> g(c->mu);
        c->idle.push_back(ws);
    }
    c->cv.notify_one();
}

// Returns the workspace to its circuit's pool once every stream of it is idle:
// a call that failed after enqueueing may have left work running on a side
// stream, and the next proof on the workspace may reallocate its scratch (on a
// success the streams are idle already and the waits return at once).
struct WsGuard {
    g16_circuit* c;
    Workspace* ws = nullptr;
    explicit WsGuard(g16_circuit* cc) : c(cc) {}
    ~WsGuard() {
        if (!ws) return;
        for (cudaStream_t s : {ws->stream, ws->side[0], ws->side[1], ws->side[2], ws->side[3]})
            if (s) cudaStreamSynchronize(s);
        release(c, ws);
    }
};

bool is_one_mont(const uint8_t* w0) {
    host_init();
    return std::memcmp(w0, FR_P.one.v, 32) == 0;
}

// r * P for a standard-form scalar given as Montgomery Fr
G1J g1_mul(const G1J& p, const g16::Fr& k) {
    uint64_t s[4];
    k.to_std(s);
    return p.mul(s);
}
G2J g2_mul(const G2J& p, const g16::Fr& k) {
    uint64_t s[4];
    k.to_std(s);
    return p.mul(s);
}

}  // namespace

namespace g16 {

BlinderTerms blinder_terms(const g16_circuit* c, const g16::Fr& r, const g16::Fr& s) {
    BlinderTerms t;
    G1J d1 = G1J::from_affine(c->delta1);
    t.d1r = g1_mul(d1, r);
    t.d1s = g1_mul(d1, s);
    t.d1rs = g1_mul(d1, r * s);
    t.d2s = g2_mul(G2J::from_affine(c->delta2), s);
    return t;
}

void assemble(const g16_circuit* c, const MsmJac& m, const BlinderTerms& t, const g16::Fr& r, const g16::Fr& s,
              g16_proof* out) {
    G1J pi_a = m.a.add_affine(c->alpha1) + t.d1r;
    G2J pi_b = m.b2.add_affine(c->beta2) + t.d2s;
    G1J pib1 = m.b1.add_affine(c->beta1) + t.d1s;
    G1J pi_c = m.l + m.h + g1_mul(pi_a, s) + g1_mul(pib1, r) + t.d1rs.neg();
    G1J g1s[2] = {pi_a, pi_c};
    G1A g1a[2];
    batch_to_affine(g1s, g1a, 2);
    G2A g2a = pi_b.to_affine();
    pack(out->a, g1a[0]);
    pack(out->b, g2a);
    pack(out->c, g1a[1]);
}

void to_outputs(const MsmJac& m, g16_msm_outputs* o) {
    G1J g1s[4] = {m.a, m.b1, m.l, m.h};
    G1A a[4];
    batch_to_affine(g1s, a, 4);
    pack(o->a_g1, a[0]);
    pack(o->b_g1, a[1]);
    pack(o->l_g1, a[2]);
    pack(o->h_g1, a[3]);
    pack(o->b_g2, m.b2.to_affine());
}

int check_witness(const g16_circuit* c, size_t n, const uint8_t* w_host) {
    if (n != c->n_vars)
        return fail(G16_ERR_WITNESS_LENGTH, "witness has %zu values, the circuit has %u wires", n, c->n_vars);
    if (w_host && !is_one_mont(w_host)) return fail(G16_ERR_CONSTANT_WIRE, "witness[0] is not 1");
    return G16_OK;
}

}  // namespace g16

namespace {

uint64_t elapsed_us(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        (void)cudaGetLastError();   // an unrecorded stage event is not a launch failure
        return 0;
    }
    return (uint64_t)(ms * 1000.0);
}

// Stage boundary event.  Inside a stream capture a plain record only orders
// the captured work; the external flag turns it into an event-record node, so
// that every graph replay records it and the stage timings stay live.
cudaError_t stage_event(cudaEvent_t e, cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t err = cudaStreamIsCapturing(st, &cs);
    if (err != cudaSuccess) return err;
    return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal)
                                               : cudaEventRecord(e, st);
}

// stages 0-4 on the device witness; H left in h_out (device)
int run_h(g16_circuit* c, Workspace* ws, const void* d_w, void* h_out) {
    cudaStream_t st = ws->stream;
    uint8_t* abc = (uint8_t*)ws->d_abc;
    size_t vb = (size_t)c->n * 32;
    CK(stage_event(ws->ev[0], st), "event");
    {
        TimedLaunch tl("gather", st);
        g16d::k_gather<<<blocks_for(c->n, 256), 256, 0, st>>>(
            c->d_rp[0], c->d_sig[0], c->d_vid[0], c->d_rp[1], c->d_sig[1], c->d_vid[1], (const uint4*)c->d_values,
            (const uint4*)d_w, c->n, (uint4*)abc, (uint4*)(abc + vb), (uint4*)(abc + 2 * vb));
    }
    CK(cudaGetLastError(), "gather launch");
    CK(stage_event(ws->ev[1], st), "event");
    CK(ntt_h_pipeline(c->ntt, abc, abc + vb, abc + 2 * vb, h_out, st), "NTT pipeline");
    CK(stage_event(ws->ev[2], st), "event");
    return G16_OK;
}

// Stages 5-9.  The witness sort and the A, B1, L, B2 accumulations depend only
// on the witness, so they run on four side streams, one per MSM (ordered after
// the witness upload; the sort on the first), while the main stream does
// gather -> NTT -> H sort -> H accumulate; the main stream joins them before
// the results are read back.
int enqueue_witness_msms(g16_circuit* c, Workspace* ws, const void* d_w) {
    const size_t WIN_SLOT = ws->win_slot;
    // window tables: entry w rows + rank of a table of rows W points; compact:
    // entry rank of the plain bases
    const uint32_t W = c->tables ? (uint32_t)msm_windows(c->c_w) : 1u;
    cudaStream_t st[4];
    for (int i = 0; i < 4; i++) st[i] = c->serial ? ws->stream : ws->side[i];
    CK(cudaEventRecord(ws->ev_fork, ws->stream), "event");
    CK(cudaStreamWaitEvent(st[0], ws->ev_fork, 0), "stream wait");
    // one pass over the witness digits sorts the A, B and L live sets
    for (auto& x : ws->sort_w) x.reduce_pieces = witness_reduce_pieces();
    MsmLiveSets sets;
    sets.count = 3;
    for (int j = 0; j < 3; j++) {
        sets.d_rank[j] = c->d_rank[j];
        sets.rows[j] = c->rows[j];
    }
    CK(msm_sort_sets(ws->sort_w, sets, d_w, c->n_vars, true, c->c_w, st[0], c->be->constant_work, c->tables),
       "witness sort");
    CK(cudaEventRecord(ws->ev_sort, st[0]), "event");
    for (int i = 1; i < 4; i++) CK(cudaStreamWaitEvent(st[i], ws->ev_sort, 0), "stream wait");
    // acc slots: 0 A, 1 B2, 2 B1, 3 L (4 is H); one stream per MSM so that
    // their latency-bound reduction tails run side by side
    const bool t = c->tables;
    CK(msm_accumulate_g1(ws->sort_w[0], ws->acc[0], t ? c->t_a : c->d_a, 0, c->rows[0] * W, st[0]), "A accumulate");
    CK(msm_accumulate_g1(ws->sort_w[1], ws->acc[2], t ? c->t_b1 : c->d_b1, 0, c->rows[1] * W, st[1]), "B1 accumulate");
    CK(msm_accumulate_g1(ws->sort_w[2], ws->acc[3], t ? c->t_l : c->d_l, 0, c->rows[2] * W, st[2]), "L accumulate");
    CK(msm_accumulate_g2(ws->sort_w[1], ws->acc[1], t ? c->t_b2 : c->d_b2, 0, c->rows[1] * W, st[3]), "B2 accumulate");
    const int stream_of[4] = {0, 3, 1, 2};   // acc slot -> stream
    for (int i = 0; i < 4; i++) {
        cudaStream_t s_i = st[stream_of[i]];
        const size_t bytes = ws->acc[i].result_bytes(i == 1 ? XYZZ_G2_BYTES : XYZZ_G1_BYTES);
        if (bytes > WIN_SLOT) return fail(G16_ERR_BACKEND, "MSM result of %zu bytes exceeds its slot", bytes);
        CK(cudaMemcpyAsync(ws->h_win + i * WIN_SLOT, ws->acc[i].d_windows, bytes, cudaMemcpyDeviceToHost, s_i),
           "window readback");
        if (timer().enabled)
            CK(cudaMemcpyAsync(ws->h_work + i, ws->acc[i].d_work, 8, cudaMemcpyDeviceToHost, s_i), "work readback");
    }
    for (int i = 0; i < 4; i++) CK(cudaEventRecord(ws->ev_side[i], st[i]), "event");
    return G16_OK;
}

int enqueue_h_msm(g16_circuit* c, Workspace* ws, const void* d_h) {
    const size_t WIN_SLOT = ws->win_slot;
    cudaStream_t st = ws->stream;
    const uint32_t nh = c->h_count * (c->tables ? (uint32_t)msm_windows(c->c_h) : 1u);
    // the H reduction runs last on the main stream, mostly alone: shorter chains pay
    // (2^21 prove +0.5%, 2^18 +1.5%, 2^20 +1.3% against the 8192-piece default)
    ws->sort_h.reduce_pieces = MSM_REDUCE_PIECES_ALONE;
    CK(msm_sort(ws->sort_h, d_h, c->h_count, true, c->c_h, st, c->tables, c->be->constant_work), "H sort");
    CK(msm_accumulate_g1(ws->sort_h, ws->acc[4], c->tables ? c->t_h : c->d_h, 0, nh, st), "H accumulate");
    const size_t bytes = ws->acc[4].result_bytes(XYZZ_G1_BYTES);
    if (bytes > WIN_SLOT) return fail(G16_ERR_BACKEND, "MSM result of %zu bytes exceeds its slot", bytes);
    CK(cudaMemcpyAsync(ws->h_win + 4 * WIN_SLOT, ws->acc[4].d_windows, bytes, cudaMemcpyDeviceToHost, st),
       "window readback");
    if (timer().enabled)
        CK(cudaMemcpyAsync(ws->h_work + 4, ws->acc[4].d_work, 8, cudaMemcpyDeviceToHost, st), "work readback");
    return G16_OK;
}

int enqueue_join(Workspace* ws) {
    for (int i = 0; i < 4; i++) CK(cudaStreamWaitEvent(ws->stream, ws->ev_side[i], 0), "stream wait");
    CK(stage_event(ws->ev[3], ws->stream), "event");
    return G16_OK;
}

int collect_msms(g16_circuit* c, Workspace* ws, MsmJac& out) {
    const size_t WIN_SLOT = ws->win_slot;
    CK(cudaStreamSynchronize(ws->stream), "MSM stages");
    timer().collect();
    {
        std::lock_guard<std::mutex> g(c->mu);
        c->readback_bytes = 0;
        for (int i = 0; i < 5; i++) c->readback_bytes += ws->acc[i].result_bytes(i == 1 ? XYZZ_G2_BYTES : XYZZ_G1_BYTES);
    }
    if (timer().enabled) {
        timer().add_units("msm_accumulate_g1",
                          (double)(ws->h_work[0] + ws->h_work[2] + ws->h_work[3] + ws->h_work[4]));
        timer().add_units("msm_accumulate_g2", (double)ws->h_work[1]);
    }
    out.a = msm_combine_g1(ws->h_win + 0 * WIN_SLOT, ws->acc[0].plan, c->c_w);
    out.b2 = msm_combine_g2(ws->h_win + 1 * WIN_SLOT, ws->acc[1].plan, c->c_w);
    out.b1 = msm_combine_g1(ws->h_win + 2 * WIN_SLOT, ws->acc[2].plan, c->c_w);
    out.l = msm_combine_g1(ws->h_win + 3 * WIN_SLOT, ws->acc[3].plan, c->c_w);
    out.h = msm_combine_g1(ws->h_win + 4 * WIN_SLOT, ws->acc[4].plan, c->c_h);
    return G16_OK;
}

// stages 0-9 for a witness already in device memory, enqueued on ws's streams
int enqueue_proof(g16_circuit* c, Workspace* ws, const void* d_w) {
    int rc = enqueue_witness_msms(c, ws, d_w);
    if (rc == G16_OK) rc = run_h(c, ws, d_w, ws->d_hpoly);
    if (rc == G16_OK) rc = enqueue_h_msm(c, ws, ws->d_hpoly);
    if (rc == G16_OK) rc = enqueue_join(ws);
    return rc;
}

// Stages 0-9.  From the second proof on a workspace (when every scratch buffer
// has reached its size) the whole enqueue sequence is captured once as a CUDA
// graph over the workspace's five streams and replayed, one launch per proof.
int run_proof(g16_circuit* c, Workspace* ws, const void* d_w, MsmJac& out) {
    bool use_graph = c->graphs && !c->serial && !timer().enabled && ws->proofs > 0;
    if (use_graph) {
        if (d_w != ws->d_w)
            CK(cudaMemcpyAsync(ws->d_w, d_w, 32ull * c->n_vars, cudaMemcpyDeviceToDevice, ws->stream), "witness copy");
        if (ws->graph && ws->graph_constant_work != c->be->constant_work) {   // captured in the other mode
            cudaGraphExecDestroy(ws->graph);
            ws->graph = nullptr;
        }
        if (!ws->graph) {
            ws->graph_constant_work = c->be->constant_work;
            uint64_t k0 = timer().launches.load();
            CK(cudaStreamBeginCapture(ws->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
            int rc = enqueue_proof(c, ws, ws->d_w);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(ws->stream, &g);
            if (rc != G16_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            CK(e, "graph capture");
            e = cudaGraphInstantiate(&ws->graph, g, 0);
            cudaGraphDestroy(g);
            CK(e, "graph instantiate");
            ws->graph_kernels = timer().launches.load() - k0;
            timer().launches.fetch_sub(ws->graph_kernels);   // counted when replayed
        }
        CK(cudaGraphLaunch(ws->graph, ws->stream), "graph launch");
        timer().launches.fetch_add(ws->graph_kernels);
    } else {
        int rc = enqueue_proof(c, ws, d_w);
        if (rc != G16_OK) return rc;
    }
    int rc = collect_msms(c, ws, out);
    if (rc == G16_OK) ws->proofs++;
    return rc;
}

void add_timings(g16_circuit* c, Workspace* ws, bool h, bool msm, uint64_t assemble_us) {
    std::lock_guard<std::mutex> g(c->mu);
    if (h) {
        c->t.gather_us += elapsed_us(ws->ev[0], ws->ev[1]);
        c->t.ntt_us += elapsed_us(ws->ev[1], ws->ev[2]);
    }
    if (msm) c->t.msm_us += elapsed_us(ws->ev[2], ws->ev[3]);
    c->t.assemble_us += assemble_us;
}

int prove_on_device(g16_circuit* c, Workspace* ws, const void* d_w, const uint8_t* r_mont, const uint8_t* s_mont,
                    g16_proof* out) {
    g16::Fr r = g16::Fr::raw((const uint64_t*)r_mont), s = g16::Fr::raw((const uint64_t*)s_mont);
    uint64_t rr[4], ss[4];
    std::memcpy(rr, r_mont, 32);
    std::memcpy(ss, s_mont, 32);
    if (!g16::Fr::canonical(rr) || !g16::Fr::canonical(ss)) return fail(G16_ERR_INVALID_ARGUMENT, "r or s not below r");
    auto terms = std::async(std::launch::async, [&] { return blinder_terms(c, r, s); });
    MsmJac m;
    int rc = run_proof(c, ws, d_w, m);
    BlinderTerms t = terms.get();
    if (rc != G16_OK) return rc;
    auto t0 = std::chrono::steady_clock::now();
    assemble(c, m, t, r, s, out);
    auto t1 = std::chrono::steady_clock::now();
    add_timings(c, ws, true, true, (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count());
    return G16_OK;
}

// Stages 1-9 from the caller's A.w and B.w rows (stage 0 handed over): the
// witness MSMs fork as in a proof, the main stream pads the rows to the
// domain, forms C = A B and runs the NTT chain and the H MSM.
int run_rows_proof(g16_circuit* c, Workspace* ws, const void* d_w, const uint8_t* a_rows, const uint8_t* b_rows,
                   size_t rows, MsmJac& out) {
    cudaStream_t st = ws->stream;
    uint8_t* abc = (uint8_t*)ws->d_abc;
    const size_t vb = (size_t)c->n * 32;
    int rc = enqueue_witness_msms(c, ws, d_w);
    if (rc) return rc;
    CK(stage_event(ws->ev[0], st), "event");
    for (int m = 0; m < 2; m++) {
        uint8_t* dst = abc + m * vb;
        if (rows) CK(cudaMemcpyAsync(dst, m ? b_rows : a_rows, rows * 32, cudaMemcpyHostToDevice, st), "rows upload");
        if (rows < c->n) CK(cudaMemsetAsync(dst + rows * 32, 0, vb - rows * 32, st), "rows padding");
    }
    {
        TimedLaunch tl("gather", st);
        g16d::k_rows_c<<<blocks_for(c->n, 256), 256, 0, st>>>((const uint4*)abc, (const uint4*)(abc + vb),
                                                               (uint4*)(abc + 2 * vb), c->n);
    }
    CK(cudaGetLastError(), "rows launch");
    CK(stage_event(ws->ev[1], st), "event");
    CK(ntt_h_pipeline(c->ntt, abc, abc + vb, abc + 2 * vb, ws->d_hpoly, st), "NTT pipeline");
    if (c->rows_only) {
        // gnark's basis: H's coefficients (times -2) in bit-reversed order; the
        // last one, coefficient n - 1, comes back to be checked for zero
        CK(ntt_to_gnark_coefficients(c->ntt, ws->d_hpoly, st), "gnark coefficients");
        CK(cudaMemcpyAsync(ws->h_work + 8, (const uint8_t*)ws->d_hpoly + 32ull * (c->n - 1), 32,
                           cudaMemcpyDeviceToHost, st),
           "coefficient readback");
    }
    CK(stage_event(ws->ev[2], st), "event");
    if ((rc = enqueue_h_msm(c, ws, ws->d_hpoly)) || (rc = enqueue_join(ws))) return rc;
    if ((rc = collect_msms(c, ws, out))) return rc;
    if (c->rows_only) {
        // A B - C vanishes on the domain and has degree at most 2n - 2, so its
        // quotient by t has degree at most n - 2 (to_gnark_coefficients,
        // crates/groth16/src/cpu.rs:265-286)
        if (ws->h_work[8] | ws->h_work[9] | ws->h_work[10] | ws->h_work[11])
            return fail(G16_ERR_BACKEND, "H has a nonzero coefficient %u, so the quotient by the vanishing polynomial "
                                         "is not exact", c->n - 1);
        // gnark's Z bases carry t(tau) / delta; on the odd coset t = -2
        out.h = g1_mul(out.h, -g16::Fr::from_u64(2).inv());
    }
    ws->proofs++;
    return G16_OK;
}

// The gather-path entry points need the constraint matrices a gnark key lacks.
int gather_ok(const g16_circuit* c) {
    if (c->rows_only)
        return fail(G16_ERR_BACKEND, "this key has no constraint matrices (a gnark key): it proves only from A.w and "
                                     "B.w rows (g16_prove_with_blinders_from_rows)");
    return G16_OK;
}

int check_rows(const g16_circuit* c, const uint8_t* a_rows, const uint8_t* b_rows, size_t rows) {
    if (rows && (!a_rows || !b_rows)) return fail(G16_ERR_INVALID_ARGUMENT, "null rows");
    if (rows > c->n)
        return fail(G16_ERR_BACKEND, "A.w and B.w have %zu rows; both must be one per constraint, at most the domain "
                                     "size %u", rows, c->n);
    return G16_OK;
}

int upload_witness(Workspace* ws, const uint8_t* w, size_t n) {
    CK(cudaMemcpyAsync(ws->d_w, w, n * 32, cudaMemcpyHostToDevice, ws->stream), "witness upload");
    return G16_OK;
}

// ---- per-instance tuning ----

// Minimum over reps of the device time of enqueue() on ws->stream (after one
// untimed run); negative on failure, with the error already set.
template <class Fn>
double time_on_stream(Workspace* ws, int reps, Fn&& enqueue) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        cuda_fail(cudaGetLastError(), "tuning events");
        return -1.0;
    }
    double best = -1.0;
    for (int i = 0; i <= reps; i++) {
        cudaError_t e = cudaEventRecord(e0, ws->stream);
        if (e != cudaSuccess) {
            cuda_fail(e, "tuning");
            best = -1.0;
            break;
        }
        if (enqueue() != G16_OK) {
            best = -1.0;
            break;
        }
        e = cudaEventRecord(e1, ws->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
        if (e != cudaSuccess) {
            cuda_fail(e, "tuning");
            best = -1.0;
            break;
        }
        if (i > 0 && (best < 0 || ms < best)) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return best;
}

// Holds the circuit's proof path for tuning: the one workspace in ws is the
// only one out of the pool, no other proof can start until release.
struct TuningLock {
    g16_circuit* c;
    Workspace* ws = nullptr;            // the first workspace (also in all[0])
    std::vector<Workspace*> all;        // every workspace the tuner holds
    bool held = false;
    explicit TuningLock(g16_circuit* cc) : c(cc) {}
    // Take one workspace; the circuit must have no proof in flight.  Then
    // up to `want` workspaces in all (idle ones first, new ones while the
    // memory budget allows), for the concurrent objective.
    int take(int want = 1) {
        int rc = acquire(c, &ws);
        if (rc) return rc;
        all.push_back(ws);
        std::unique_lock<std::mutex> g(c->mu);
        if (c->idle.size() + 1 != c->pool.size())
            return fail(G16_ERR_INVALID_ARGUMENT, "tuning needs a circuit with no proof in flight");
        c->tuning = true;
        held = true;
        c->cv.wait(g, [&] { return c->batch_users == 0; });   // batched submissions reading the tables finish first
        while ((int)all.size() < want) {
            if (!c->idle.empty()) {
                all.push_back(c->idle.back());
                c->idle.pop_back();
                continue;
            }
            if (c->pool.size() >= c->max_workspaces || c->be->vram_used + c->ws_estimate > c->be->vram_limit) break;
            auto w = std::make_unique<Workspace>();
            if (w->init(c->n_vars, c->n, win_slot(c)) != cudaSuccess) {
                w->release();
                cudaGetLastError();
                break;
            }
            c->device_bytes += c->ws_estimate;
            c->be->vram_used += c->ws_estimate;
            all.push_back(w.get());
            c->pool.push_back(std::move(w));
        }
        return G16_OK;
    }
    ~TuningLock() {
        if (held) {
            // captured graphs hold the old tables and launch shapes: capture again
            for (auto& w : c->pool) {
                if (w->graph) cudaGraphExecDestroy(w->graph);
                w->graph = nullptr;
                w->proofs = 0;
            }
            c->ws_estimate = workspace_estimate(c->n_vars, c->n, c->c_w, c->c_h, c->rows[0], c->rows[1], c->rows[2], c->tables);
        }
        {
            std::lock_guard<std::mutex> g(c->mu);
            for (Workspace* w : all) c->idle.push_back(w);
            if (held) c->tuning = false;
        }
        c->cv.notify_all();
    }
};

// Device time per proof with stages 0-9 of one proof on every workspace in
// flight together (the batched / served objective): the minimum over reps of
// (last workspace done - common start) / workspaces.  Negative on failure.
double time_concurrent(g16_circuit* c, const std::vector<Workspace*>& all, int reps) {
    std::vector<cudaEvent_t> ev(all.size() + 1, nullptr);
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) {
            for (auto& x : ev)
                if (x) cudaEventDestroy(x);
            cuda_fail(cudaGetLastError(), "tuning events");
            return -1.0;
        }
    double best = -1.0;
    for (int r = 0; r <= reps && best != -2.0; r++) {
        cudaError_t e = cudaEventRecord(ev[0], all[0]->stream);
        for (size_t i = 1; i < all.size() && e == cudaSuccess; i++) e = cudaStreamWaitEvent(all[i]->stream, ev[0], 0);
        if (e != cudaSuccess) {
            cuda_fail(e, "tuning");
            best = -2.0;
            break;
        }
        for (size_t i = 0; i < all.size(); i++) {
            if (enqueue_proof(c, all[i], all[i]->d_w) != G16_OK) {
                best = -2.0;
                break;
            }
            e = cudaEventRecord(ev[i + 1], all[i]->stream);
            if (e != cudaSuccess) {
                cuda_fail(e, "tuning");
                best = -2.0;
                break;
            }
        }
        if (best == -2.0) break;
        float worst = 0;
        for (size_t i = 0; i < all.size(); i++) {
            float ms = 0;
            e = cudaEventSynchronize(ev[i + 1]);
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[i + 1]);
            if (e != cudaSuccess) {
                cuda_fail(e, "tuning");
                best = -2.0;
                break;
            }
            worst = ms > worst ? ms : worst;
        }
        double per = worst / (double)all.size();
        if (best != -2.0 && r > 0 && (best < 0 || per < best)) best = per;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    return best == -2.0 ? -1.0 : best;
}

// The witness MSMs' live sets, computed on the host at prepare: per set the
// compacted bases and, per wire, its row in them (MSM_DEAD where its base is
// the point at infinity).  Set 0 is A, 1 is B (B1 and B2), 2 is L.
struct LiveSetsHost {
    std::vector<uint8_t> a, b1, b2, l;
    std::vector<uint32_t> rank[3];
    uint32_t rows[3] = {0, 0, 0};
};

bool all_zero(const uint8_t* p, size_t bytes) {
    for (size_t i = 0; i < bytes; i++)
        if (p[i]) return false;
    return true;
}

LiveSetsHost live_sets(const g16_zkey_view& k) {
    LiveSetsHost r;
    const size_t nv = k.n_vars, first = (size_t)k.n_public + 1;
    for (auto& x : r.rank) x.assign(nv, MSM_DEAD);
    for (size_t i = 0; i < nv; i++) {
        const uint8_t* a = k.a_query + 64 * i;
        if (!all_zero(a, 64)) {
            r.rank[0][i] = r.rows[0]++;
            r.a.insert(r.a.end(), a, a + 64);
        }
        const uint8_t *b1 = k.b_g1_query + 64 * i, *b2 = k.b_g2_query + 128 * i;
        if (!all_zero(b1, 64) || !all_zero(b2, 128)) {
            r.rank[1][i] = r.rows[1]++;
            r.b1.insert(r.b1.end(), b1, b1 + 64);
            r.b2.insert(r.b2.end(), b2, b2 + 128);
        }
        if (i >= first) {
            const uint8_t* l = k.l_query + 64 * (i - first);
            if (!all_zero(l, 64)) {
                r.rank[2][i] = r.rows[2]++;
                r.l.insert(r.l.end(), l, l + 64);
            }
        }
    }
    return r;
}

bool window_bits_ok(int b) { return b >= 8 && b <= 20; }

// How a key is held (g16_plan_key): the window tables when the key, its tables
// and one workspace fit in free_bytes, else the compact key (plain bases, one
// bucket set per window) when it and one workspace fit, else DEVICE_MEMORY.
// G16_CUDA_WINDOW_TABLES=0 takes the compact key whenever it fits.
int plan_key(const g16_zkey_view& k, const uint32_t rows[3], uint64_t free_bytes, g16_key_plan* out) {
    const uint64_t nv = k.n_vars, n = k.domain_size;
    const uint64_t ra = rows[0], rb = rows[1], rl = rows[2];
    // CSR, interned values, compacted bases, rank arrays, H bases, twiddles and coset table
    const uint64_t plain = 4ull * (n + 1) * 2 + 8ull * (k.nnz[0] + k.nnz[1]) + 32ull * k.n_values + ra * 64 +
                           rb * (64 + 128) + rl * 64 + 12 * nv + n * 64 + n * 32 * 2 + 32;
    const char* env = std::getenv("G16_CUDA_WINDOW_TABLES");
    const bool allow_tables = !(env && std::strcmp(env, "0") == 0);
    g16_key_plan t = {};
    t.window_tables = 1;
    t.msm_window_bits_witness = msm_shared_window_bits(nv / 2 + 1);
    t.msm_window_bits_h = msm_shared_window_bits(n);
    {
        const uint64_t Ww = (uint64_t)msm_windows(t.msm_window_bits_witness), Wh = (uint64_t)msm_windows(t.msm_window_bits_h);
        t.key_bytes = plain + (ra + rl) * Ww * 64 + rb * Ww * (64 + 128) + n * Wh * 64;
        t.workspace_bytes = workspace_estimate(nv, n, t.msm_window_bits_witness, t.msm_window_bits_h, ra, rb, rl, true);
    }
    g16_key_plan m = {};
    m.window_tables = 0;
    m.msm_window_bits_witness = msm_window_bits(std::max<uint64_t>(1, std::max(ra, std::max(rb, rl))));
    m.msm_window_bits_h = msm_window_bits(n);
    m.key_bytes = plain;
    m.workspace_bytes = workspace_estimate(nv, n, m.msm_window_bits_witness, m.msm_window_bits_h, ra, rb, rl, false);
    for (const g16_key_plan* p : {&t, &m}) {
        // sorted entries are 31-bit indices in either form
        const uint64_t Ww = (uint64_t)msm_windows(p->msm_window_bits_witness), Wh = (uint64_t)msm_windows(p->msm_window_bits_h);
        if (nv * Ww >= 0x80000000ull || n * Wh >= 0x80000000ull)
            return fail(G16_ERR_BACKEND, "circuit too large for 31-bit MSM entry indices");
    }
    if (allow_tables && t.key_bytes + t.workspace_bytes <= free_bytes) {
        *out = t;
        return G16_OK;
    }
    if (m.key_bytes + m.workspace_bytes <= free_bytes) {
        *out = m;
        return G16_OK;
    }
    return fail(G16_ERR_DEVICE_MEMORY,
                "circuit needs about %llu MiB of device memory with window tables and %llu MiB as a compact key; "
                "%llu MiB are free",
                (unsigned long long)((t.key_bytes + t.workspace_bytes) >> 20),
                (unsigned long long)((m.key_bytes + m.workspace_bytes) >> 20), (unsigned long long)(free_bytes >> 20));
}

int apply_tuning(g16_circuit* c, Workspace* ws, const g16_tuning& t) {
    NttTiling tl = {(uint32_t)t.ntt_tile_log, (uint32_t)t.ntt_outer_log_l};
    if (!window_bits_ok(t.msm_window_bits_witness) || !window_bits_ok(t.msm_window_bits_h) || t.ntt_tile_log < 2 ||
        t.ntt_outer_log_l < 0 || !ntt_tiling_valid(tl))
        return fail(G16_ERR_INVALID_ARGUMENT, "tuning out of range: window bits %d/%d (8..20), NTT tile 2^%d, %d",
                    t.msm_window_bits_witness, t.msm_window_bits_h, t.ntt_tile_log, t.ntt_outer_log_l);
    int rc = G16_OK;
    if (t.msm_window_bits_witness != c->c_w) rc = build_witness_tables(c, t.msm_window_bits_witness, ws->stream);
    if (rc == G16_OK && t.msm_window_bits_h != c->c_h) rc = build_h_table(c, t.msm_window_bits_h, ws->stream);
    if (rc == G16_OK) c->ntt.tiling = tl;
    return rc;
}

g16_tuning current_tuning(const g16_circuit* c) {
    g16_tuning t = c->tuned;
    t.msm_window_bits_witness = c->c_w;
    t.msm_window_bits_h = c->c_h;
    t.ntt_tile_log = (int32_t)c->ntt.tiling.tile_log;
    t.ntt_outer_log_l = (int32_t)c->ntt.tiling.outer_log_l;
    return t;
}

// Hill-climb one window size: try the neighbours of the current value and keep
// moving while the timed stage gets faster.
template <class Build, class Time>
int climb_window(int start, Build&& build, Time&& time_it, int* best_out) {
    double t0 = time_it();
    if (t0 < 0) return G16_ERR_DEVICE;
    int best = start;
    double best_t = t0;
    for (int dir : {+1, -1}) {
        int b = best + dir;
        while (window_bits_ok(b) && b != start) {
            int rc = build(b);
            if (rc) return rc;
            double t = time_it();
            if (t < 0) return G16_ERR_DEVICE;
            if (t < best_t * 0.99) {
                best_t = t;
                best = b;
                b += dir;
            } else {
                break;
            }
        }
        if (best != start) break;   // improved upward: do not try downward
    }
    int rc = build(best);
    if (rc) return rc;
    *best_out = best;
    return G16_OK;
}

}  // namespace

// ---------------------------------------------------------------- C ABI
extern "C" {

size_t g16_last_error(char* buf, size_t len) {
    const std::string& e = g_err;
    if (buf && len) {
        size_t k = e.size() < len - 1 ? e.size() : len - 1;
        std::memcpy(buf, e.data(), k);
        buf[k] = 0;
    }
    return e.size();
}

int g16_cuda_error_class(int cuda_error) { return error_class(cuda_error); }

int g16_backend_fault(const g16_backend* b) {
    if (!b) return 0;
    const int f = b->fault.load();
    return f ? f : g16::device_fault(b->ordinal);
}

int g16_backend_inject_fault(g16_backend* b, int cuda_error) {
    if (!b || cuda_error < 0) return fail(G16_ERR_INVALID_ARGUMENT, "g16_backend_inject_fault: need a backend and a status >= 0");
    b->inject = cuda_error;
    return G16_OK;
}

int g16_backend_set_constant_work(g16_backend* b, int on) {
    if (!b) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    b->constant_work = on != 0;
    return G16_OK;
}

int g16_backend_open(int ordinal, uint64_t vram_limit, g16_backend** out) {
    if (!out) return fail(G16_ERR_INVALID_ARGUMENT, "null output handle");
    host_init();
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(G16_ERR_DEVICE, "no CUDA device: %s", e != cudaSuccess ? cudaGetErrorString(e) : "count is 0");
    if (ordinal < 0 || ordinal >= count) return fail(G16_ERR_DEVICE, "CUDA device %d of %d", ordinal, count);
    if (const int f = g16::device_fault(ordinal))
        return fail(G16_ERR_DEVICE, "CUDA device %d is out of use after %s: a sticky fault earlier in this process", ordinal,
                    cudaGetErrorString((cudaError_t)f));
    CK(cudaSetDevice(ordinal), "cudaSetDevice");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, ordinal), "cudaGetDeviceProperties");
    if (prop.major < 10) return fail(G16_ERR_DEVICE, "device %d is sm_%d%d; this build targets sm_100a", ordinal, prop.major, prop.minor);
    auto b = std::make_unique<g16_backend>();
    b->ordinal = ordinal;
    size_t free_b = 0, total_b = 0;
    CK(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    b->vram_limit = vram_limit ? vram_limit : (uint64_t)free_b;
    CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
    *out = b.release();
    return G16_OK;
}

void g16_backend_free(g16_backend* b) {
    if (!b) return;
    cudaSetDevice(b->ordinal);
    batch_free(b);
    cudaStreamSynchronize(b->stream);
    b->sort.release();
    b->acc.release();
    cudaFree(b->d_in);
    cudaFree(b->d_in2);
    for (auto& t : b->ntt)
        if (t) t->release();
    cudaFreeHost(b->h_pinned);
    if (b->h_work) cudaFreeHost(b->h_work);
    cudaStreamDestroy(b->stream);
    delete b;
}

const char* g16_backend_name(const g16_backend*) { return "cuda-b200"; }
uint64_t g16_backend_vram_used(const g16_backend* b) { return b ? b->vram_used.load() : 0; }

// ---- formats ----
int g16_zkey_parse(const uint8_t* bytes, size_t len, int check_points, g16_zkey** out) {
    if (!bytes || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    auto z = std::make_unique<g16_zkey>();
    int rc = zkey_parse(bytes, len, check_points != 0, z->k);
    if (rc != G16_OK) return rc;
    *out = z.release();
    return G16_OK;
}

int g16_gnark_key_parse(const uint8_t* pk, size_t pk_len, const uint8_t* vk, size_t vk_len, g16_zkey** out) {
    if (!pk || !vk || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    auto z = std::make_unique<g16_zkey>();
    int rc = gnark_key_parse(pk, pk_len, vk, vk_len, z->k);
    if (rc != G16_OK) return rc;
    *out = z.release();
    return G16_OK;
}

int g16_gnark_witness_parse(const uint8_t* bytes, size_t len, uint8_t* w, size_t w_cap, uint8_t* aw, uint8_t* bw,
                            size_t rows_cap, size_t* n_w, size_t* n_rows) {
    if (!bytes) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint8_t> parts[3];
    int rc = gnark_witness_parse(bytes, len, parts);
    if (rc != G16_OK) return rc;
    const size_t nw = parts[0].size() / 32, nr = parts[1].size() / 32;
    if (n_w) *n_w = nw;
    if (n_rows) *n_rows = nr;
    if (w) {
        if (w_cap < nw) return fail(G16_ERR_INVALID_ARGUMENT, "witness buffer holds %zu of %zu values", w_cap, nw);
        std::memcpy(w, parts[0].data(), parts[0].size());
    }
    if (aw || bw) {
        if (!aw || !bw || rows_cap < nr) return fail(G16_ERR_INVALID_ARGUMENT, "row buffers hold %zu of %zu rows", rows_cap, nr);
        std::memcpy(aw, parts[1].data(), parts[1].size());
        std::memcpy(bw, parts[2].data(), parts[2].size());
    }
    return G16_OK;
}

int g16_zkey_view_get(const g16_zkey* k, g16_zkey_view* out) {
    if (!k || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    zkey_view(k->k, *out);
    return G16_OK;
}

void g16_zkey_free(g16_zkey* k) { delete k; }

int g16_wtns_parse(const uint8_t* bytes, size_t len, uint8_t* out_mont, size_t cap, size_t* n_out) {
    if (!bytes || !n_out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint8_t> w;
    int rc = wtns_parse(bytes, len, w);
    if (rc != G16_OK) return rc;
    *n_out = w.size() / 32;
    if (!out_mont) return G16_OK;
    if (cap < *n_out) return fail(G16_ERR_INVALID_ARGUMENT, "witness buffer holds %zu of %zu values", cap, *n_out);
    std::memcpy(out_mont, w.data(), w.size());
    return G16_OK;
}

int g16_wtns_write(const uint8_t* w_mont, size_t n, uint8_t* out, size_t cap, size_t* len_out) {
    if (!w_mont || !len_out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint8_t> b = wtns_write(w_mont, n);
    *len_out = b.size();
    if (!out) return G16_OK;
    if (cap < b.size()) return fail(G16_ERR_INVALID_ARGUMENT, "buffer too small");
    std::memcpy(out, b.data(), b.size());
    return G16_OK;
}


// ---- prepare ----
int g16_prepare(g16_backend* b, const g16_zkey_view* k, g16_circuit** out) {
    if (!b || !k || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    uint32_t n = k->domain_size;
    if (n < 2 || (n & (n - 1)) || n > (1u << 27)) return fail(G16_ERR_BACKEND, "domain size %u is not a power of two in [2, 2^27]", n);
    if ((uint64_t)k->n_public + 1 > k->n_vars) return fail(G16_ERR_BACKEND, "n_public %u exceeds n_vars %u", k->n_public, k->n_vars);
    if (k->n_vars >= 0x80000000u || n >= 0x80000000u) return fail(G16_ERR_BACKEND, "more than 2^31 wires");
    if (k->h_basis > G16_H_GNARK) return fail(G16_ERR_BACKEND, "unknown H basis %u", k->h_basis);
    // a gnark key has no constraint matrices: it proves only from A.w and B.w rows
    const bool gnark = k->h_basis == G16_H_GNARK;
    // CSR structure (Coefficients::check_structure, formats/src/lib.rs:185-270)
    for (int m = 0; m < 2 && !gnark; m++) {
        const uint32_t* rp = k->row_ptr[m];
        if (!rp || rp[0] != 0 || rp[n] != k->nnz[m]) return fail(G16_ERR_BACKEND, "matrix %d row_ptr is malformed", m);
        for (uint32_t i = 0; i < n; i++)
            if (rp[i + 1] < rp[i]) return fail(G16_ERR_BACKEND, "matrix %d row_ptr is not monotone at row %u", m, i);
        for (uint32_t i = 0; i < k->nnz[m]; i++) {
            if (k->signal[m][i] >= k->n_vars) return fail(G16_ERR_BACKEND, "matrix %d nonzero %u references signal %u", m, i, k->signal[m][i]);
            if (k->value_id[m][i] >= k->n_values) return fail(G16_ERR_BACKEND, "matrix %d nonzero %u references value %u", m, i, k->value_id[m][i]);
        }
    }
    uint64_t nv = k->n_vars;
    // live sets (the reference's key_live, crates/cuda/src/msm.rs:1308, and
    // prescan's infinity filter, crates/msm/src/lib.rs:554-563): a wire whose
    // base is the point at infinity adds nothing to that MSM, so its bases are
    // compacted out and its digits never become entries.  A: a_query finite;
    // B: b_g1_query or b_g2_query finite (B1 and B2 share one sort); L: a
    // private wire whose l_query point is finite.
    LiveSetsHost live = live_sets(*k);
    // memory budget, refused before any allocation (backend.rs:367-381); the
    // compact key when the window tables do not fit
    g16_key_plan plan;
    const uint64_t free_bytes = b->vram_limit - std::min<uint64_t>(b->vram_limit, b->vram_used);
    int rc = plan_key(*k, live.rows, free_bytes, &plan);
    if (rc) return rc;
    const int c_w = plan.msm_window_bits_witness, c_h = plan.msm_window_bits_h;
    auto c = std::make_unique<g16_circuit>();
    c->be = b;
    c->n_vars = k->n_vars;
    c->n_public = k->n_public;
    c->n = n;
    c->tables = plan.window_tables != 0;
    c->ws_estimate = plan.workspace_bytes;
    c->rows_only = gnark;
    c->h_count = gnark ? n - 1 : n;
    for (int j = 0; j < 3; j++) c->rows[j] = live.rows[j];
    if (const char* g = std::getenv("G16_CUDA_GRAPHS")) c->graphs = std::strcmp(g, "0") != 0;
    while ((1u << c->log_n) < n) c->log_n++;
    if (!unpack(c->alpha1, k->alpha_g1) || !unpack(c->beta1, k->beta_g1) || !unpack(c->delta1, k->delta_g1) ||
        !unpack(c->beta2, k->beta_g2) || !unpack(c->delta2, k->delta_g2))
        return fail(G16_ERR_BACKEND, "non-canonical header point");
    if (c->alpha1.inf || c->beta1.inf || c->delta1.inf || c->beta2.inf || c->delta2.inf)
        return fail(G16_ERR_BACKEND, "a header point is the point at infinity");
    if (k->gamma_g2 && !unpack(c->gamma2, k->gamma_g2)) return fail(G16_ERR_BACKEND, "non-canonical gamma_g2");
    if (!k->gamma_g2) c->gamma2.inf = true;
    if (k->ic) {
        c->ic.resize((size_t)k->n_public + 1);
        for (size_t i = 0; i <= k->n_public; i++)
            if (!unpack(c->ic[i], k->ic + 64 * i)) return fail(G16_ERR_BACKEND, "non-canonical IC point %zu", i);
    }
    struct Up {
        void** dst;
        const void* src;
        size_t bytes;
    } ups[] = {
        {(void**)&c->d_rp[0], k->row_ptr[0], gnark ? 0 : 4ull * (n + 1)},
        {(void**)&c->d_rp[1], k->row_ptr[1], gnark ? 0 : 4ull * (n + 1)},
        {(void**)&c->d_sig[0], k->signal[0], gnark ? 0 : 4ull * k->nnz[0]},
        {(void**)&c->d_sig[1], k->signal[1], gnark ? 0 : 4ull * k->nnz[1]},
        {(void**)&c->d_vid[0], k->value_id[0], gnark ? 0 : 4ull * k->nnz[0]},
        {(void**)&c->d_vid[1], k->value_id[1], gnark ? 0 : 4ull * k->nnz[1]},
        {&c->d_values, k->values, gnark ? 0 : 32ull * k->n_values},
        {&c->d_a, live.a.data(), live.a.size()},
        {&c->d_b1, live.b1.data(), live.b1.size()},
        {&c->d_b2, live.b2.data(), live.b2.size()},
        {&c->d_l, live.l.data(), live.l.size()},
        {(void**)&c->d_rank[0], live.rank[0].data(), 4ull * nv},
        {(void**)&c->d_rank[1], live.rank[1].data(), 4ull * nv},
        {(void**)&c->d_rank[2], live.rank[2].data(), 4ull * nv},
        {&c->d_h, k->h_query, 64ull * (gnark ? n - 1 : n)},
    };
    g16_circuit* cp = c.get();
    cudaStream_t st = b->stream;
    std::lock_guard<std::mutex> bg(b->mu);   // the backend stream does the uploads
    auto cleanup = [&] { g16_circuit_free(c.release()); };
    for (auto& u : ups) {
        cudaError_t e = circuit_alloc(cp, u.dst, u.bytes);
        if (e == cudaSuccess && u.bytes) e = cudaMemcpyAsync(*u.dst, u.src, u.bytes, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            int rc = cuda_fail(e, "key upload");
            cleanup();
            return rc;
        }
    }
    cudaError_t e = ntt_tables(cp->ntt, cp->log_n, st);
    if (e == cudaSuccess && gnark) e = ntt_gnark_table(cp->ntt, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        int rc = cuda_fail(e, "prepare");
        cleanup();
        return rc;
    }
    cp->device_bytes += 3ull * 32 * n / 2 * 2;
    // window-shifted base tables (none for a compact key)
    rc = build_witness_tables(cp, c_w, st);
    if (rc == G16_OK) rc = build_h_table(cp, c_h, st);
    if (rc != G16_OK) {
        cleanup();
        return rc;
    }
    *out = c.release();
    return G16_OK;
}

void g16_circuit_free(g16_circuit* c) {
    if (!c) return;
    cudaSetDevice(c->be->ordinal);
    batch_forget(c->be, c);
    for (auto& ws : c->pool) ws->release();
    c->pool.clear();
    c->idle.clear();
    for (void* p : c->allocs) cudaFree(p);
    c->be->vram_used -= std::min<uint64_t>(c->be->vram_used, c->device_bytes);
    c->ntt.release();
    delete c;
}

uint32_t g16_circuit_n_vars(const g16_circuit* c) { return c ? c->n_vars : 0; }
uint32_t g16_circuit_n_public(const g16_circuit* c) { return c ? c->n_public : 0; }
uint32_t g16_circuit_domain_size(const g16_circuit* c) { return c ? c->n : 0; }
uint64_t g16_circuit_device_bytes(const g16_circuit* c) { return c ? c->device_bytes : 0; }
int g16_circuit_window_tables(const g16_circuit* c) { return c && c->tables ? 1 : 0; }

int g16_plan_key(const g16_zkey_view* k, uint64_t free_bytes, g16_key_plan* out) {
    if (!k || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (k->domain_size < 2 || (k->domain_size & (k->domain_size - 1)) || (uint64_t)k->n_public + 1 > k->n_vars)
        return fail(G16_ERR_BACKEND, "malformed key shape");
    const LiveSetsHost live = live_sets(*k);
    return plan_key(*k, live.rows, free_bytes, out);
}

// ---- stages ----
int g16_compute_h(g16_circuit* c, const uint8_t* w, size_t n, g16_hpoly** out) {
    if (!c || !w || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    int rc = check_witness(c, n, w);
    if (rc) return rc;
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    auto h = std::make_unique<g16_hpoly>();
    h->owner = c;
    h->n = c->n;
    CK(g16::dev_malloc(&h->d_h, 32ull * c->n), "H allocation");
    if ((rc = upload_witness(g.ws, w, n)) || (rc = run_h(c, g.ws, g.ws->d_w, h->d_h))) {
        cudaFree(h->d_h);
        return rc;
    }
    CK(cudaStreamSynchronize(g.ws->stream), "stages 0-4");
    timer().collect();
    add_timings(c, g.ws, true, false, 0);
    *out = h.release();
    return G16_OK;
}

int g16_h_to_host(const g16_hpoly* h, uint8_t* out, size_t cap) {
    if (!h || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (cap < h->n) return fail(G16_ERR_INVALID_ARGUMENT, "buffer holds %zu of %u values", cap, h->n);
    CK(cudaSetDevice(h->owner->be->ordinal), "cudaSetDevice");
    CK(cudaMemcpy(out, h->d_h, 32ull * h->n, cudaMemcpyDeviceToHost), "H readback");
    return G16_OK;
}

void g16_hpoly_free(g16_hpoly* h) {
    if (!h) return;
    cudaFree(h->d_h);
    delete h;
}

int g16_msms(g16_circuit* c, const uint8_t* w, size_t n, const g16_hpoly* h, g16_msm_outputs* out) {
    if (!c || !w || !h || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (h->owner != c) return fail(G16_ERR_BACKEND, "H handle was computed by another circuit");
    int rc = check_witness(c, n, w);
    if (rc) return rc;
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    if ((rc = upload_witness(g.ws, w, n))) return rc;
    CK(cudaEventRecord(g.ws->ev[2], g.ws->stream), "event");
    MsmJac m;
    if ((rc = enqueue_witness_msms(c, g.ws, g.ws->d_w)) || (rc = enqueue_h_msm(c, g.ws, h->d_h)) ||
        (rc = enqueue_join(g.ws)) || (rc = collect_msms(c, g.ws, m)))
        return rc;
    add_timings(c, g.ws, false, true, 0);
    to_outputs(m, out);
    return G16_OK;
}

int g16_h_and_msms(g16_circuit* c, const uint8_t* w, size_t n, g16_msm_outputs* out) {
    if (!c || !w || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    int rc = check_witness(c, n, w);
    if (rc) return rc;
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    if ((rc = upload_witness(g.ws, w, n))) return rc;
    MsmJac m;
    if ((rc = run_proof(c, g.ws, g.ws->d_w, m))) return rc;
    add_timings(c, g.ws, true, true, 0);
    to_outputs(m, out);
    return G16_OK;
}

int g16_h_and_msms_from_rows(g16_circuit* c, const uint8_t* w, size_t n, const uint8_t* a_rows,
                             const uint8_t* b_rows, size_t rows, g16_msm_outputs* out) {
    if (!c || !w || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    int rc = check_witness(c, n, w);
    if (rc || (rc = check_rows(c, a_rows, b_rows, rows))) return rc;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    if ((rc = upload_witness(g.ws, w, n))) return rc;
    MsmJac m;
    if ((rc = run_rows_proof(c, g.ws, g.ws->d_w, a_rows, b_rows, rows, m))) return rc;
    add_timings(c, g.ws, true, true, 0);
    to_outputs(m, out);
    return G16_OK;
}

int g16_prove_with_blinders_from_rows(g16_circuit* c, const uint8_t* w, size_t n, const uint8_t* a_rows,
                                      const uint8_t* b_rows, size_t rows, const uint8_t* r_mont,
                                      const uint8_t* s_mont, g16_proof* out) {
    if (!c || !w || !r_mont || !s_mont || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    int rc = check_witness(c, n, w);
    if (rc || (rc = check_rows(c, a_rows, b_rows, rows))) return rc;
    uint64_t rr[4], ss[4];
    std::memcpy(rr, r_mont, 32);
    std::memcpy(ss, s_mont, 32);
    if (!g16::Fr::canonical(rr) || !g16::Fr::canonical(ss)) return fail(G16_ERR_INVALID_ARGUMENT, "r or s not below r");
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    if ((rc = upload_witness(g.ws, w, n))) return rc;
    g16::Fr r = g16::Fr::raw(rr), s = g16::Fr::raw(ss);
    auto terms = std::async(std::launch::async, [&] { return blinder_terms(c, r, s); });
    MsmJac m;
    rc = run_rows_proof(c, g.ws, g.ws->d_w, a_rows, b_rows, rows, m);
    BlinderTerms t = terms.get();
    if (rc) return rc;
    auto t0 = std::chrono::steady_clock::now();
    assemble(c, m, t, r, s, out);
    auto t1 = std::chrono::steady_clock::now();
    add_timings(c, g.ws, true, true, (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count());
    return G16_OK;
}

int g16_prove_with_blinders(g16_circuit* c, const uint8_t* w, size_t n, const uint8_t* r, const uint8_t* s,
                            g16_proof* out) {
    if (!c || !w || !r || !s || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    int rc = check_witness(c, n, w);
    if (rc) return rc;
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    if ((rc = upload_witness(g.ws, w, n))) return rc;
    return prove_on_device(c, g.ws, g.ws->d_w, r, s, out);
}

int g16_circuit_warm(g16_circuit* c, uint32_t count) {
    if (!c) return fail(G16_ERR_INVALID_ARGUMENT, "null circuit");
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    // hold up to `count` workspaces at once: idle ones, or new ones while the pool
    // and the device budget allow (never waiting, since they may all be held here)
    std::vector<std::unique_ptr<WsGuard>> held;
    {
        std::unique_lock<std::mutex> lk(c->mu);
        c->cv.wait(lk, [&] { return !c->tuning; });
        while (held.size() < count) {
            Workspace* ws = nullptr;
            if (!c->idle.empty()) {
                ws = c->idle.back();
                c->idle.pop_back();
            } else if (c->pool.size() < c->max_workspaces && c->be->vram_used + c->ws_estimate <= c->be->vram_limit) {
                auto w = std::make_unique<Workspace>();
                cudaError_t e = w->init(c->n_vars, c->n, win_slot(c));
                if (e != cudaSuccess) {
                    w->release();
                    cudaGetLastError();
                    break;
                }
                c->device_bytes += c->ws_estimate;
                c->be->vram_used += c->ws_estimate;
                ws = w.get();
                c->pool.push_back(std::move(w));
            } else {
                break;
            }
            held.push_back(std::make_unique<WsGuard>(c));
            held.back()->ws = ws;
        }
    }
    // a throwaway witness: the constant wire 1, every other wire 0; r = s = 1
    host_init();
    std::vector<uint8_t> w(32ull * c->n_vars, 0);
    std::memcpy(w.data(), FR_P.one.v, 32);
    const uint8_t* one = (const uint8_t*)FR_P.one.v;
    g16_proof p;
    for (int pass = 0; pass < 2; pass++)   // the first sizes the scratch, the second captures the graph
        for (auto& g : held) {
            int rc = upload_witness(g->ws, w.data(), c->n_vars);
            if (rc == G16_OK) rc = prove_on_device(c, g->ws, g->ws->d_w, one, one, &p);
            if (rc != G16_OK) return rc;
        }
    return G16_OK;
}

int g16_prove_with_blinders_device(g16_circuit* c, const void* d_w, size_t n, const uint8_t* r, const uint8_t* s,
                                   g16_proof* out) {
    if (!c || !d_w || !r || !s || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    int rc = check_witness(c, n, nullptr);
    if (rc) return rc;
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    WsGuard g(c);
    if ((rc = acquire(c, &g.ws))) return rc;
    return prove_on_device(c, g.ws, d_w, r, s, out);
}

int g16_prove(g16_circuit* c, const uint8_t* w, size_t n, g16_proof* out) {
    if (!c || !w || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    // Fr::rand: uniform in [0, r) by rejection on 254-bit draws
    uint8_t rs[2][32];
    for (auto& x : rs) {
        for (;;) {
            uint64_t v[4];
            size_t got = 0;
            while (got < sizeof v) {
                ssize_t k = getrandom((uint8_t*)v + got, sizeof v - got, 0);
                if (k <= 0) return fail(G16_ERR_BACKEND, "getrandom failed");
                got += (size_t)k;
            }
            v[3] &= (1ull << 62) - 1;
            if (!g16::Fr::canonical(v)) continue;
            if ((v[0] | v[1] | v[2] | v[3]) == 0) return fail(G16_ERR_BACKEND, "drew a zero blinder");
            g16::Fr m = g16::Fr::from_std(v);
            std::memcpy(x, m.x.v, 32);
            break;
        }
    }
    int rc = g16_prove_with_blinders(c, w, n, rs[0], rs[1], out);
    if (rc) return rc;
    auto t0 = std::chrono::steady_clock::now();
    rc = g16_circuit_verify(c, w + 32, c->n_public, out);
    uint64_t us = (uint64_t)std::chrono::duration_cast<std::chrono::microseconds>(
                      std::chrono::steady_clock::now() - t0).count();
    {
        std::lock_guard<std::mutex> g(c->mu);
        c->t.verify_us += us;
    }
    if (rc == G16_ERR_VERIFY || rc == G16_ERR_FORMAT) {
        std::string why = g_err;
        return fail(G16_ERR_SELF_VERIFY, "the proof did not verify against its own key: %s", why.c_str());
    }
    return rc;
}

static int verify_status(VerifyResult v, const std::string& why) {
    switch (v) {
        case VerifyResult::Ok: return G16_OK;
        case VerifyResult::PublicInputCount: return fail(G16_ERR_INVALID_ARGUMENT, "verify: %s", why.c_str());
        case VerifyResult::EmptyKey:
        case VerifyResult::UnsafeKey: return fail(G16_ERR_FORMAT, "verify: %s", why.c_str());
        default: return fail(G16_ERR_VERIFY, "verify: %s", why.c_str());
    }
}

int g16_verify(const uint8_t* alpha_g1, const uint8_t* beta_g2, const uint8_t* gamma_g2, const uint8_t* delta_g2,
               const uint8_t* ic, size_t n_ic, const uint8_t* pub, size_t n_public, const g16_proof* proof) {
    if (!alpha_g1 || !beta_g2 || !gamma_g2 || !delta_g2 || (n_ic && !ic) || (n_public && !pub) || !proof)
        return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    host_init();
    VerifyingKey vk;
    std::vector<G1A> pts(n_ic);
    if (!unpack(vk.alpha1, alpha_g1) || !unpack(vk.beta2, beta_g2) || !unpack(vk.gamma2, gamma_g2) ||
        !unpack(vk.delta2, delta_g2))
        return fail(G16_ERR_FORMAT, "verify: non-canonical verifying-key point");
    for (size_t i = 0; i < n_ic; i++)
        if (!unpack(pts[i], ic + 64 * i)) return fail(G16_ERR_FORMAT, "verify: non-canonical IC point %zu", i);
    vk.ic = pts.data();
    vk.n_ic = n_ic;
    G1A a, c;
    G2A b;
    if (!unpack(a, proof->a) || !unpack(b, proof->b) || !unpack(c, proof->c))
        return fail(G16_ERR_VERIFY, "verify: a proof coordinate is not below q");
    for (size_t i = 0; i < n_public; i++) {
        uint64_t v[4];
        std::memcpy(v, pub + 32 * i, 32);
        if (!g16::Fr::canonical(v)) return fail(G16_ERR_INVALID_ARGUMENT, "verify: public input %zu is not below r", i);
    }
    std::string why;
    return verify_status(groth16_verify(vk, pub, n_public, a, b, c, &why), why);
}

int g16_circuit_verify(const g16_circuit* c, const uint8_t* pub, size_t n_public, const g16_proof* proof) {
    if (!c || (n_public && !pub) || !proof) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (c->ic.empty()) return fail(G16_ERR_FORMAT, "verify: the key carried no IC section");
    uint8_t alpha[64], beta[128], gamma[128], delta[128];
    pack(alpha, c->alpha1);
    pack(beta, c->beta2);
    pack(gamma, c->gamma2);
    pack(delta, c->delta2);
    std::vector<uint8_t> ic(64 * c->ic.size());
    for (size_t i = 0; i < c->ic.size(); i++) pack(ic.data() + 64 * i, c->ic[i]);
    return g16_verify(alpha, beta, gamma, delta, ic.data(), c->ic.size(), pub, n_public, proof);
}

int g16_pairing_check(const uint8_t* g1, const uint8_t* g2, size_t n) {
    if (n && (!g1 || !g2)) return -fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    host_init();
    std::vector<G1A> p(n);
    std::vector<G2A> q(n);
    for (size_t i = 0; i < n; i++)
        if (!unpack(p[i], g1 + 64 * i) || !unpack(q[i], g2 + 128 * i) || !on_curve(p[i]) || !on_curve(q[i]))
            return -fail(G16_ERR_INVALID_ARGUMENT, "pairing input %zu is not a canonical curve point", i);
    return pairing_product_is_one(p.data(), q.data(), n) ? 1 : 0;
}

int g16_stage_timings_get(const g16_circuit* c, g16_stage_timings* out) {
    if (!c || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    *out = c->t;
    return G16_OK;
}

// Several proofs in flight at once: `lanes` host threads each take the next job
// and prove it on a workspace of its circuit, so the jobs' kernels, copies and
// host-side assembly overlap.  Each result is the same as a single call's.
int g16_prove_batch_timed(g16_backend* b, size_t count, g16_circuit* const* circuits,
                          const uint8_t* const* witnesses, const size_t* lens, const uint8_t* r, const uint8_t* s,
                          g16_proof* out, double* done_ms);

int g16_batch_reserve(g16_backend* b, size_t count, g16_circuit* const* circuits) {
    if (!b || (count && !circuits)) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    bool all_tables = true;
    for (size_t i = 0; i < count; i++) {
        if (!circuits[i]) return fail(G16_ERR_INVALID_ARGUMENT, "null circuit %zu", i);
        if (circuits[i]->be != b) return fail(G16_ERR_INVALID_ARGUMENT, "circuit %zu belongs to another backend", i);
        if (int rc_g = gather_ok(circuits[i])) return rc_g;
        all_tables &= circuits[i]->tables;
    }
    if (int rc_dev = device_usable(b)) return rc_dev;
    // the same choice as g16_prove_batch_timed: only the engine path has buffers to size
    const char* eng = std::getenv("G16_BATCH_ENGINE");
    if (!count || b->constant_work || !all_tables || (eng && std::strcmp(eng, "0") == 0)) return G16_OK;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    return reserve_batch_engines(b, circuits, count);
}

int g16_prove_batch(g16_backend* b, size_t count, g16_circuit* const* circuits, const uint8_t* const* witnesses,
                    const size_t* lens, const uint8_t* r, const uint8_t* s, g16_proof* out) {
    return g16_prove_batch_timed(b, count, circuits, witnesses, lens, r, s, out, nullptr);
}

int g16_prove_batch_timed(g16_backend* b, size_t count, g16_circuit* const* circuits,
                          const uint8_t* const* witnesses, const size_t* lens, const uint8_t* r, const uint8_t* s,
                          g16_proof* out, double* done_ms) {
    const auto t_start = std::chrono::steady_clock::now();
    if (!b || (count && (!circuits || !witnesses || !lens || !r || !s || !out)))
        return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t i = 0; i < count; i++) {
        if (!circuits[i] || !witnesses[i]) return fail(G16_ERR_INVALID_ARGUMENT, "null job %zu", i);
        if (circuits[i]->be != b) return fail(G16_ERR_INVALID_ARGUMENT, "job %zu belongs to another backend", i);
        if (int rc_g = gather_ok(circuits[i])) return rc_g;
        int rc = check_witness(circuits[i], lens[i], witnesses[i]);
        if (rc) return rc;
    }
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    // one launch per stage for every job; host lanes only for constant-work MSMs, when
    // G16_BATCH_ENGINE=0, or when the batch's working set does not fit the device budget
    const char* eng = std::getenv("G16_BATCH_ENGINE");
    bool all_tables = true;   // the engine reads window tables; compact keys take the lanes
    for (size_t i = 0; i < count; i++) all_tables &= circuits[i]->tables;
    if (!b->constant_work && all_tables && !(eng && std::strcmp(eng, "0") == 0)) {
        int rc = prove_batch_engine(b, count, circuits, witnesses, lens, r, s, out, done_ms);
        if (rc != G16_ERR_DEVICE_MEMORY) return rc;
    }
    size_t lanes = 8;
    if (const char* e = std::getenv("G16_BATCH_LANES")) lanes = (size_t)std::max(1, std::atoi(e));
    lanes = std::min(lanes, count);
    std::atomic<size_t> next{0};
    std::vector<int> rcs(count, G16_OK);
    std::vector<std::string> errs(count);
    auto work = [&] {
        cudaSetDevice(b->ordinal);
        for (size_t i; (i = next.fetch_add(1)) < count;) {
            rcs[i] = g16_prove_with_blinders(circuits[i], witnesses[i], lens[i], r + 32 * i, s + 32 * i, out + i);
            if (rcs[i]) errs[i] = g_err;
            if (done_ms)
                done_ms[i] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start)
                                 .count();
        }
    };
    std::vector<std::thread> pool;
    for (size_t t = 1; t < lanes; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    for (size_t i = 0; i < count; i++)
        if (rcs[i]) {
            set_error("job %zu: %s", i, errs[i].c_str());
            return rcs[i];
        }
    return G16_OK;
}


// ---- primitives ----
static int grow_dev(void*& p, size_t& cap, size_t need) {
    if (need <= cap && p) return G16_OK;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    CK(g16::dev_malloc(&p, need ? need : 32), "scratch allocation");
    cap = need;
    return G16_OK;
}

static int msm_device_impl(g16_backend* b, const void* d_bases, const void* d_scalars, size_t n, int form, bool g2,
                           uint8_t* out) {
    if (form != G16_SCALARS_STANDARD && form != G16_SCALARS_MONTGOMERY)
        return fail(G16_ERR_INVALID_ARGUMENT, "unknown scalar form %d", form);
    if (n == 0) {
        std::memset(out, 0, g2 ? 128 : 64);
        return G16_OK;
    }
    cudaStream_t st = b->stream;
    CK(msm_sort(b->sort, d_scalars, n, form == G16_SCALARS_MONTGOMERY, 0, st, false, b->constant_work), "MSM sort");
    if (g2) CK(msm_accumulate_g2(b->sort, b->acc, d_bases, 0, (uint32_t)n, st), "MSM accumulate");
    else CK(msm_accumulate_g1(b->sort, b->acc, d_bases, 0, (uint32_t)n, st), "MSM accumulate");
    const size_t bytes = b->acc.result_bytes(g2 ? XYZZ_G2_BYTES : XYZZ_G1_BYTES);
    if (bytes > b->cap_pinned) {
        cudaFreeHost(b->h_pinned);
        b->h_pinned = nullptr;
        b->cap_pinned = 0;
        CK(cudaMallocHost((void**)&b->h_pinned, bytes), "pinned buffer");
        b->cap_pinned = bytes;
    }
    CK(cudaMemcpyAsync(b->h_pinned, b->acc.d_windows, bytes, cudaMemcpyDeviceToHost, st), "window readback");
    if (timer().enabled) {
        // [0] mixed additions, [1] sorted entries (for the scatter's bytes)
        if (!b->h_work) CK(cudaMallocHost((void**)&b->h_work, 2 * sizeof(unsigned long long)), "pinned buffer");
        b->h_work[1] = 0;
        CK(cudaMemcpyAsync(b->h_work, b->acc.d_work, 8, cudaMemcpyDeviceToHost, st), "work readback");
        CK(cudaMemcpyAsync(&b->h_work[1], b->sort.d_total, 4, cudaMemcpyDeviceToHost, st), "work readback");
    }
    CK(cudaStreamSynchronize(st), "MSM");
    timer().collect();
    if (timer().enabled) {
        timer().add_units(g2 ? "msm_accumulate_g2" : "msm_accumulate_g1", (double)b->h_work[0]);
        timer().add_bytes("msm_scatter", 32.0 * n + 4.0 * (double)b->h_work[1]);   // scalars in, entries out
    }
    if (g2) pack(out, msm_combine_g2(b->h_pinned, b->acc.plan, b->sort.c).to_affine());
    else pack(out, msm_combine_g1(b->h_pinned, b->acc.plan, b->sort.c).to_affine());
    return G16_OK;
}

static int msm_host_impl(g16_backend* b, const uint8_t* bases, const uint8_t* scalars, size_t n, int form, bool g2,
                         uint8_t* out) {
    if (!b || (n && (!bases || !scalars)) || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(b->mu);
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    if (n == 0) {
        std::memset(out, 0, g2 ? 128 : 64);
        return G16_OK;
    }
    size_t bb = n * (g2 ? 128 : 64);
    int rc;
    if ((rc = grow_dev(b->d_in, b->cap_in, bb))) return rc;
    if ((rc = grow_dev(b->d_in2, b->cap_in2, n * 32))) return rc;
    CK(cudaMemcpyAsync(b->d_in, bases, bb, cudaMemcpyHostToDevice, b->stream), "bases upload");
    CK(cudaMemcpyAsync(b->d_in2, scalars, n * 32, cudaMemcpyHostToDevice, b->stream), "scalars upload");
    return msm_device_impl(b, b->d_in, b->d_in2, n, form, g2, out);
}

int g16_msm_g1(g16_backend* b, const uint8_t* bases, const uint8_t* scalars, size_t n, int form, uint8_t* out64) {
    return msm_host_impl(b, bases, scalars, n, form, false, out64);
}
int g16_msm_g2(g16_backend* b, const uint8_t* bases, const uint8_t* scalars, size_t n, int form, uint8_t* out128) {
    return msm_host_impl(b, bases, scalars, n, form, true, out128);
}
int g16_msm_g1_device(g16_backend* b, const void* d_bases, const void* d_scalars, size_t n, int form, uint8_t* out64) {
    if (!b || !out64) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(b->mu);
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    return msm_device_impl(b, d_bases, d_scalars, n, form, false, out64);
}
int g16_msm_g2_device(g16_backend* b, const void* d_bases, const void* d_scalars, size_t n, int form, uint8_t* out128) {
    if (!b || !out128) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(b->mu);
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    return msm_device_impl(b, d_bases, d_scalars, n, form, true, out128);
}

static int ntt_device_impl(g16_backend* b, int mode, uint32_t log_n, void* d, const uint8_t* shift_mont) {
    if (log_n < 1 || log_n > 27) return fail(G16_ERR_INVALID_ARGUMENT, "log_n %u outside [1, 27]", log_n);
    if (b->ntt.size() <= log_n) b->ntt.resize(log_n + 1);
    if (!b->ntt[log_n]) b->ntt[log_n] = std::make_unique<NttTables>();
    NttTables& t = *b->ntt[log_n];
    CK(ntt_tables(t, (int)log_n, b->stream), "NTT tables");
    cudaStream_t st = b->stream;
    size_t n = (size_t)1 << log_n;
    uint64_t shift[4];
    if (shift_mont) std::memcpy(shift, shift_mont, 32);
    else std::memcpy(shift, t.shift, 32);
    switch (mode) {
        case G16_NTT_FORWARD: CK(ntt_forward(t, d, st), "NTT"); break;
        case G16_NTT_INVERSE: CK(ntt_inverse(t, d, st), "iNTT"); break;
        case G16_NTT_INTT_COSET_NTT:
            if (shift_mont && std::memcmp(shift_mont, t.shift, 32) != 0)
                return fail(G16_ERR_INVALID_ARGUMENT, "intt_coset_ntt runs on the proving coset only");
            CK(ntt_intt_coset_ntt(t, d, st), "iNTT-coset-NTT");
            break;
        case G16_NTT_COSET_FORWARD:
            CK(ntt_distribute_powers(d, n, shift, st), "distribute powers");
            CK(ntt_forward(t, d, st), "NTT");
            break;
        case G16_NTT_COSET_INVERSE: {
            g16::Fr si = g16::Fr::raw(shift).inv();
            CK(ntt_inverse(t, d, st), "iNTT");
            CK(ntt_distribute_powers(d, n, si.x.v, st), "distribute powers");
            break;
        }
        default: return fail(G16_ERR_INVALID_ARGUMENT, "unknown NTT mode %d", mode);
    }
    return G16_OK;
}

int g16_ntt(g16_backend* b, int mode, uint32_t log_n, uint8_t* data, const uint8_t* shift_mont) {
    if (!b || !data) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(b->mu);
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    if (log_n < 1 || log_n > 27) return fail(G16_ERR_INVALID_ARGUMENT, "log_n %u outside [1, 27]", log_n);
    size_t bytes = ((size_t)1 << log_n) * 32;
    int rc;
    if ((rc = grow_dev(b->d_in, b->cap_in, bytes))) return rc;
    CK(cudaMemcpyAsync(b->d_in, data, bytes, cudaMemcpyHostToDevice, b->stream), "NTT upload");
    if ((rc = ntt_device_impl(b, mode, log_n, b->d_in, shift_mont))) return rc;
    CK(cudaMemcpyAsync(data, b->d_in, bytes, cudaMemcpyDeviceToHost, b->stream), "NTT readback");
    CK(cudaStreamSynchronize(b->stream), "NTT");
    timer().collect();
    return G16_OK;
}

int g16_ntt_device(g16_backend* b, int mode, uint32_t log_n, void* d, const uint8_t* shift_mont) {
    if (!b || !d) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(b->mu);
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    int rc = ntt_device_impl(b, mode, log_n, d, shift_mont);
    if (rc) return rc;
    CK(cudaStreamSynchronize(b->stream), "NTT");
    timer().collect();
    return G16_OK;
}

// ---- timing ----
void g16_kernel_timing_enable(int on) { timer().enabled = on != 0; }
void g16_kernel_timing_reset(void) { timer().reset(); }
size_t g16_kernel_timing_report(char* buf, size_t len) {
    timer().collect();
    std::string s;
    {
        std::lock_guard<std::mutex> g(timer().mu);
        for (auto& kv : timer().totals) {
            char line[256];
            auto u = timer().units.find(kv.first);
            auto by = timer().bytes.find(kv.first);
            snprintf(line, sizeof line, "%s %.6f %ld %.0f %.0f\n", kv.first.c_str(), kv.second.first, kv.second.second,
                     u == timer().units.end() ? 0.0 : u->second, by == timer().bytes.end() ? 0.0 : by->second);
            s += line;
        }
    }
    if (buf && len) {
        size_t k = s.size() < len - 1 ? s.size() : len - 1;
        std::memcpy(buf, s.data(), k);
        buf[k] = 0;
    }
    return s.size();
}

int g16_tuning_get(const g16_circuit* c, g16_tuning* out) {
    if (!c || !out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    *out = current_tuning(c);
    return G16_OK;
}

int g16_tuning_set(g16_circuit* c, const g16_tuning* t) {
    if (!c || !t) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    TuningLock lock(c);
    int rc = lock.take();
    if (rc) return rc;
    return apply_tuning(c, lock.ws, *t);
}

int g16_autotune(g16_circuit* c, const uint8_t* w, size_t n, int concurrency, g16_tuning* out) {
    if (!c || !w) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (concurrency < 1 || concurrency > 8) return fail(G16_ERR_INVALID_ARGUMENT, "concurrency must be 1..8");
    int rc = check_witness(c, n, w);
    if (rc) return rc;
    if (int rc_g = gather_ok(c)) return rc_g;
    if (int rc_dev = device_usable(c->be)) return rc_dev;
    CK(cudaSetDevice(c->be->ordinal), "cudaSetDevice");
    TuningLock lock(c);
    if ((rc = lock.take(concurrency))) return rc;
    Workspace* ws = lock.ws;
    const bool serial = c->serial;
    for (Workspace* x : lock.all)
        if ((rc = upload_witness(x, w, n))) return rc;
    const int reps = 3;
    const bool together = lock.all.size() > 1;
    // the objective: one proof alone, or stages 0-9 of every held workspace in flight together
    auto whole = [&] {
        return together ? time_concurrent(c, lock.all, reps)
                        : time_on_stream(ws, reps, [&] { return enqueue_proof(c, ws, ws->d_w); });
    };
    const g16_tuning model = current_tuning(c);
    double model_ms = whole();
    if (model_ms < 0) return G16_ERR_DEVICE;
    // 1. NTT tiling: gather + NTT chain alone (or the concurrent objective)
    {
        NttTiling best = c->ntt.tiling;
        double best_t = -1;
        for (uint32_t tl : {10u, 11u, 12u})
            for (uint32_t ll : {1u, 2u, 3u}) {
                if ((uint32_t)c->log_n <= 10 && !(tl == best.tile_log && ll == best.outer_log_l)) continue;
                c->ntt.tiling = {tl, ll};
                double t = together ? whole()
                                    : time_on_stream(ws, reps, [&] { return run_h(c, ws, ws->d_w, ws->d_hpoly); });
                if (t < 0) return G16_ERR_DEVICE;
                if (best_t < 0 || t < best_t) {
                    best_t = t;
                    best = c->ntt.tiling;
                }
            }
        c->ntt.tiling = best;
    }
    // 2. H MSM window (H from the tiling just chosen is in d_hpoly)
    {
        int best = c->c_h;
        rc = climb_window(
            c->c_h, [&](int b) { return b == c->c_h ? G16_OK : build_h_table(c, b, ws->stream); },
            [&] {
                return together ? whole()
                                : time_on_stream(ws, reps, [&] { return enqueue_h_msm(c, ws, ws->d_hpoly); });
            },
            &best);
        if (rc) return rc;
    }
    // 3. witness MSM window: the four MSMs serialised on one stream (or the concurrent objective)
    {
        c->serial = !together;
        int best = c->c_w;
        rc = climb_window(
            c->c_w, [&](int b) { return b == c->c_w ? G16_OK : build_witness_tables(c, b, ws->stream); },
            [&] {
                if (together) return whole();
                return time_on_stream(ws, reps, [&] {
                    int r = enqueue_witness_msms(c, ws, ws->d_w);
                    return r ? r : enqueue_join(ws);
                });
            },
            &best);
        c->serial = serial;
        if (rc) return rc;
    }
    // 4. keep the tuned set only if the objective got better
    double tuned_ms = whole();
    if (tuned_ms < 0) return G16_ERR_DEVICE;
    if (tuned_ms > model_ms) {
        if ((rc = apply_tuning(c, ws, model))) return rc;
        tuned_ms = model_ms;
    }
    c->tuned.model_ms = model_ms;
    c->tuned.tuned_ms = tuned_ms;
    if (out) *out = current_tuning(c);
    return G16_OK;
}

uint64_t g16_launch_count(void) { return timer().launches.load(); }
uint64_t g16_device_alloc_count(void) { return timer().device_allocs.load(); }

uint64_t g16_circuit_readback_bytes(const g16_circuit* c) { return c ? c->readback_bytes : 0; }

int g16_circuit_set_serial(g16_circuit* c, int serial) {
    if (!c) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(c->mu);
    c->serial = serial != 0;
    return G16_OK;
}

int g16_imad_peak(g16_backend* b, double* imad_per_s) {
    if (!b || !imad_per_s) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> g(b->mu);
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->ordinal), "attribute");
    unsigned blocks = (unsigned)sms * 8, threads = 256;
    uint32_t iters = 4096;
    uint32_t* d = nullptr;
    CK(g16::dev_malloc(&d, (size_t)blocks * threads * 4), "probe buffer");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0, b->stream);
        {
            TimedLaunch tl("imad_peak", b->stream);
            g16d::k_imad_peak<<<blocks, threads, 0, b->stream>>>(d, iters, (uint32_t)rep);
        }
        cudaEventRecord(e1, b->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
            cudaFree(d);
            return cuda_fail(e, "IMAD probe");
        }
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep && ms < best) best = ms;   // first run is warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    // 8 chains x (mad.lo + mad.hi) x 4 unrolled per iteration
    double ops = (double)blocks * threads * iters * 64.0;
    *imad_per_s = ops / (best * 1e-3);
    return G16_OK;
}

// ---- device memory helpers ----
int g16_device_alloc(g16_backend* b, size_t bytes, void** d_out) {
    if (!b || !d_out) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    CK(g16::dev_malloc(d_out, bytes ? bytes : 32), "device allocation");
    return G16_OK;
}
int g16_device_free(g16_backend* b, void* d) {
    if (!b) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    CK(cudaFree(d), "device free");
    return G16_OK;
}
int g16_device_upload(g16_backend* b, void* d_dst, const void* src, size_t bytes) {
    if (!b || !d_dst || !src) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    // complete on return: a plain cudaMemcpy from pageable memory may return
    // before its DMA lands, and kernels on non-blocking streams would not wait for it
    CK(cudaMemcpyAsync(d_dst, src, bytes, cudaMemcpyHostToDevice, b->stream), "upload");
    CK(cudaStreamSynchronize(b->stream), "upload");
    return G16_OK;
}
int g16_device_sync(g16_backend* b) {
    if (!b) return fail(G16_ERR_INVALID_ARGUMENT, "null argument");
    if (int rc_dev = device_usable(b)) return rc_dev;
    CK(cudaSetDevice(b->ordinal), "cudaSetDevice");
    CK(cudaDeviceSynchronize(), "device synchronize");
    return G16_OK;
}

}  // extern "C"
