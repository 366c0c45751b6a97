/*
 * g16b200: B200-native Groth16 / BN254 proving hot path behind a C ABI.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns a status code (G16_OK = 0).  The text of the last error on the
 * calling thread is available from g16_last_error().  No entry point panics,
 * aborts or throws across the boundary.
 *
 * Byte layouts (identical to the reference's crates/gpu-layout packing,
 * crates/gpu-layout/src/lib.rs:30-200, 351):
 *   Fr / Fq element   32 bytes, 4 x u64 (= 8 x u32) little-endian limbs,
 *                     Montgomery form with R = 2^256 -- the in-memory bits of
 *                     arkworks' Fp, i.e. a Rust &[Fr] can be passed as is;
 *   scalar, standard  32 bytes little-endian integer in [0, r);
 *   G1 affine         64 bytes: x, y (Montgomery Fq);
 *   G2 affine         128 bytes: x.c0, x.c1, y.c0, y.c1;
 *   point at infinity all-zero bytes.
 * Host buffers are owned by the caller and only read (or written, for
 * outputs) during the call.  Handles are owned by the library and released
 * by their *_free function.
 */
#ifndef G16B200_H
#define G16B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, mirroring ProveError (crates/groth16/src/lib.rs:81-154) and
 * ZkeyError (crates/formats/src/lib.rs). */
enum {
    G16_OK = 0,
    G16_ERR_WITNESS_LENGTH = 1,   /* ProveError::WitnessLength */
    G16_ERR_CONSTANT_WIRE = 2,    /* ProveError::ConstantWire: w[0] != 1 */
    G16_ERR_BACKEND = 3,          /* ProveError::Backend: malformed key or shape */
    G16_ERR_DEVICE = 4,           /* ProveError::Device: a CUDA call failed */
    G16_ERR_DEVICE_MEMORY = 5,    /* ProveError::DeviceMemory: refused before allocating */
    G16_ERR_SELF_VERIFY = 6,      /* ProveError::SelfVerify: g16_prove's proof failed its check */
    G16_ERR_TIMEOUT = 7,          /* reserved for a bounded device wait that gives up; no
                                     entry point waits on the device that way, so none returns it */
    G16_ERR_INVALID_ARGUMENT = 8, /* null pointer, bad size, bad enum */
    G16_ERR_FORMAT = 9,           /* ZkeyError: malformed .zkey / .wtns bytes */
    G16_ERR_VERIFY = 10           /* verify::VerifyError: the proof does not verify */
};

/* Scalar encodings accepted by the MSM entry points. */
enum { G16_SCALARS_STANDARD = 0, G16_SCALARS_MONTGOMERY = 1 };

/* NTT modes (crates/ntt/src/lib.rs:415-584). */
enum {
    G16_NTT_FORWARD = 0,         /* CpuNtt::ntt(.., Forward): natural in/out */
    G16_NTT_INVERSE = 1,         /* CpuNtt::ntt(.., Inverse): includes 1/n */
    G16_NTT_INTT_COSET_NTT = 2,  /* CpuNtt::intt_coset_ntt with the proving coset shift */
    G16_NTT_COSET_FORWARD = 3,   /* distribute_powers(shift) then forward */
    G16_NTT_COSET_INVERSE = 4    /* inverse then distribute_powers(1/shift) */
};

typedef struct g16_backend g16_backend;   /* CudaBackend (crates/cuda/src/backend.rs:94-232) */
typedef struct g16_circuit g16_circuit;   /* CudaCircuit: PreparedCircuit (crates/groth16/src/lib.rs:371-455) */
typedef struct g16_hpoly g16_hpoly;       /* HPoly::Device (crates/groth16/src/lib.rs:207-308) */
typedef struct g16_zkey g16_zkey;         /* ProvingKey (crates/formats/src/lib.rs:35-65) */

/* StageTimings (crates/groth16/src/lib.rs:322-338), microseconds, accumulated. */
typedef struct {
    uint64_t gather_us, ntt_us, pointwise_us, msm_us, assemble_us, verify_us;
} g16_stage_timings;

/* Proof (crates/groth16/src/lib.rs:187-192), affine packed. */
typedef struct {
    uint8_t a[64];
    uint8_t b[128];
    uint8_t c[64];
} g16_proof;

/* MsmOutputs (crates/groth16/src/lib.rs:311-318), affine packed. */
typedef struct {
    uint8_t a_g1[64];
    uint8_t b_g2[128];
    uint8_t b_g1[64];
    uint8_t l_g1[64];
    uint8_t h_g1[64];
} g16_msm_outputs;

/* A parsed proving key, field by field (ProvingKey, crates/formats/src/lib.rs:35-65,
 * section 4 in CSR form with interned values as in Coefficients, :140-223). */
typedef struct {
    uint32_t n_vars, n_public, domain_size;
    const uint8_t *alpha_g1, *beta_g1, *beta_g2, *gamma_g2, *delta_g1, *delta_g2;
    const uint8_t *ic;            /* (n_public + 1) G1 */
    const uint32_t *row_ptr[2];   /* [A, B], domain_size + 1 each */
    const uint32_t *signal[2];    /* nnz[m] each, < n_vars */
    const uint32_t *value_id[2];  /* nnz[m] each, < n_values */
    uint32_t nnz[2];
    const uint8_t *values;        /* n_values Fr, Montgomery */
    uint32_t n_values;
    const uint8_t *a_query;       /* n_vars G1 (section 5) */
    const uint8_t *b_g1_query;    /* n_vars G1 (section 6) */
    const uint8_t *b_g2_query;    /* n_vars G2 (section 7) */
    const uint8_t *l_query;       /* n_vars - n_public - 1 G1 (section 8) */
    const uint8_t *h_query;       /* domain_size G1 (section 9), or domain_size - 1 for the gnark basis */
    uint32_t h_basis;             /* G16_H_SNARKJS or G16_H_GNARK (HBasis, crates/formats/src/lib.rs:60-90) */
} g16_zkey_view;

/* H bases of a key (HBasis): snarkjs' zkey section 9, the Lagrange bases of the
 * odd coset (domain_size of them; H is taken on the coset as it is), or gnark's
 * pk.G1.Z, [tau^bitrev(j) t(tau) / delta] for j < domain_size - 1 (H's
 * coefficients in bit-reversed order, the MSM result times -1/2).  A gnark key
 * has no constraint matrices (row_ptr, signal, value_id and values are NULL,
 * nnz 0) and proves only from A.w and B.w rows. */
enum { G16_H_SNARKJS = 0, G16_H_GNARK = 1 };

/* ---------------- errors ---------------- */
/* Copies the calling thread's last error text into buf (NUL-terminated);
 * returns its full length. */
size_t g16_last_error(char *buf, size_t len);

/* ---------------- backend (CudaBackend::new, backend.rs:137-190) ---------------- */
/* Opens CUDA device `ordinal`.  vram_limit caps this backend's device
 * allocations in bytes (0 = the device's free memory).  Fails with
 * G16_ERR_DEVICE when no CUDA device is present: there is no CPU fallback. */
int g16_backend_open(int ordinal, uint64_t vram_limit, g16_backend **out);
void g16_backend_free(g16_backend *b);

/* ---------------- device faults (crates/cuda/src/context.rs:134-215) ----------------
 * A CUDA status is a device fault when the device failed rather than the call
 * being one the driver rejects every time (out of memory, ECC, a kernel
 * exception, the watchdog, MPS, an unknown internal error), and sticky when
 * the runtime documents it as leaving the context unusable ("any further CUDA
 * work will return the same error": the kernel exceptions, the watchdog, a
 * contained hardware error).  A sticky fault met by any entry point marks the
 * device for the rest of the process: from then on every entry point that
 * would use it returns G16_ERR_DEVICE with that reason, without a CUDA call,
 * and so does g16_backend_open on that device.  Out of memory stays
 * G16_ERR_DEVICE_MEMORY; every other CUDA failure is G16_ERR_DEVICE. */
enum { G16_FAULT_DEVICE = 1, G16_FAULT_STICKY = 2 };
/* The classes of a cudaError_t value: 0, G16_FAULT_DEVICE, or
 * G16_FAULT_DEVICE | G16_FAULT_STICKY.  Pure; needs no device. */
int g16_cuda_error_class(int cuda_error);
/* The sticky cudaError_t value that put this backend out of use (its device's
 * in this process, or one injected below), or 0. */
int g16_backend_fault(const g16_backend *b);
/* Fault injection for tests, on the host: the next entry point on this backend
 * that would use the device (prepare, prove, batch, MSM, NTT, tuning) fails as
 * if its first CUDA call had returned cuda_error, and does no device work.  A
 * sticky value puts this backend alone out of use (a real sticky fault takes
 * the device for the process).  0 cancels a pending injection. */
int g16_backend_inject_fault(g16_backend *b, int cuda_error);
const char *g16_backend_name(const g16_backend *b);   /* "cuda-b200" */
uint64_t g16_backend_vram_used(const g16_backend *b);
/* CudaBackend::constant_work (crates/cuda/src/backend.rs:100-118; the CPU
 * MSM's Work::Constant, crates/msm/src/lib.rs:206-220): every MSM this backend
 * runs afterwards (proofs, batches, servers, g16_msm_*) sends every window of
 * every scalar through the buckets, zero digits into a bucket no reduction
 * reads, so the sorted-entry count, launch sizes and additions follow the key
 * and not the witness.  Results are unchanged.  Not for
 * g16_msm_g1_device_noalloc. */
int g16_backend_set_constant_work(g16_backend *b, int on);

/* ---------------- .zkey / .wtns (crates/formats) ---------------- */
/* ProvingKey::load (formats/src/lib.rs:430-505).  check_points != 0 also runs
 * the on-curve check of every query point (load vs load_unchecked). */
int g16_zkey_parse(const uint8_t *bytes, size_t len, int check_points, g16_zkey **out);
/* A gnark v0.14 Groth16 BN254 key (crates/gnark/src/pk.rs, vk.rs): the proving
 * key's WriteDump bytes and the verifying key's WriteTo / WriteRawTo bytes,
 * checked against each other (alpha, beta, delta; one K point per public
 * wire), every point on its curve, no BSB22 commitments.  The key gets the
 * gnark H basis; its view serves g16_prepare like a .zkey's. */
int g16_gnark_key_parse(const uint8_t *pk_dump, size_t pk_len, const uint8_t *vk, size_t vk_len, g16_zkey **out);
/* A gnark witness dump (marker, then W, A.w and B.w as dumped Montgomery Fr
 * slices; crates/gnark/src/witness.rs).  Pass NULL outputs to learn the
 * counts: *n_w wires, *n_rows rows of A.w and of B.w. */
int g16_gnark_witness_parse(const uint8_t *bytes, size_t len, uint8_t *w_mont, size_t w_cap, uint8_t *aw_mont,
                            uint8_t *bw_mont, size_t rows_cap, size_t *n_w, size_t *n_rows);
int g16_zkey_view_get(const g16_zkey *k, g16_zkey_view *out);
void g16_zkey_free(g16_zkey *k);
/* Witness::load (formats/src/wtns.rs:17-40): values out in Montgomery form.
 * Pass out = NULL to learn the count. */
int g16_wtns_parse(const uint8_t *bytes, size_t len, uint8_t *out_mont, size_t cap, size_t *n_out);
/* .wtns writer (plain little-endian values), for tooling. out = NULL sizes. */
int g16_wtns_write(const uint8_t *w_mont, size_t n, uint8_t *out, size_t cap, size_t *len_out);

/* ---------------- circuits (Backend::prepare, backend.rs:325-457) ---------------- */
/* How a key is held on the device.  With window tables (the default) each
 * witness and H MSM reads bases 2^(c w) P_i laid out per window, so all
 * windows share one bucket set: about ten times the key's bases in memory.  A
 * compact key holds the plain bases only and runs one bucket set per window
 * with a Horner step on the host: slower, a tenth of the memory, the same
 * proofs.  This replaces the reference's runs of MSMs that do not fit VRAM
 * (resident_schedule / fit_run, crates/cuda/src/msm.rs:966,1117). */
typedef struct {
    int window_tables;             /* 1 window tables, 0 compact key */
    int msm_window_bits_witness;   /* c of the A, B1, L, B2 MSMs */
    int msm_window_bits_h;         /* c of the H MSM */
    uint64_t key_bytes;            /* device bytes of the prepared key */
    uint64_t workspace_bytes;      /* device bytes of one proof in flight */
} g16_key_plan;
/* The plan g16_prepare follows with free_bytes of device memory: window tables
 * when the key, its tables and one workspace fit; else the compact key when it
 * and one workspace fit (also whenever the environment sets
 * G16_CUDA_WINDOW_TABLES=0); else G16_ERR_DEVICE_MEMORY.  Host only. */
int g16_plan_key(const g16_zkey_view *key, uint64_t free_bytes, g16_key_plan *out);
/* Prepares a key on the device, refused with G16_ERR_DEVICE_MEMORY before any
 * allocation when g16_plan_key finds no plan within the backend's budget.
 * Batched submissions that include a compact key run it on host lanes. */
int g16_prepare(g16_backend *b, const g16_zkey_view *key, g16_circuit **out);
/* 1 when the circuit holds window tables, 0 for a compact key. */
int g16_circuit_window_tables(const g16_circuit *c);
void g16_circuit_free(g16_circuit *c);
uint32_t g16_circuit_n_vars(const g16_circuit *c);
uint32_t g16_circuit_n_public(const g16_circuit *c);
uint32_t g16_circuit_domain_size(const g16_circuit *c);
uint64_t g16_circuit_device_bytes(const g16_circuit *c);

/* PreparedCircuit::compute_h (stages 0-4; lib.rs:397-400, cuda stages.rs:929).
 * witness: n Fr in Montgomery form (a &[Fr]). */
int g16_compute_h(g16_circuit *c, const uint8_t *witness_mont, size_t n, g16_hpoly **out);
/* PreparedCircuit::h_to_host: n = domain_size Fr, Montgomery. */
int g16_h_to_host(const g16_hpoly *h, uint8_t *out_mont, size_t cap);
void g16_hpoly_free(g16_hpoly *h);
/* PreparedCircuit::msms (stages 5-9; lib.rs:401-412). */
int g16_msms(g16_circuit *c, const uint8_t *witness_mont, size_t n, const g16_hpoly *h, g16_msm_outputs *out);
/* PreparedCircuit::h_and_msms (stages 0-9; lib.rs:420-423). */
int g16_h_and_msms(g16_circuit *c, const uint8_t *witness_mont, size_t n, g16_msm_outputs *out);
/* prove_with_blinders (crates/groth16/src/prove.rs:175-184): stages 0-11 with
 * the caller's r and s (Montgomery Fr). */
int g16_prove_with_blinders(g16_circuit *c, const uint8_t *witness_mont, size_t n, const uint8_t *r_mont,
                            const uint8_t *s_mont, g16_proof *out);
/* PreparedCircuit::h_and_msms_from_rows (crates/groth16/src/lib.rs:425-444;
 * the CPU backend's crates/groth16/src/cpu.rs:384-471) for a snarkjs-basis key:
 * stage 0 handed over as a_rows[i] = A_i.w and b_rows[i] = B_i.w, rows <=
 * domain_size Montgomery Fr each, every row past them zero.  The outputs
 * equal g16_h_and_msms when the rows are the witness's own. */
int g16_h_and_msms_from_rows(g16_circuit *c, const uint8_t *witness_mont, size_t n, const uint8_t *a_rows,
                             const uint8_t *b_rows, size_t rows, g16_msm_outputs *out);
/* Stages 0-11 of prove_from_rows (crates/groth16/src/prove.rs:93-117) with the
 * caller's r and s; the self-check is g16_circuit_verify. */
int g16_prove_with_blinders_from_rows(g16_circuit *c, const uint8_t *witness_mont, size_t n, const uint8_t *a_rows,
                                      const uint8_t *b_rows, size_t rows, const uint8_t *r_mont,
                                      const uint8_t *s_mont, g16_proof *out);
/* The same with the witness already resident in device memory (a device
 * pointer to n Montgomery Fr); no host-to-device copy. */
int g16_prove_with_blinders_device(g16_circuit *c, const void *d_witness_mont, size_t n, const uint8_t *r_mont,
                                   const uint8_t *s_mont, g16_proof *out);
int g16_stage_timings_get(const g16_circuit *c, g16_stage_timings *out);
/* Readies up to `count` workspaces of c (one per proof in flight; as many as
 * its pool, 8, and the device budget allow) by proving a throwaway witness
 * (the constant wire 1, every other wire 0, r = s = 1) twice on each: the
 * first proof sizes the workspace's scratch, the second captures its CUDA
 * graph.  Up to that many concurrent proofs of c then allocate nothing and
 * replay graphs.  The throwaway proofs count in c's stage timings.  Gather-path
 * keys only. */
int g16_circuit_warm(g16_circuit *c, uint32_t count);
/* prove::prove (crates/groth16/src/prove.rs:34-92): r and s drawn from the
 * operating system's CSPRNG, stages 0-11, then the proof is verified against
 * the circuit's verifying key (timed as verify_us); G16_ERR_SELF_VERIFY when
 * it does not verify. */
int g16_prove(g16_circuit *c, const uint8_t *witness_mont, size_t n, g16_proof *out);

/* ---------------- verification (crates/groth16/src/verify.rs:49-175) ----------------
 * verify::verify on the host: key structure, proof elements (on the curve, B
 * in the prime-order subgroup, none at infinity), then
 * e(-A, B) e(alpha, beta) e(L, gamma) e(C, delta) = 1 with one final
 * exponentiation.  public_mont: n_public Montgomery Fr (the witness's wires
 * 1..n_public).  G16_OK when the proof verifies; G16_ERR_VERIFY when it does
 * not or an element is invalid; G16_ERR_FORMAT for an unsafe key;
 * G16_ERR_INVALID_ARGUMENT for a public-input count that does not match. */
int g16_verify(const uint8_t *alpha_g1, const uint8_t *beta_g2, const uint8_t *gamma_g2, const uint8_t *delta_g2,
               const uint8_t *ic, size_t n_ic, const uint8_t *public_mont, size_t n_public, const g16_proof *proof);
/* The same against a prepared circuit's verifying key. */
int g16_circuit_verify(const g16_circuit *c, const uint8_t *public_mont, size_t n_public, const g16_proof *proof);
/* prod_i e(P_i, Q_i) == 1 for n packed affine pairs (G1 64 B, G2 128 B):
 * returns 1, 0, or G16_ERR_INVALID_ARGUMENT (as a negative value) for
 * non-canonical or off-curve input. */
int g16_pairing_check(const uint8_t *g1_points, const uint8_t *g2_points, size_t n);

/* ---------------- per-instance tuning (no reference counterpart) ----------------
 * The MSM window sizes and the NTT tiling of a prepared circuit.  g16_prepare
 * picks them from a cost model; g16_autotune times candidates on the device
 * with one of the circuit's witnesses and keeps the fastest (the proof's
 * values do not depend on them).  Window-size changes rebuild the circuit's
 * window-shifted base tables. */
typedef struct {
    int32_t msm_window_bits_witness; /* c of the A, B1, L, B2 MSMs */
    int32_t msm_window_bits_h;       /* c of the H MSM */
    int32_t ntt_tile_log;            /* inner NTT pass: tiles of 2^ntt_tile_log elements (2..12) */
    int32_t ntt_outer_log_l;         /* outer passes: 2^ntt_outer_log_l columns per tile row */
    double model_ms;                 /* device ms per proof with the cost model's choice (autotune only) */
    double tuned_ms;                 /* the same with the kept choice (autotune only) */
} g16_tuning;
int g16_tuning_get(const g16_circuit *c, g16_tuning *out);
/* Applies explicit choices (window bits 8..20); no proof may be in flight on c. */
int g16_tuning_set(g16_circuit *c, const g16_tuning *t);
/* Times the candidates with one witness (n Montgomery Fr) and keeps the
 * fastest; no proof may be in flight on c.  concurrency 1 minimises one
 * proof's latency (stage by stage); 2..8 minimises device time per proof
 * with that many proofs in flight together on as many workspaces (the
 * batched and served objective).  model_ms / tuned_ms are per proof.  out
 * may be NULL. */
int g16_autotune(g16_circuit *c, const uint8_t *witness_mont, size_t n, int concurrency, g16_tuning *out);

/* ---------------- batched and served proving ---------------- */
/* Proves count independent jobs (circuits may repeat or differ) in one
 * submission; outputs are bit-identical to count single calls.
 * witnesses[i] has lens[i] Montgomery Fr; r, s: count x 32 bytes. */
int g16_prove_batch(g16_backend *b, size_t count, g16_circuit *const *circuits, const uint8_t *const *witnesses,
                    const size_t *lens, const uint8_t *r_mont, const uint8_t *s_mont, g16_proof *out);
/* The same, and done_ms[i] (count doubles, NULL to skip) receives the
 * milliseconds from the call's start until job i's proof was complete: the
 * per-proof latency of a batch submitted at once. */
int g16_prove_batch_timed(g16_backend *b, size_t count, g16_circuit *const *circuits,
                          const uint8_t *const *witnesses, const size_t *lens, const uint8_t *r_mont,
                          const uint8_t *s_mont, g16_proof *out, double *done_ms);

/* Served proving (no reference counterpart; the reference proves one request
 * per call).  A request loop with continuous batching: each of `lanes`
 * workers, as soon as it is free, takes every small request queued at that
 * moment (in arrival order, up to the batch limits) and proves them together
 * as one g16_prove_batch submission, so requests that arrive while others are
 * on the GPU are admitted with the next free worker's batch, and the workers'
 * batches overlap on the device.  A request of at least 2^19 witness wires
 * (G16_SERVE_SOLO_WIRES; 0 batches every size) is proved alone by the next
 * free worker when it reaches the head of the queue: it fills the device by
 * itself, and the small requests of a batch would otherwise wait for it (a
 * batch's proofs complete together).  A batch of one request is a plain
 * g16_prove_with_blinders call.  Registered keys are prepared on first use
 * and stay resident in HBM while their device bytes fit key_budget_bytes
 * (0 = unlimited); a key that does not fit evicts least recently used idle
 * keys.  A batch starts when its working set fits the backend's device-memory
 * budget.  Results equal single g16_prove_with_blinders calls.  Limits: at
 * most 64 requests and about 2^21 witness wires per batch (G16_SERVE_BATCH,
 * G16_SERVE_BATCH_WIRES). */
typedef struct g16_server g16_server;
typedef struct {
    uint64_t submitted, completed, prepared, evicted, resident_keys, resident_bytes, queued;
    uint64_t batches;        /* batched submissions of two or more requests */
    uint64_t batched;        /* requests proved in those */
    uint64_t alone;          /* requests proved alone */
} g16_server_stats;
int g16_server_new(g16_backend *b, uint64_t key_budget_bytes, int lanes, g16_server **out);
/* Requests per batch (at least 1); 1 proves each request alone on a
 * workspace: plain one-proof-at-a-time serving. */
int g16_server_set_max_batch(g16_server *s, size_t max_batch);
/* Keeps a host copy of the .zkey bytes; the key is prepared when first needed. */
int g16_server_register_key(g16_server *s, uint32_t key_id, const uint8_t *zkey, size_t len);
/* Copies the witness (n Montgomery Fr) and the blinders; returns a ticket. */
int g16_server_submit(g16_server *s, uint32_t key_id, const uint8_t *witness_mont, size_t n, const uint8_t *r_mont,
                      const uint8_t *s_mont, uint64_t *ticket);
/* Blocks until the ticket's proof is done.  queue_ms: submit to start;
 * latency_ms: submit to finish.  Each ticket can be waited for once. */
int g16_server_wait(g16_server *s, uint64_t ticket, g16_proof *out, double *queue_ms, double *latency_ms);
int g16_server_stats_get(g16_server *s, g16_server_stats *out);
/* Finishes the queued requests, then frees every resident key. */
void g16_server_free(g16_server *s);

/* Counters of a backend's batched-proving engines since it was opened. */
typedef struct {
    uint64_t submissions;    /* g16_prove_batch calls run by an engine */
    uint64_t layouts;        /* of those, ones that laid out a new mix of circuits */
    uint64_t replays;        /* ones that replayed a captured CUDA graph */
    uint64_t grown_bytes;    /* device bytes the engines allocated (buffers only grow) */
    uint64_t engines;        /* engines built */
} g16_batch_stats;
int g16_batch_stats_get(const g16_backend *b, g16_batch_stats *out);
/* Sizes the backend's batched-proving engines for a batch of these circuits
 * (repeats allowed) without proving it: every engine lays the batch out once,
 * so that its buffers, which only grow, are at that batch's sizes; a later
 * g16_prove_batch of that mix allocates nothing on any engine, and smaller mixes
 * of the same circuits need at most small additions.  Takes each
 * engine in turn when it is idle.  The engines' device bytes count against the backend's
 * budget (G16_ERR_DEVICE_MEMORY when they do not fit).  Nothing to do, and
 * G16_OK, for a batch that g16_prove_batch would prove on host lanes (compact
 * keys, constant-work MSMs, G16_BATCH_ENGINE=0).  Gather-path keys only, as
 * g16_prove_batch. */
int g16_batch_reserve(g16_backend *b, size_t count, g16_circuit *const *circuits);

/* ---------------- primitives (MsmBackend, crates/msm/src/lib.rs:52-82) ---------------- */
/* sum_i scalars[i] * bases[i]; host buffers; result affine packed. */
int g16_msm_g1(g16_backend *b, const uint8_t *bases, const uint8_t *scalars, size_t n, int scalars_form,
               uint8_t *out64);
int g16_msm_g2(g16_backend *b, const uint8_t *bases, const uint8_t *scalars, size_t n, int scalars_form,
               uint8_t *out128);
/* Device-resident inputs (device pointers), for callers that keep bases in HBM. */
int g16_msm_g1_device(g16_backend *b, const void *d_bases, const void *d_scalars, size_t n, int scalars_form,
                      uint8_t *out64);
int g16_msm_g2_device(g16_backend *b, const void *d_bases, const void *d_scalars, size_t n, int scalars_form,
                      uint8_t *out128);

/* A G1 MSM that allocates no memory -- no counterpart in the reference.
 * For callers that cannot call cudaMalloc: their device memory belongs to
 * another allocator, or an allocation (and its implicit device
 * synchronisation) is not acceptable in their request path.  Same result as
 * g16_msm_g1_device, computed inside one fixed scratch array (about 12 MiB)
 * that is part of the library image and that every GPU which loads the
 * library holds until the process exits.  At most 16384 points (larger n is
 * refused with G16_ERR_INVALID_ARGUMENT); runs on `device`'s legacy default
 * stream and returns with the result on the host.  The first call on a device
 * looks up the array's address (make it before any stream capture); under
 * CUDA's lazy module loading it is also when the device commits the array and
 * loads the MSM kernels, so make it at start-up (a full device fails it with
 * G16_ERR_DEVICE_MEMORY).  Resetting the device after that first call is not
 * supported.  All calls share the array: calls whose device work overlaps
 * race and must be serialised by the caller.  Kernel timing must be off. */
int g16_msm_g1_device_noalloc(int device, const void *d_bases, const void *d_scalars, size_t n, int scalars_form,
                              uint8_t *out64);

/* ---------------- NTT (CpuNtt API, crates/ntt/src/lib.rs:415-584) ---------------- */
/* In place on 2^log_n Montgomery Fr in host memory.  shift_mont is the coset
 * shift for the COSET modes (NULL = the proving coset shift omega_2n). */
int g16_ntt(g16_backend *b, int mode, uint32_t log_n, uint8_t *data_mont, const uint8_t *shift_mont);
/* The same on a device pointer. */
int g16_ntt_device(g16_backend *b, int mode, uint32_t log_n, void *d_data_mont, const uint8_t *shift_mont);

/* ---------------- kernel timing (CUDA events on the launching stream) ---------------- */
void g16_kernel_timing_enable(int on);
void g16_kernel_timing_reset(void);
/* Writes "name total_ms launches work_units\n" lines; returns the full length.
 * work_units: mixed additions for the MSM accumulate kernels, else 0. */
size_t g16_kernel_timing_report(char *buf, size_t len);
/* Kernels launched by this library since load (every launch site counts). */
uint64_t g16_launch_count(void);
/* Device allocations (cudaMalloc calls) this library has made since load. */
uint64_t g16_device_alloc_count(void);
/* serial != 0 runs every stage of this circuit's proofs on one stream (no
 * overlap), so per-kernel event times do not include concurrent work: for
 * profiling.  Results are identical either way. */
int g16_circuit_set_serial(g16_circuit *c, int serial);
/* Device-to-host bytes the last proof on this circuit read back. */
uint64_t g16_circuit_readback_bytes(const g16_circuit *c);
/* Measured issue rate of 32-bit mad.lo/mad.hi on this device (per second):
 * the peak of the integer-multiply roofline the field kernels run against. */
int g16_imad_peak(g16_backend *b, double *imad_per_s);

/* ---------------- device memory helpers (for callers without a CUDA runtime) ---------------- */
int g16_device_alloc(g16_backend *b, size_t bytes, void **d_out);
int g16_device_free(g16_backend *b, void *d);
int g16_device_upload(g16_backend *b, void *d_dst, const void *src, size_t bytes);
int g16_device_sync(g16_backend *b);

/* ---------------- synthetic circuits, witnesses and keys ---------------- */
/* A seeded R1CS: wire 0 = 1, n_inputs input wires (the first n_public of them
 * public), one new wire per constraint w_k = (A.w)(B.w) with 2-3 terms per A
 * and B row on earlier wires.  Witness values about 60% {0,1}, 20% below
 * 2^32, 20% uniform.  The key is written as a snarkjs .zkey from seeded
 * toxic waste (tau, alpha, beta, delta; gamma = 1): the key a one-
 * contribution snarkjs/snarkrs ceremony + setup + zkey contribute yields. */
typedef struct g16_synth g16_synth;
int g16_synth_new(uint64_t seed, uint32_t n_constraints, uint32_t n_inputs, uint32_t n_public, g16_synth **out);
void g16_synth_free(g16_synth *s);
uint32_t g16_synth_n_vars(const g16_synth *s);
uint32_t g16_synth_domain_size(const g16_synth *s);
/* n_vars Montgomery Fr; inputs drawn from witness_seed. */
int g16_synth_witness(const g16_synth *s, uint64_t witness_seed, uint8_t *out_mont);
/* .zkey bytes; out = NULL to size. threads = 0 uses all cores. */
int g16_synth_zkey(const g16_synth *s, uint64_t toxic_seed, int threads, uint8_t *out, size_t cap, size_t *len_out);
/* The same .zkey bytes with the point sections (fixed-base multiplications of
 * the generators, ~4.4M G1 and 1.1M G2 points at 2^21) computed on the GPU
 * `device`; G16_ERR_DEVICE if a CUDA call fails. */
int g16_synth_zkey_device(const g16_synth *s, uint64_t toxic_seed, int device, uint8_t *out, size_t cap,
                          size_t *len_out);
/* circom .r1cs bytes; out = NULL to size. */
int g16_synth_r1cs(const g16_synth *s, uint8_t *out, size_t cap, size_t *len_out);
/* n affine points k_i G with k_i uniform in [1, r) (group 1 = G1, 64 B each;
 * group 2 = G2, 128 B each); threads = 0 uses all cores. */
int g16_synth_points(int group, uint64_t seed, size_t n, int threads, uint8_t *out);
/* n standard-form scalars: dist 0 uniform in [0, r); dist 1 = 35% zero,
 * 35% one, 30% uniform (the "70% in {0,1}" distribution). */
int g16_synth_scalars(uint64_t seed, size_t n, int dist, uint8_t *out_std);

#ifdef __cplusplus
}
#endif
#endif /* G16B200_H */
