/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * The timed CPU baseline's MSM: a restatement, for speed, of the reference
 * CPU prover's Pippenger (crates/msm/src/lib.rs), the portable path it takes
 * where AVX-512 IFMA is absent:
 *   - prescan (:534-620): zero scalars and infinity bases dropped, scalars
 *     equal to 1 folded into one running sum, the rest kept by index;
 *   - window_size (:160-172) over the m kept scalars, signed_digit (:319-333)
 *     over RECODE_BITS = 255 bits, 2^(c-1) buckets per window;
 *   - windows of c >= 9 (batch_size >= MIN_BATCH, :120-142) fill affine
 *     buckets by batched affine additions sharing one inversion per round
 *     (BatchFill, :764-1010): a busy map allows one pending addition per
 *     bucket and round, a conflict waits for the next round, a second
 *     conflict on the same bucket goes to XYZZ side buckets;
 *   - narrower windows use the XYZZ fill (window_chunk, :703-760);
 *   - each window's point range is cut into parts so that there are about
 *     twice as many tasks as threads (:1740-1760; the reference hands the
 *     last windows out piece by piece, ganged_windows :1555, to the same end);
 *   - the parts' buckets are summed into a running sum over ranges of
 *     REDUCE_CHUNK = 2048 buckets in parallel, the ranges' offsets settled at
 *     the end (chunked_running_sum :1086-1135), then Horner over the windows.
 * The one simplification: the running sum over the buckets is the XYZZ one
 * (:1049-1075) rather than the segmented affine one (:1137-1300).
 *
 * Scheduling is OpenMP tasks, so that several MSMs called as tasks of one
 * parallel region share the pool (the prover runs its five concurrently,
 * crates/groth16/src/cpu.rs:585-621).
 */
#include "port.h"
#include "port_curve.h"
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RECODE_BITS 255
#define MAX_WINDOW 16
#define SCAN_CHUNK 4096
#define BATCH 1024
#define MIN_BATCH 128
#define REDUCE_CHUNK 2048
#define CHUNK_BUCKET_RATIO 16

static int window_size(size_t m) {
    int best = 3;
    unsigned __int128 best_cost = ~(unsigned __int128)0;
    for (int c = 3; c <= MAX_WINDOW; c++) {
        unsigned __int128 w = (RECODE_BITS + c - 1) / c;
        unsigned __int128 cost = w * ((unsigned __int128)m + 3 * ((unsigned __int128)1 << (c - 1)));
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static uint64_t read_bits(const uint64_t *l, int off, int width) {
    int idx = off >> 6;
    if (idx >= 4) return 0;
    int sh = off & 63;
    uint64_t b = l[idx] >> sh;
    if (sh + width > 64 && idx + 1 < 4) b |= l[idx + 1] << (64 - sh);
    return b & ((1ULL << width) - 1);
}

static int signed_digit(const uint64_t *l, int w, int c) {
    int off = w * c;
    int64_t b = (int64_t)read_bits(l, off, c);
    int64_t d = b - ((b >> (c - 1)) << c);
    return (int)(d + (off ? (int64_t)read_bits(l, off - 1, 1) : 0));
}

static int n_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ===================================================================== *
 * One MSM over a group, instantiated for G1 (Fq) and G2 (Fq2).
 *   F      field element type
 *   AFF    affine point type of the oracle (x, y, inf)
 *   JAC    Jacobian point type of the oracle
 *   P      prefix of the field functions (pq / pq2)
 * ===================================================================== */
#define PORT_DEFINE_MSM(G, F, AFF, JAC, P, ZERO_F, ONE_F)                                               \
/* ---- the batch-affine fill (BatchFill) ---- */                                                    \
typedef struct { uint32_t b; F x, y; } G##_pend;                                                     \
typedef struct {                                                                                      \
    size_t nb, batch;                                                                                 \
    F (*xy)[2];                                                                                       \
    uint8_t *occ, *busy;                                                                              \
    G##_pend *pending; size_t np;                                                                     \
    G##_pend *retry; size_t nr;                                                                       \
    uint32_t *side_slot; G##_xyzz *side; size_t nside, cap_side;                                      \
    F *dens, *prefix; uint8_t *ops;                                                                   \
} G##_fill;                                                                                           \
                                                                                                      \
static void G##_fill_init(G##_fill *f, size_t nb, size_t batch) {                                     \
    memset(f, 0, sizeof *f);                                                                          \
    f->nb = nb;                                                                                       \
    f->batch = batch;                                                                                 \
    f->xy = malloc(nb * sizeof *f->xy);                                                               \
    f->occ = calloc(nb, 1);                                                                           \
    f->busy = calloc(nb, 1);                                                                          \
    size_t cap = batch + batch / 2 + 2;                                                               \
    f->pending = malloc(cap * sizeof(G##_pend));                                                      \
    f->retry = malloc((batch + 2) * sizeof(G##_pend));                                               \
    f->dens = malloc(cap * sizeof(F));                                                                \
    f->prefix = malloc(cap * sizeof(F));                                                              \
    f->ops = malloc(cap);                                                                             \
}                                                                                                     \
                                                                                                      \
static void G##_fill_free(G##_fill *f) {                                                              \
    free(f->xy); free(f->occ); free(f->busy); free(f->pending); free(f->retry);                       \
    free(f->side_slot); free(f->side); free(f->dens); free(f->prefix); free(f->ops);                 \
}                                                                                                     \
                                                                                                      \
static G##_xyzz *G##_side_entry(G##_fill *f, size_t b) {                                              \
    if (!f->side_slot) {                                                                              \
        f->side_slot = calloc(f->nb, sizeof(uint32_t));                                               \
        f->cap_side = 64;                                                                             \
        f->side = malloc(f->cap_side * sizeof(G##_xyzz));                                             \
        G##_set_id(&f->side[0]);                                                                      \
        f->nside = 1;                                                                                 \
    }                                                                                                 \
    if (!f->side_slot[b]) {                                                                           \
        if (f->nside == f->cap_side) {                                                                \
            f->cap_side *= 2;                                                                         \
            f->side = realloc(f->side, f->cap_side * sizeof(G##_xyzz));                               \
        }                                                                                             \
        G##_set_id(&f->side[f->nside]);                                                               \
        f->side_slot[b] = (uint32_t)f->nside++;                                                       \
    }                                                                                                 \
    return &f->side[f->side_slot[b]];                                                                 \
}                                                                                                     \
                                                                                                      \
/* one round: classify, one shared inversion (Montgomery's trick), apply */                          \
static void G##_flush(G##_fill *f) {                                                                  \
    size_t n = f->np;                                                                                 \
    if (!n) return;                                                                                   \
    F acc = ONE_F;                                                                                    \
    for (size_t k = 0; k < n; k++) {                                                                  \
        G##_pend *e = &f->pending[k];                                                                 \
        F *bxy = f->xy[e->b];                                                                         \
        F den;                                                                                        \
        P##_sub(&den, &e->x, &bxy[0]);                                                                \
        if (!P##_is_zero(&den)) f->ops[k] = 0;                                                        \
        else if (P##_eq(&e->y, &bxy[1])) { f->ops[k] = 1; P##_dbl(&den, &bxy[1]); }                   \
        else { f->ops[k] = 2; den = ONE_F; }                                                          \
        f->dens[k] = den;                                                                             \
        f->prefix[k] = acc;                                                                           \
        P##_mul(&acc, &acc, &den);                                                                    \
    }                                                                                                 \
    F inv;                                                                                            \
    P##_inv(&inv, &acc);                                                                              \
    for (size_t k = n; k-- > 0;) {                                                                    \
        G##_pend *e = &f->pending[k];                                                                 \
        F d, lam, t, x3;                                                                              \
        P##_mul(&d, &inv, &f->prefix[k]);                                                             \
        P##_mul(&inv, &inv, &f->dens[k]);                                                             \
        F *bxy = f->xy[e->b];                                                                         \
        if (f->ops[k] == 0) {                                                                         \
            P##_sub(&t, &e->y, &bxy[1]);                                                              \
            P##_mul(&lam, &t, &d);                                                                    \
            P##_sqr(&x3, &lam);                                                                       \
            P##_sub(&x3, &x3, &bxy[0]);                                                               \
            P##_sub(&x3, &x3, &e->x);                                                                 \
            P##_sub(&t, &bxy[0], &x3);                                                                \
            P##_mul(&t, &lam, &t);                                                                    \
            P##_sub(&bxy[1], &t, &bxy[1]);                                                            \
            bxy[0] = x3;                                                                              \
        } else if (f->ops[k] == 1) {                                                                  \
            F xx;                                                                                     \
            P##_sqr(&xx, &bxy[0]);                                                                    \
            P##_dbl(&t, &xx);                                                                         \
            P##_add(&t, &t, &xx);                                                                     \
            P##_mul(&lam, &t, &d);                                                                    \
            P##_sqr(&x3, &lam);                                                                       \
            P##_sub(&x3, &x3, &bxy[0]);                                                               \
            P##_sub(&x3, &x3, &bxy[0]);                                                               \
            P##_sub(&t, &bxy[0], &x3);                                                                \
            P##_mul(&t, &lam, &t);                                                                    \
            P##_sub(&bxy[1], &t, &bxy[1]);                                                            \
            bxy[0] = x3;                                                                              \
        } else {                                                                                      \
            f->occ[e->b] = 0;                                                                         \
        }                                                                                             \
        f->busy[e->b] = 0;                                                                            \
    }                                                                                                 \
    f->np = 0;                                                                                        \
}                                                                                                     \
                                                                                                      \
static void G##_reschedule(G##_fill *f) {                                                             \
    while (f->nr) {                                                                                   \
        G##_pend e = f->retry[--f->nr];                                                               \
        if (!f->occ[e.b]) { f->xy[e.b][0] = e.x; f->xy[e.b][1] = e.y; f->occ[e.b] = 1; }              \
        else if (f->busy[e.b]) G##_madd(G##_side_entry(f, e.b), &e.x, &e.y);                           \
        else { f->busy[e.b] = 1; f->pending[f->np++] = e; }                                           \
    }                                                                                                 \
}                                                                                                     \
                                                                                                      \
static void G##_insert(G##_fill *f, uint32_t b, const F *x, const F *y) {                            \
    if (!f->occ[b]) { f->xy[b][0] = *x; f->xy[b][1] = *y; f->occ[b] = 1; return; }                   \
    G##_pend e; e.b = b; e.x = *x; e.y = *y;                                                          \
    if (f->busy[b]) {                                                                                 \
        f->retry[f->nr++] = e;                                                                        \
        if (f->nr >= f->batch) { G##_flush(f); G##_reschedule(f); }                                   \
        return;                                                                                       \
    }                                                                                                 \
    f->busy[b] = 1;                                                                                   \
    f->pending[f->np++] = e;                                                                          \
    if (f->np >= f->batch) { G##_flush(f); G##_reschedule(f); }                                       \
}                                                                                                     \
                                                                                                      \
static void G##_settle(G##_fill *f) { G##_flush(f); G##_reschedule(f); G##_flush(f); }                \
                                                                                                      \
typedef struct {                                                                                      \
    const AFF *bases;                                                                                 \
    const uint32_t *idx;                                                                              \
    const fp_t *sc;      /* kept scalars, standard form, in prescan order */                          \
    size_t m;                                                                                         \
    int c, W, parts, batched;                                                                         \
    size_t nb, part_len;                                                                              \
    G##_fill *fills;     /* W x parts, batched */                                                     \
    G##_xyzz *xb;        /* W x parts x nb, XYZZ fill */                                              \
    G##_xyzz *wsum;      /* W window sums */                                                          \
} G##_plan;                                                                                           \
                                                                                                      \
static void G##_fill_task(G##_plan *pl, int w, int part) {                                           \
    size_t lo = (size_t)part * pl->part_len, hi = lo + pl->part_len < pl->m ? lo + pl->part_len : pl->m; \
    if (pl->batched) {                                                                                \
        G##_fill *f = &pl->fills[(size_t)w * pl->parts + part];                                       \
        G##_fill_init(f, pl->nb, BATCH < pl->nb / 2 ? BATCH : pl->nb / 2);                            \
        for (size_t k = lo; k < hi; k++) {                                                            \
            int d = signed_digit(pl->sc[k].v, w, pl->c);                                              \
            if (!d) continue;                                                                         \
            const AFF *b = &pl->bases[pl->idx[k]];                                                    \
            if (d > 0) G##_insert(f, (uint32_t)(d - 1), &b->x, &b->y);                                \
            else { F ny; P##_neg(&ny, &b->y); G##_insert(f, (uint32_t)(-d - 1), &b->x, &ny); }         \
        }                                                                                             \
        G##_settle(f);                                                                                \
    } else {                                                                                          \
        G##_xyzz *bk = pl->xb + ((size_t)w * pl->parts + part) * pl->nb;                              \
        for (size_t j = 0; j < pl->nb; j++) G##_set_id(&bk[j]);                                       \
        for (size_t k = lo; k < hi; k++) {                                                            \
            int d = signed_digit(pl->sc[k].v, w, pl->c);                                              \
            if (!d) continue;                                                                         \
            const AFF *b = &pl->bases[pl->idx[k]];                                                    \
            if (d > 0) G##_madd(&bk[d - 1], &b->x, &b->y);                                            \
            else { F ny; P##_neg(&ny, &b->y); G##_madd(&bk[-d - 1], &b->x, &ny); }                     \
        }                                                                                             \
    }                                                                                                 \
}                                                                                                     \
                                                                                                      \
/* bucket j of window w summed over the parts, added into acc */                                    \
static inline void G##_bucket_into(G##_plan *pl, int w, size_t j, G##_xyzz *acc) {                    \
    for (int p = 0; p < pl->parts; p++) {                                                             \
        if (pl->batched) {                                                                            \
            G##_fill *f = &pl->fills[(size_t)w * pl->parts + p];                                      \
            if (f->occ[j]) G##_madd(acc, &f->xy[j][0], &f->xy[j][1]);                                 \
            if (f->side_slot && f->side_slot[j]) G##_add(acc, &f->side[f->side_slot[j]]);             \
        } else {                                                                                      \
            G##_add(acc, &pl->xb[((size_t)w * pl->parts + p) * pl->nb + j]);                          \
        }                                                                                             \
    }                                                                                                 \
}                                                                                                     \
                                                                                                      \
/* running sums over buckets [lo, hi) of window w, counting them from 1: */                         \
/* tot = sum_j (j - lo + 1) S_j, plain = sum_j S_j */                                                \
static void G##_range_sum(G##_plan *pl, int w, size_t lo, size_t hi, G##_xyzz *tot, G##_xyzz *plain) { \
    G##_xyzz run, t;                                                                                  \
    G##_set_id(&run);                                                                                 \
    G##_set_id(&t);                                                                                   \
    for (size_t j = hi; j-- > lo;) {                                                                  \
        G##_bucket_into(pl, w, j, &run);                                                              \
        G##_add(&t, &run);                                                                            \
    }                                                                                                 \
    *tot = t;                                                                                         \
    *plain = run;                                                                                     \
}                                                                                                     \
                                                                                                      \
static void port_##G##_msm_impl(JAC *out, const AFF *bases, const fp_t *scalars, size_t n, int threads) { \
    /* prescan */                                                                                     \
    size_t nchunks = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;                                               \
    size_t *cnt = calloc(nchunks + 1, sizeof(size_t));                                                \
    G##_xyzz *ones = malloc((nchunks ? nchunks : 1) * sizeof(G##_xyzz));                              \
    _Pragma("omp taskloop num_tasks(port_tasks())")                                                              \
    for (size_t ch = 0; ch < nchunks; ch++) {                                                         \
        size_t lo = ch * SCAN_CHUNK, hi = lo + SCAN_CHUNK < n ? lo + SCAN_CHUNK : n, k = 0;           \
        G##_set_id(&ones[ch]);                                                                        \
        for (size_t i = lo; i < hi; i++) {                                                            \
            const uint64_t *s = scalars[i].v;                                                         \
            if (!(s[0] | s[1] | s[2] | s[3]) || bases[i].inf) continue;                               \
            if (s[0] == 1 && !(s[1] | s[2] | s[3])) { G##_madd(&ones[ch], &bases[i].x, &bases[i].y); continue; } \
            k++;                                                                                      \
        }                                                                                             \
        cnt[ch + 1] = k;                                                                              \
    }                                                                                                 \
    for (size_t ch = 0; ch < nchunks; ch++) cnt[ch + 1] += cnt[ch];                                   \
    size_t m = cnt[nchunks];                                                                          \
    uint32_t *idx = malloc((m ? m : 1) * sizeof(uint32_t));                                           \
    fp_t *sc = malloc((m ? m : 1) * sizeof(fp_t));                                                    \
    _Pragma("omp taskloop num_tasks(port_tasks())")                                                              \
    for (size_t ch = 0; ch < nchunks; ch++) {                                                         \
        size_t lo = ch * SCAN_CHUNK, hi = lo + SCAN_CHUNK < n ? lo + SCAN_CHUNK : n, k = cnt[ch];     \
        for (size_t i = lo; i < hi; i++) {                                                            \
            const uint64_t *s = scalars[i].v;                                                         \
            if (!(s[0] | s[1] | s[2] | s[3]) || bases[i].inf) continue;                               \
            if (s[0] == 1 && !(s[1] | s[2] | s[3])) continue;                                         \
            idx[k] = (uint32_t)i;                                                                     \
            sc[k] = scalars[i];                                                                       \
            k++;                                                                                      \
        }                                                                                             \
    }                                                                                                 \
    G##_xyzz ones_sum;                                                                                \
    G##_set_id(&ones_sum);                                                                            \
    for (size_t ch = 0; ch < nchunks; ch++) G##_add(&ones_sum, &ones[ch]);                            \
    free(ones);                                                                                       \
    free(cnt);                                                                                        \
    if (m == 0) {                                                                                     \
        G##_to_jac(out, &ones_sum);                                                                   \
        free(idx); free(sc);                                                                          \
        return;                                                                                       \
    }                                                                                                 \
    G##_plan pl;                                                                                      \
    memset(&pl, 0, sizeof pl);                                                                        \
    pl.bases = bases; pl.idx = idx; pl.sc = sc; pl.m = m;                                             \
    pl.c = window_size(m);                                                                            \
    pl.W = (RECODE_BITS + pl.c - 1) / pl.c;                                                           \
    pl.nb = (size_t)1 << (pl.c - 1);                                                                  \
    pl.batched = (BATCH < pl.nb / 2 ? BATCH : pl.nb / 2) >= MIN_BATCH;                                \
    if (threads < 1) threads = 1;                                                                     \
    size_t parts = (2 * (size_t)threads + pl.W - 1) / pl.W;                                           \
    if (pl.batched) {                                                                                 \
        size_t grain = pl.nb / 4 > 1024 ? pl.nb / 4 : 1024;                                           \
        size_t maxp = (m + grain - 1) / grain;                                                        \
        if (parts > maxp) parts = maxp;                                                               \
    } else {                                                                                          \
        size_t maxp = m / (CHUNK_BUCKET_RATIO * pl.nb);                                               \
        if (maxp < 1) maxp = 1;                                                                       \
        if (parts > maxp) parts = maxp;                                                               \
    }                                                                                                 \
    if (parts < 1) parts = 1;                                                                         \
    pl.parts = (int)parts;                                                                            \
    pl.part_len = (m + parts - 1) / parts;                                                            \
    if (pl.batched) pl.fills = calloc((size_t)pl.W * parts, sizeof(G##_fill));                        \
    else pl.xb = malloc((size_t)pl.W * parts * pl.nb * sizeof(G##_xyzz));                             \
    pl.wsum = malloc((size_t)pl.W * sizeof(G##_xyzz));                                                \
    long tasks = (long)pl.W * (long)parts;                                                            \
    _Pragma("omp taskloop num_tasks(port_tasks())")                                                              \
    for (long t = 0; t < tasks; t++) G##_fill_task(&pl, (int)(t / (long)parts), (int)(t % (long)parts)); \
    /* per window: the bucket range in chunks of REDUCE_CHUNK, each a task */                         \
    size_t rc = pl.nb < REDUCE_CHUNK ? pl.nb : REDUCE_CHUNK;                                          \
    size_t nr = (pl.nb + rc - 1) / rc;                                                                \
    G##_xyzz *tot = malloc((size_t)pl.W * nr * sizeof(G##_xyzz));                                     \
    G##_xyzz *plain = malloc((size_t)pl.W * nr * sizeof(G##_xyzz));                                   \
    long rtasks = (long)pl.W * (long)nr;                                                              \
    _Pragma("omp taskloop num_tasks(port_tasks())")                                                              \
    for (long t = 0; t < rtasks; t++) {                                                               \
        int w = (int)(t / (long)nr);                                                                  \
        size_t r = (size_t)(t % (long)nr), lo = r * rc, hi = lo + rc < pl.nb ? lo + rc : pl.nb;       \
        G##_range_sum(&pl, w, lo, hi, &tot[t], &plain[t]);                                            \
    }                                                                                                 \
    for (int w = 0; w < pl.W; w++) {                                                                  \
        G##_xyzz sum, run, owed;                                                                      \
        G##_set_id(&sum); G##_set_id(&run); G##_set_id(&owed);                                        \
        for (size_t r = nr; r-- > 0;) {                                                               \
            G##_add(&sum, &tot[(size_t)w * nr + r]);                                                  \
            if (r > 0) { G##_add(&run, &plain[(size_t)w * nr + r]); G##_add(&owed, &run); }           \
        }                                                                                             \
        for (size_t s = rc; s > 1; s >>= 1) { G##_xyzz d; G##_dbl(&d, &owed); owed = d; }            \
        G##_add(&sum, &owed);                                                                         \
        pl.wsum[w] = sum;                                                                             \
    }                                                                                                 \
    /* Horner over the windows */                                                                    \
    G##_xyzz acc = pl.wsum[pl.W - 1];                                                                 \
    for (int w = pl.W - 2; w >= 0; w--) {                                                             \
        for (int k = 0; k < pl.c; k++) { G##_xyzz d; G##_dbl(&d, &acc); acc = d; }                   \
        G##_add(&acc, &pl.wsum[w]);                                                                   \
    }                                                                                                 \
    G##_add(&acc, &ones_sum);                                                                         \
    G##_to_jac(out, &acc);                                                                            \
    if (pl.batched) {                                                                                 \
        for (long t = 0; t < tasks; t++) G##_fill_free(&pl.fills[t]);                                 \
        free(pl.fills);                                                                               \
    } else free(pl.xb);                                                                               \
    free(pl.wsum); free(tot); free(plain); free(idx); free(sc);                                       \
}

PORT_DEFINE_MSM(pg1, fp_t, g1a_t, g1j_t, pq, PF_ZERO, PF_QONE)
PORT_DEFINE_MSM(pg2, fq2_t, g2a_t, g2j_t, pq2, PF2_ZERO, PF2_ONE)

/* Called from inside an OpenMP parallel region (as a task or from the single
 * thread): the MSM's work is spawned as tasks of the enclosing region. */
void port_msm_g1_tasks(g1j_t *out, const g1a_t *bases, const fp_t *scalars_std, size_t n, int threads) {
    if (n == 0) {
        g1j_set_inf(out);
        return;
    }
    port_pg1_msm_impl(out, bases, scalars_std, n, threads);
}

void port_msm_g2_tasks(g2j_t *out, const g2a_t *bases, const fp_t *scalars_std, size_t n, int threads) {
    if (n == 0) {
        g2j_set_inf(out);
        return;
    }
    port_pg2_msm_impl(out, bases, scalars_std, n, threads);
}

void port_msm_g1(g1j_t *out, const g1a_t *bases, const fp_t *scalars_std, size_t n) {
    int th = n_threads();
#pragma omp parallel
#pragma omp single
    port_msm_g1_tasks(out, bases, scalars_std, n, th);
}

void port_msm_g2(g2j_t *out, const g2a_t *bases, const fp_t *scalars_std, size_t n) {
    int th = n_threads();
#pragma omp parallel
#pragma omp single
    port_msm_g2_tasks(out, bases, scalars_std, n, th);
}
