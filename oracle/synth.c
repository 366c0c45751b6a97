/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * The synthetic workload's inputs, generated on the oracle's side so that the
 * timed reference arm runs without the product library: a restatement of the
 * seeded circuit, witness and .zkey generator the benchmarks are defined by.
 * The same seeds give the same bytes as the product's generator (the CPU
 * tests compare the two), so both provers read identical inputs.
 *
 * Circuit (seed): wire 0 = 1, n_inputs input wires (the first n_public
 * public), one new wire per constraint w_k = (A.w)(B.w).  Each constraint is
 * given a value class up front -- 0 (30%), 1 (30%), a 16-bit value (10%), a
 * 32-bit value (10%), uniform (20%) -- and its rows are shaped so the product
 * lands in that class for every choice of inputs; extra terms sit on zero
 * wires (coefficients uniform in Fr or +-1), so they change no value.
 *
 * Key (toxic seed): tau, alpha, beta, delta drawn from the seed, gamma = 1,
 * the snarkjs zkey_new + zkey_contribute semantics as the reference restates
 * them (crates/ceremony/src/setup.rs:16-20, 125-170, 835-846):
 *   domain n = 2^(floor(log2(n_constraints + n_public)) + 1);
 *   one extra A row per public signal j (row n_constraints + j, coefficient 1);
 *   A_j = [u_j(tau)]_1, B1_j = [v_j(tau)]_1, B2_j = [v_j(tau)]_2;
 *   IC_j = [beta u_j + alpha v_j + w_j]_1 (j <= n_public);
 *   L_j = [(beta u_j + alpha v_j + w_j) / delta]_1 (private wires);
 *   H_i = [L^(2n)_(2i+1)(tau) / delta]_1, the odd Lagrange basis of 2n;
 *   section 4 the A and B coefficients as double-Montgomery records;
 *   sections in snarkjs order 1, 2, 4, 3, 9, 8, 5, 6, 7, 10.
 * Fixed-base points are sums of 8-bit-window table entries in XYZZ,
 * normalised with one inversion per run of points (Montgomery's trick).
 */
#include "port.h"
#include "port_curve.h"
#include <stdlib.h>
#include <string.h>

/* ---- SplitMix64 and the draws made from it ---- */
typedef struct { uint64_t s; } smix_t;

static uint64_t sm_next(smix_t *r) {
    r->s += 0x9E3779B97F4A7C15ULL;
    uint64_t z = r->s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double sm_uniform(smix_t *r) { return (double)(sm_next(r) >> 11) * (1.0 / 9007199254740992.0); }
static uint32_t sm_below(smix_t *r, uint32_t n) { return (uint32_t)(((unsigned __int128)sm_next(r) * n) >> 64); }

static int ge_r(const uint64_t *v) {
    for (int i = 3; i >= 0; i--) {
        if (v[i] != FR.p[i]) return v[i] > FR.p[i];
    }
    return 1;
}
static void sub_r(uint64_t *v) {
    unsigned __int128 d;
    uint64_t bw = 0;
    for (int i = 0; i < 4; i++) {
        d = (unsigned __int128)v[i] - FR.p[i] - bw;
        v[i] = (uint64_t)d;
        bw = (uint64_t)(d >> 64) & 1;
    }
}
/* uniform in [0, r): 254 random bits, one conditional subtraction; Montgomery out */
static fp_t sm_fr(smix_t *r) {
    fp_t s;   /* C leaves the order of initializer evaluations open: draw the limbs in order */
    s.v[0] = sm_next(r);
    s.v[1] = sm_next(r);
    s.v[2] = sm_next(r);
    s.v[3] = sm_next(r) & ((1ULL << 62) - 1);
    if (ge_r(s.v)) sub_r(s.v);
    fp_t m;
    fp_to_mont(&FR, &m, &s);
    return m;
}
static fp_t sm_fr_nonzero(smix_t *r) {
    for (;;) {
        fp_t x = sm_fr(r);
        if (!pf_is_zero(&x)) return x;
    }
}

/* ---- the circuit ---- */
enum { C_ZERO = 0, C_ONE = 1, C_S16 = 2, C_S32 = 3, C_UNIF = 4 };

typedef struct { uint32_t sig; fp_t coef; } term_t;
typedef struct { uint32_t *v; size_t n, cap; } vec_u32;
typedef struct { term_t *v; size_t n, cap; } vec_term;

static void vu_push(vec_u32 *a, uint32_t x) {
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 64;
        a->v = realloc(a->v, a->cap * sizeof *a->v);
    }
    a->v[a->n++] = x;
}
static void vt_push(vec_term *a, uint32_t sig, fp_t coef) {
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 64;
        a->v = realloc(a->v, a->cap * sizeof *a->v);
    }
    a->v[a->n].sig = sig;
    a->v[a->n].coef = coef;
    a->n++;
}

typedef struct {
    uint32_t n_constraints, n_inputs, n_public, n_vars, domain;
    uint32_t *ptr[2];   /* CSR by constraint */
    vec_term terms[2];
} osynth_t;

typedef struct {
    smix_t *rng;
    vec_u32 *pool;
    fp_t one, minus_one;
} gen_ctx;

static fp_t draw_coef(gen_ctx *g) {
    if (sm_next(g->rng) & 1) return sm_fr(g->rng);
    return (sm_next(g->rng) & 1) ? g->one : g->minus_one;
}
static uint32_t pick(gen_ctx *g, int c) { return g->pool[c].v[sm_below(g->rng, (uint32_t)g->pool[c].n)]; }
static void fill_zeros(gen_ctx *g, vec_term *row, size_t lo, uint32_t want) {
    while (row->n - lo < want && g->pool[C_ZERO].n) {
        uint32_t s = pick(g, C_ZERO);
        vt_push(row, s, draw_coef(g));
    }
}
static void fill_any(gen_ctx *g, vec_term *row, size_t lo, uint32_t want, uint32_t below) {
    while (row->n - lo < want) {
        uint32_t s = sm_below(g->rng, below);
        vt_push(row, s, draw_coef(g));
    }
}

void *oracle_synth_new(uint64_t seed, uint32_t n_constraints, uint32_t n_inputs, uint32_t n_public) {
    if (!n_constraints || !n_inputs || n_public > n_inputs) return NULL;
    bn254_init();
    osynth_t *s = calloc(1, sizeof *s);
    s->n_constraints = n_constraints;
    s->n_inputs = n_inputs;
    s->n_public = n_public;
    s->n_vars = 1 + n_inputs + n_constraints;
    uint64_t total = (uint64_t)n_constraints + n_public;
    int p = 0;
    while ((1ULL << (p + 1)) <= total) p++;
    s->domain = 1u << (p + 1);
    smix_t rng = {seed};
    vec_u32 pool[5] = {{0}};
    gen_ctx g = {&rng, pool, FR.one, FR.one};
    fp_neg(&FR, &g.minus_one, &FR.one);
    vu_push(&pool[C_ONE], 0);
    for (uint32_t i = 1; i <= n_inputs; i++) vu_push(&pool[C_UNIF], i);
    for (int m = 0; m < 2; m++) {
        s->ptr[m] = malloc(((size_t)n_constraints + 1) * sizeof(uint32_t));
        s->ptr[m][0] = 0;
    }
    vec_term *A = &s->terms[0], *B = &s->terms[1];
    for (uint32_t k = 0; k < n_constraints; k++) {
        uint32_t out = 1 + n_inputs + k;
        double r = sm_uniform(&rng);
        int cls = r < 0.30 ? C_ZERO : r < 0.60 ? C_ONE : r < 0.70 ? C_S16 : r < 0.80 ? C_S32 : C_UNIF;
        if (cls == C_ZERO && pool[C_ONE].n < 2) cls = C_ONE;
        if (cls == C_S32 && pool[C_S16].n == 0) cls = C_S16;
        uint32_t na = 2 + (uint32_t)(sm_next(&rng) & 1);
        uint32_t nb = 2 + (uint32_t)(sm_next(&rng) & 1);
        size_t a0 = A->n, b0 = B->n;
        switch (cls) {
            case C_ONE:
                vt_push(A, pick(&g, C_ONE), g.one);
                vt_push(B, pick(&g, C_ONE), g.one);
                fill_zeros(&g, A, a0, na);
                fill_zeros(&g, B, b0, nb);
                break;
            case C_ZERO: {
                uint32_t o1 = pick(&g, C_ONE), o2;
                do o2 = pick(&g, C_ONE);
                while (o2 == o1);
                vt_push(A, o1, g.one);
                vt_push(A, o2, g.minus_one);
                fill_zeros(&g, A, a0, na);
                fill_any(&g, B, b0, nb, out);
                break;
            }
            case C_S16: {
                uint64_t v = 2 + sm_below(&rng, (1u << 16) - 2);
                fp_t cv;
                fp_from_u64(&FR, &cv, v);
                vt_push(A, pick(&g, C_ONE), cv);
                vt_push(B, pick(&g, C_ONE), g.one);
                fill_zeros(&g, A, a0, na);
                fill_zeros(&g, B, b0, nb);
                break;
            }
            case C_S32:
                vt_push(A, pick(&g, C_S16), g.one);
                vt_push(B, pick(&g, C_S16), g.one);
                fill_zeros(&g, A, a0, na);
                fill_zeros(&g, B, b0, nb);
                break;
            default: {
                uint32_t sa = pick(&g, C_UNIF);
                fp_t ca = sm_fr_nonzero(&rng);
                vt_push(A, sa, ca);
                uint32_t sb = pick(&g, C_UNIF);
                fp_t cb = sm_fr_nonzero(&rng);
                vt_push(B, sb, cb);
                fill_any(&g, A, a0, na, out);
                fill_any(&g, B, b0, nb, out);
                break;
            }
        }
        vu_push(&pool[cls], out);
        s->ptr[0][k + 1] = (uint32_t)A->n;
        s->ptr[1][k + 1] = (uint32_t)B->n;
    }
    for (int c = 0; c < 5; c++) free(pool[c].v);
    return s;
}

void oracle_synth_free(void *sv) {
    osynth_t *s = sv;
    if (!s) return;
    for (int m = 0; m < 2; m++) {
        free(s->ptr[m]);
        free(s->terms[m].v);
    }
    free(s);
}

void oracle_synth_info(const void *sv, uint32_t *out2) {
    const osynth_t *s = sv;
    out2[0] = s->n_vars;
    out2[1] = s->domain;
}

static fp_t row_dot(const osynth_t *s, int m, uint32_t k, const fp_t *w) {
    fp_t acc = {{0, 0, 0, 0}};
    for (uint32_t t = s->ptr[m][k]; t < s->ptr[m][k + 1]; t++) {
        fp_t p;
        pr_mul(&p, &s->terms[m].v[t].coef, &w[s->terms[m].v[t].sig]);
        pr_add(&acc, &acc, &p);
    }
    return acc;
}

/* n_vars Montgomery Fr: inputs from the witness seed, then w_k = (A_k.w)(B_k.w) */
void oracle_synth_witness(const void *sv, uint64_t wseed, uint8_t *out) {
    const osynth_t *s = sv;
    smix_t rng = {wseed ^ 0x5bd1e995a3c5f7e1ULL};
    fp_t *w = (fp_t *)out;
    memset(w, 0, (size_t)s->n_vars * sizeof(fp_t));
    w[0] = FR.one;
    for (uint32_t i = 1; i <= s->n_inputs; i++) w[i] = sm_fr(&rng);
    for (uint32_t k = 0; k < s->n_constraints; k++) {
        fp_t a = row_dot(s, 0, k, w), b = row_dot(s, 1, k, w);
        pr_mul(&w[1 + s->n_inputs + k], &a, &b);
    }
}

/* ---- fixed-base multiplication: table[w][d] = d 2^(8w) G, affine ---- */
#define FB_RUN 256

static void fr_to_std(const fp_t *m, uint64_t out[4]) {
    static const fp_t one_std = {{1, 0, 0, 0}};
    fp_t s;
    pr_mul(&s, m, &one_std);
    memcpy(out, s.v, 32);
}

/* affine (x, y) = (X / ZZ, Y / ZZZ) for a run of XYZZ points sharing one inversion */
#define DEFINE_NORMALIZE(G, F, P, ONE_F)                                                              \
typedef struct { F x, y; } G##_aff;                                                                \
static void G##_normalize(const G##_xyzz *in, G##_aff *out, size_t n) {                             \
    F *pre = malloc((n ? n : 1) * sizeof(F));                                                       \
    F acc = ONE_F;                                                                                  \
    for (size_t i = 0; i < n; i++) {                                                                \
        pre[i] = acc;                                                                               \
        if (!G##_is_id(&in[i])) { F d; P##_mul(&d, &in[i].zz, &in[i].zzz); P##_mul(&acc, &acc, &d); } \
    }                                                                                               \
    F inv;                                                                                          \
    P##_inv(&inv, &acc);                                                                            \
    for (size_t i = n; i-- > 0;) {                                                                  \
        if (G##_is_id(&in[i])) { memset(&out[i], 0, sizeof out[i]); continue; }                     \
        F d, id, t;                                                                                 \
        P##_mul(&d, &in[i].zz, &in[i].zzz);                                                         \
        P##_mul(&id, &inv, &pre[i]);      /* 1 / (ZZ ZZZ) */                                        \
        P##_mul(&inv, &inv, &d);                                                                    \
        P##_mul(&t, &id, &in[i].zzz);     /* 1 / ZZ */                                              \
        P##_mul(&out[i].x, &in[i].x, &t);                                                           \
        P##_mul(&t, &id, &in[i].zz);      /* 1 / ZZZ */                                             \
        P##_mul(&out[i].y, &in[i].y, &t);                                                           \
    }                                                                                               \
    free(pre);                                                                                      \
}

DEFINE_NORMALIZE(pg1, fp_t, pq, PF_QONE)
DEFINE_NORMALIZE(pg2, fq2_t, pq2, PF2_ONE)

static void pack_aff1(uint8_t *o, const pg1_aff *a) {
    memcpy(o, a->x.v, 32);
    memcpy(o + 32, a->y.v, 32);
}
static void pack_aff2(uint8_t *o, const pg2_aff *a) {
    memcpy(o, a->x.c0.v, 32);
    memcpy(o + 32, a->x.c1.v, 32);
    memcpy(o + 64, a->y.c0.v, 32);
    memcpy(o + 96, a->y.c1.v, 32);
}

/* table[w][d] = d 2^(8w) G affine; out[i] = k_i G packed (infinity all-zero), k_i Montgomery Fr */
#define DEFINE_FIXED_BASE(G, F, AFF, P, PACK, PB, ONE_F)                                              \
static G##_aff *G##_table(const AFF *gen) {                                                         \
    G##_aff *t = malloc(32 * 256 * sizeof(G##_aff));                                                \
    G##_xyzz *tmp = malloc(32 * 256 * sizeof(G##_xyzz));                                            \
    G##_xyzz base;                                                                                  \
    base.x = gen->x; base.y = gen->y; base.zz = ONE_F; base.zzz = ONE_F;                            \
    for (int w = 0; w < 32; w++) {                                                                  \
        G##_xyzz cur;                                                                               \
        G##_set_id(&cur);                                                                           \
        for (int d = 0; d < 256; d++) {                                                             \
            tmp[w * 256 + d] = cur;                                                                 \
            G##_add(&cur, &base);                                                                   \
        }                                                                                           \
        for (int k = 0; k < 8; k++) { G##_xyzz b2; G##_dbl(&b2, &base); base = b2; }               \
    }                                                                                               \
    G##_normalize(tmp, t, 32 * 256);                                                                \
    free(tmp);                                                                                      \
    return t;                                                                                       \
}                                                                                                   \
static void G##_points(const G##_aff *tab, const fp_t *k, size_t n, uint8_t *out) {                \
    _Pragma("omp parallel for schedule(dynamic, 1)")                                                \
    for (long r = 0; r < (long)((n + FB_RUN - 1) / FB_RUN); r++) {                                  \
        size_t lo = (size_t)r * FB_RUN, hi = lo + FB_RUN < n ? lo + FB_RUN : n;                     \
        G##_xyzz acc[FB_RUN];                                                                       \
        G##_aff res[FB_RUN];                                                                        \
        for (size_t i = lo; i < hi; i++) {                                                          \
            uint64_t s[4];                                                                          \
            fr_to_std(&k[i], s);                                                                    \
            G##_set_id(&acc[i - lo]);                                                               \
            for (int w = 0; w < 32; w++) {                                                          \
                unsigned d = (unsigned)((s[w >> 3] >> (8 * (w & 7))) & 255u);                       \
                if (d) G##_madd(&acc[i - lo], &tab[w * 256 + d].x, &tab[w * 256 + d].y);             \
            }                                                                                       \
        }                                                                                           \
        G##_normalize(acc, res, hi - lo);                                                           \
        for (size_t i = lo; i < hi; i++) {                                                          \
            if (G##_is_id(&acc[i - lo])) memset(out + i * (PB), 0, PB);                             \
            else PACK(out + i * (PB), &res[i - lo]);                                                \
        }                                                                                           \
    }                                                                                               \
}

DEFINE_FIXED_BASE(pg1, fp_t, g1a_t, pq, pack_aff1, 64, PF_QONE)
DEFINE_FIXED_BASE(pg2, fq2_t, g2a_t, pq2, pack_aff2, 128, PF2_ONE)

/* ---- the .zkey (iden3 binfile) ---- */
typedef struct { uint8_t *b; size_t n, cap, sec; } bw_t;

static void bw_bytes(bw_t *w, const void *p, size_t n) {
    if (w->n + n > w->cap) {
        while (w->n + n > w->cap) w->cap = w->cap ? 2 * w->cap : 1 << 20;
        w->b = realloc(w->b, w->cap);
    }
    memcpy(w->b + w->n, p, n);
    w->n += n;
}
static uint8_t *bw_reserve(bw_t *w, size_t n) {
    if (w->n + n > w->cap) {
        while (w->n + n > w->cap) w->cap = w->cap ? 2 * w->cap : 1 << 20;
        w->b = realloc(w->b, w->cap);
    }
    uint8_t *p = w->b + w->n;
    w->n += n;
    return p;
}
static void bw_u32(bw_t *w, uint32_t x) { bw_bytes(w, &x, 4); }
static void bw_section(bw_t *w, uint32_t id) {
    uint64_t z = 0;
    bw_u32(w, id);
    w->sec = w->n;
    bw_bytes(w, &z, 8);
}
static void bw_end(bw_t *w) {
    uint64_t l = w->n - w->sec - 8;
    memcpy(w->b + w->sec, &l, 8);
}

static void batch_inv_fr(fp_t *v, size_t n) {
    fp_t *pre = malloc((n ? n : 1) * sizeof(fp_t)), run = FR.one, iv;
    for (size_t i = 0; i < n; i++) {
        pre[i] = run;
        pr_mul(&run, &run, &v[i]);
    }
    fp_inv(&FR, &iv, &run);
    for (size_t i = n; i-- > 0;) {
        fp_t x;
        pr_mul(&x, &iv, &pre[i]);
        pr_mul(&iv, &iv, &v[i]);
        v[i] = x;
    }
    free(pre);
}

static fp_t pow_u64(const fp_t *a, uint64_t e) {
    uint64_t ee[1] = {e};
    fp_t r;
    fp_pow(&FR, &r, a, ee, 1);
    return r;
}

/* The .zkey bytes for the toxic seed; *len_out gets their count.  The
 * caller frees the buffer with oracle_synth_buffer_free. */
uint8_t *oracle_synth_zkey(const void *sv, uint64_t toxic_seed, size_t *len_out) {
    const osynth_t *s = sv;
    smix_t rng = {toxic_seed ^ 0x243F6A8885A308D3ULL};
    const uint32_t n = s->domain, nv = s->n_vars, npub = s->n_public, nc = s->n_constraints;
    int log_n = 0;
    while ((1u << log_n) < n) log_n++;
    fp_t omega, shift;
    domain_root(log_n, &omega);
    domain_root(log_n + 1, &shift);
    fp_t tau, alpha, beta, delta;
    for (;;) {
        tau = sm_fr_nonzero(&rng);
        alpha = sm_fr_nonzero(&rng);
        beta = sm_fr_nonzero(&rng);
        delta = sm_fr_nonzero(&rng);
        fp_t t2n = pow_u64(&tau, 2ULL * n);
        if (!pf_eq(&t2n, &FR.one)) break;   /* tau must avoid the 2n-th roots of unity */
    }
    /* L_c(tau) = (tau^n - 1)/n * omega^c / (tau - omega^c) */
    fp_t *L = malloc((size_t)n * sizeof(fp_t)), *den = malloc((size_t)n * sizeof(fp_t)),
         *pw = malloc((size_t)n * sizeof(fp_t));
    fp_t zt = pow_u64(&tau, n), nn, factor, wc = FR.one;
    pr_sub(&zt, &zt, &FR.one);
    fp_from_u64(&FR, &nn, n);
    fp_inv(&FR, &nn, &nn);
    pr_mul(&factor, &zt, &nn);
    for (uint32_t c = 0; c < n; c++) {
        pw[c] = wc;
        pr_sub(&den[c], &tau, &wc);
        pr_mul(&wc, &wc, &omega);
    }
    batch_inv_fr(den, n);
    for (uint32_t c = 0; c < n; c++) {
        pr_mul(&L[c], &factor, &pw[c]);
        pr_mul(&L[c], &L[c], &den[c]);
    }
    fp_t *u = calloc(nv, sizeof(fp_t)), *v = calloc(nv, sizeof(fp_t)), *wq = calloc(nv, sizeof(fp_t));
    for (uint32_t k = 0; k < nc; k++) {
        for (uint32_t t = s->ptr[0][k]; t < s->ptr[0][k + 1]; t++) {
            fp_t p;
            pr_mul(&p, &s->terms[0].v[t].coef, &L[k]);
            pr_add(&u[s->terms[0].v[t].sig], &u[s->terms[0].v[t].sig], &p);
        }
        for (uint32_t t = s->ptr[1][k]; t < s->ptr[1][k + 1]; t++) {
            fp_t p;
            pr_mul(&p, &s->terms[1].v[t].coef, &L[k]);
            pr_add(&v[s->terms[1].v[t].sig], &v[s->terms[1].v[t].sig], &p);
        }
        pr_add(&wq[1 + s->n_inputs + k], &wq[1 + s->n_inputs + k], &L[k]);
    }
    for (uint32_t j = 0; j <= npub; j++) pr_add(&u[j], &u[j], &L[nc + j]);
    fp_t dinv;
    fp_inv(&FR, &dinv, &delta);
    fp_t *ic_s = malloc(((size_t)npub + 1) * sizeof(fp_t)), *l_s = malloc((size_t)(nv - npub - 1) * sizeof(fp_t) + 32);
    for (uint32_t j = 0; j < nv; j++) {
        fp_t x, y;
        pr_mul(&x, &beta, &u[j]);
        pr_mul(&y, &alpha, &v[j]);
        pr_add(&x, &x, &y);
        pr_add(&x, &x, &wq[j]);
        if (j <= npub) ic_s[j] = x;
        else pr_mul(&l_s[j - npub - 1], &x, &dinv);
    }
    /* H_i = (tau^2n - 1)/(2n) * x_i / (tau - x_i) / delta, x_i = shift omega^i */
    fp_t f2 = pow_u64(&tau, 2ULL * n), n2;
    pr_sub(&f2, &f2, &FR.one);
    fp_from_u64(&FR, &n2, 2ULL * n);
    fp_inv(&FR, &n2, &n2);
    pr_mul(&f2, &f2, &n2);
    pr_mul(&f2, &f2, &dinv);
    fp_t *h_s = malloc((size_t)n * sizeof(fp_t)), xi = shift;
    for (uint32_t i = 0; i < n; i++) {
        pw[i] = xi;
        pr_sub(&den[i], &tau, &xi);
        pr_mul(&xi, &xi, &omega);
    }
    batch_inv_fr(den, n);
    for (uint32_t i = 0; i < n; i++) {
        pr_mul(&h_s[i], &f2, &pw[i]);
        pr_mul(&h_s[i], &h_s[i], &den[i]);
    }
    free(L);
    free(den);
    free(pw);

    pg1_aff *t1 = pg1_table(&G1_GEN);
    pg2_aff *t2 = pg2_table(&G2_GEN);
    bw_t w = {0};
    bw_bytes(&w, "zkey", 4);
    bw_u32(&w, 1);
    bw_u32(&w, 10);
    bw_section(&w, 1);
    bw_u32(&w, 1);
    bw_end(&w);
    bw_section(&w, 2);
    bw_u32(&w, 32);
    bw_bytes(&w, FQ.p, 32);
    bw_u32(&w, 32);
    bw_bytes(&w, FR.p, 32);
    bw_u32(&w, nv);
    bw_u32(&w, npub);
    bw_u32(&w, n);
    fp_t one = FR.one;
    pg1_points(t1, &alpha, 1, bw_reserve(&w, 64));
    pg1_points(t1, &beta, 1, bw_reserve(&w, 64));
    pg2_points(t2, &beta, 1, bw_reserve(&w, 128));
    pg2_points(t2, &one, 1, bw_reserve(&w, 128));   /* gamma = 1 */
    pg1_points(t1, &delta, 1, bw_reserve(&w, 64));
    pg2_points(t2, &delta, 1, bw_reserve(&w, 128));
    bw_end(&w);
    /* 4: coefficients, each stored as coef R^2 (its Montgomery limbs taken as standard, times R) */
    bw_section(&w, 4);
    bw_u32(&w, (uint32_t)(s->terms[0].n + s->terms[1].n + npub + 1));
    for (int m = 0; m < 2; m++)
        for (uint32_t k = 0; k < nc; k++)
            for (uint32_t t = s->ptr[m][k]; t < s->ptr[m][k + 1]; t++) {
                fp_t stored;
                fp_to_mont(&FR, &stored, &s->terms[m].v[t].coef);
                bw_u32(&w, (uint32_t)m);
                bw_u32(&w, k);
                bw_u32(&w, s->terms[m].v[t].sig);
                bw_bytes(&w, stored.v, 32);
            }
    for (uint32_t j = 0; j <= npub; j++) {
        fp_t stored;
        fp_to_mont(&FR, &stored, &FR.one);
        bw_u32(&w, 0);
        bw_u32(&w, nc + j);
        bw_u32(&w, j);
        bw_bytes(&w, stored.v, 32);
    }
    bw_end(&w);
    struct { uint32_t id; int g2; const fp_t *k; size_t cnt; } secs[] = {
        {3, 0, ic_s, (size_t)npub + 1}, {9, 0, h_s, n}, {8, 0, l_s, (size_t)nv - npub - 1},
        {5, 0, u, nv}, {6, 0, v, nv}, {7, 1, v, nv},
    };
    for (size_t i = 0; i < sizeof secs / sizeof secs[0]; i++) {
        bw_section(&w, secs[i].id);
        uint8_t *dst = bw_reserve(&w, secs[i].cnt * (secs[i].g2 ? 128 : 64));
        if (secs[i].g2) pg2_points(t2, secs[i].k, secs[i].cnt, dst);
        else pg1_points(t1, secs[i].k, secs[i].cnt, dst);
        bw_end(&w);
    }
    bw_section(&w, 10);
    uint8_t zero64[64] = {0};
    bw_bytes(&w, zero64, 64);
    bw_u32(&w, 0);
    bw_end(&w);
    free(t1);
    free(t2);
    free(u);
    free(v);
    free(wq);
    free(ic_s);
    free(l_s);
    free(h_s);
    *len_out = w.n;
    return w.b;
}

void oracle_synth_buffer_free(uint8_t *b) { free(b); }
