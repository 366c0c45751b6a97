/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * The timed CPU baseline's iNTT -> coset -> NTT, restating
 * CpuNtt::intt_coset_ntt (crates/ntt/src/lib.rs:508-550) on its portable
 * path: the inverse runs decimation in frequency (natural in, bit-reversed
 * out, no 1/n), the table shift^bitrev(p)/n carries both the coset shift and
 * the deferred scale (build_coset :561-578), and the forward runs decimation
 * in time (bit-reversed in, natural out), so no permutation pass exists.  The
 * passes whose butterflies stay inside one aligned block of
 * CACHE_BLOCK = 2^11 elements -- the inverse's last, the table multiply and
 * the forward's first -- run per block in one sweep (:530-548); the passes
 * that cross blocks run over the whole vector, two radix-2 passes fused per
 * trip through memory.  Values are identical to the oracle's transform.
 */
#include "port.h"
#include <stdlib.h>
#include <string.h>

#define CACHE_BLOCK 2048
#define CACHE_LOG 11

struct port_ntt {
    int log_n;
    size_t n;
    fp_t *tw, *tw_inv;      /* omega^i, omega^-i for i < n/2 */
    fp_t *btw, *btw_inv;    /* the same for a 2^11 domain, for the in-block passes */
    fp_t *coset;            /* shift^bitrev(p) / n */
};

port_ntt *port_ntt_new(int log_n) {
    domain_t d;
    if (domain_init(&d, log_n) != 0) return NULL;
    port_ntt *t = calloc(1, sizeof *t);
    t->log_n = log_n;
    t->n = d.n;
    size_t h = d.n / 2 ? d.n / 2 : 1;
    t->tw = malloc(h * sizeof(fp_t));
    t->tw_inv = malloc(h * sizeof(fp_t));
    memcpy(t->tw, d.tw, (d.n / 2) * sizeof(fp_t));
    memcpy(t->tw_inv, d.tw_inv, (d.n / 2) * sizeof(fp_t));
    t->coset = malloc(d.n * sizeof(fp_t));
    memcpy(t->coset, d.coset, d.n * sizeof(fp_t));
    /* in-block twiddles: omega_2^11^i = omega_n^(i n / 2^11) */
    t->btw = malloc(CACHE_BLOCK / 2 * sizeof(fp_t));
    t->btw_inv = malloc(CACHE_BLOCK / 2 * sizeof(fp_t));
    if (log_n >= CACHE_LOG) {
        size_t st = d.n >> CACHE_LOG;
        for (size_t i = 0; i < CACHE_BLOCK / 2; i++) {
            t->btw[i] = d.tw[i * st];
            t->btw_inv[i] = d.tw_inv[i * st];
        }
    }
    domain_free(&d);
    return t;
}

void port_ntt_free(port_ntt *t) {
    if (!t) return;
    free(t->tw);
    free(t->tw_inv);
    free(t->btw);
    free(t->btw_inv);
    free(t->coset);
    free(t);
}

/* DIF butterfly: (u, v) -> (u + v, (u - v) w) */
static inline void dif_bf(fp_t *x, fp_t *y, const fp_t *w) {
    fp_t u = *x, v = *y, d;
    pr_add(x, &u, &v);
    pr_sub(&d, &u, &v);
    pr_mul(y, &d, w);
}

/* DIT butterfly: (u, v) -> (u + v w, u - v w) */
static inline void dit_bf(fp_t *x, fp_t *y, const fp_t *w) {
    fp_t u = *x, vw;
    pr_mul(&vw, y, w);
    pr_add(x, &u, &vw);
    pr_sub(y, &u, &vw);
}

/* In-block DIF passes (half len/2 .. 1), the coset multiply, in-block DIT
 * passes (half 1 .. len/2); btw / btw_inv hold the powers of a primitive
 * len-th root, so half h reads entry j len / (2h). */
static void block_fused(fp_t *blk, const fp_t *tab, const fp_t *btw_inv, const fp_t *btw, size_t len) {
    for (size_t half = len / 2; half >= 1; half >>= 1) {
        size_t st = len / (2 * half);
        for (size_t b = 0; b < len; b += 2 * half)
            for (size_t j = 0; j < half; j++) dif_bf(&blk[b + j], &blk[b + j + half], &btw_inv[j * st]);
    }
    for (size_t i = 0; i < len; i++) pr_mul(&blk[i], &blk[i], &tab[i]);
    for (size_t half = 1; half < len; half <<= 1) {
        size_t st = len / (2 * half);
        for (size_t b = 0; b < len; b += 2 * half)
            for (size_t j = 0; j < half; j++) dit_bf(&blk[b + j], &blk[b + j + half], &btw[j * st]);
    }
}

/* The outer passes' butterflies are handed out in units of UNIT consecutive
 * j of one group (every outer half is at least CACHE_BLOCK / 2 >= UNIT). */
#define UNIT 1024

/* One or two outer DIF passes (halves h and h/2) over groups of 2h elements. */
static void dif_outer(fp_t *a, size_t n, size_t h, int two, const fp_t *tw_inv) {
    const size_t groups = n / (2 * h), st1 = n / (2 * h);
    const size_t span = two ? h / 2 : h;           /* j range per group */
    const size_t per = span / UNIT, units = groups * per;
#pragma omp taskloop num_tasks(port_tasks())
    for (size_t u = 0; u < units; u++) {
        const size_t g = u / per, j0 = (u % per) * UNIT, b = g * 2 * h;
        if (!two) {
            for (size_t j = j0; j < j0 + UNIT; j++) dif_bf(&a[b + j], &a[b + j + h], &tw_inv[j * st1]);
            continue;
        }
        /* radix-4: halves h then h/2 on the elements j, j+h/2, j+h, j+3h/2 */
        const size_t q = h / 2, st2 = 2 * st1;
        for (size_t j = j0; j < j0 + UNIT; j++) {
            fp_t *x0 = &a[b + j], *x1 = &a[b + j + q], *x2 = &a[b + j + h], *x3 = &a[b + j + h + q];
            dif_bf(x0, x2, &tw_inv[j * st1]);
            dif_bf(x1, x3, &tw_inv[(j + q) * st1]);
            dif_bf(x0, x1, &tw_inv[j * st2]);
            dif_bf(x2, x3, &tw_inv[j * st2]);
        }
    }
}

/* One or two outer DIT passes (halves h and 2h) over groups of 2h (4h) elements. */
static void dit_outer(fp_t *a, size_t n, size_t h, int two, const fp_t *tw) {
    const size_t st1 = n / (2 * h);
    const size_t groups = two ? n / (4 * h) : n / (2 * h);
    const size_t per = h / UNIT, units = groups * per;
#pragma omp taskloop num_tasks(port_tasks())
    for (size_t u = 0; u < units; u++) {
        const size_t g = u / per, j0 = (u % per) * UNIT;
        if (!two) {
            const size_t b = g * 2 * h;
            for (size_t j = j0; j < j0 + UNIT; j++) dit_bf(&a[b + j], &a[b + j + h], &tw[j * st1]);
            continue;
        }
        /* radix-4: halves h then 2h on the elements j, j+h, j+2h, j+3h of a group of 4h */
        const size_t b = g * 4 * h, st2 = st1 / 2;
        for (size_t j = j0; j < j0 + UNIT; j++) {
            fp_t *x0 = &a[b + j], *x1 = &a[b + j + h], *x2 = &a[b + j + 2 * h], *x3 = &a[b + j + 3 * h];
            dit_bf(x0, x1, &tw[j * st1]);
            dit_bf(x2, x3, &tw[j * st1]);
            dit_bf(x0, x2, &tw[j * st2]);
            dit_bf(x1, x3, &tw[(j + h) * st2]);
        }
    }
}

void port_intt_coset_ntt_tasks(const port_ntt *t, fp_t *a) {
    const size_t n = t->n;
    if (n <= 1) {
        if (n == 1) pr_mul(&a[0], &a[0], &t->coset[0]);
        return;
    }
    if (n <= CACHE_BLOCK) {
        /* one block: the same passes with the domain's own twiddles */
        block_fused(a, t->coset, t->tw_inv, t->tw, n);
        return;
    }
    /* outer DIF passes: halves n/2 .. CACHE_BLOCK */
    size_t h = n / 2;
    while (h >= CACHE_BLOCK) {
        int two = h / 2 >= CACHE_BLOCK;
        dif_outer(a, n, h, two, t->tw_inv);
        h >>= two ? 2 : 1;
    }
    const size_t blocks = n / CACHE_BLOCK;
#pragma omp taskloop num_tasks(port_tasks())
    for (size_t b = 0; b < blocks; b++)
        block_fused(a + b * CACHE_BLOCK, t->coset + b * CACHE_BLOCK, t->btw_inv, t->btw, CACHE_BLOCK);
    /* outer DIT passes: halves CACHE_BLOCK .. n/2 */
    h = CACHE_BLOCK;
    while (h < n) {
        int two = 2 * h < n;
        dit_outer(a, n, h, two, t->tw);
        h <<= two ? 2 : 1;
    }
}

void port_intt_coset_ntt(const port_ntt *t, fp_t *a) {
#pragma omp parallel
#pragma omp single
    port_intt_coset_ntt_tasks(t, a);
}
