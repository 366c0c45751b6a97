/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * The evaluation domain and radix-2 NTTs over Fr, restating
 *   - Domain::new / group_gen / size_inv / proving_coset_shift / twiddles
 *     (crates/field/src/lib.rs:46-140): omega_n = TWO_ADIC_ROOT^(2^(28-log n)),
 *     coset shift = omega_{2n};
 *   - CpuNtt::ntt (crates/ntt/src/lib.rs:244-273, 415): natural order in and
 *     out, the inverse scaled by 1/n;
 *   - intt_to_bitrev / coset_scale_bitrev / ntt_from_bitrev and their fused
 *     form intt_coset_ntt (crates/ntt/src/lib.rs:429-578): DIF inverse to
 *     bit-reversed order, a[p] *= shift^bitrev(p)/n, DIT forward back to
 *     natural order;
 *   - distribute_powers (crates/ntt/src/lib.rs:582): a[i] *= shift^i.
 * The output of each is a field-element vector fixed by the mathematics
 * (a DFT), so pass order and blocking do not affect it.
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>

#define R (&FR)

/* omega_{2^28}: the multiplicative generator 5 raised to (r-1)/2^28 */
static fp_t two_adic_root(void) {
    uint64_t e[4];
    memcpy(e, FR.p, sizeof e);
    e[0] -= 1;   /* r - 1, r is odd so no borrow */
    for (int k = 0; k < 28; k++)
        for (int i = 0; i < 4; i++) e[i] = (e[i] >> 1) | (i < 3 ? (e[i + 1] << 63) : 0);
    fp_t g, root;
    fp_from_u64(R, &g, 5);
    fp_pow(R, &root, &g, e, 4);
    return root;
}

int domain_root(int log_n, fp_t *out) {
    if (log_n < 0 || log_n > 28) return -1;
    fp_t w = two_adic_root();
    for (int i = log_n; i < 28; i++) fp_sqr(R, &w, &w);
    *out = w;
    return 0;
}

static size_t bitrev(size_t x, int bits) {
    size_t r = 0;
    for (int i = 0; i < bits; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

int domain_init(domain_t *d, int log_n) {
    memset(d, 0, sizeof *d);
    if (log_n < 0 || log_n > 27) return -1;
    d->log_n = log_n;
    d->n = (size_t)1 << log_n;
    domain_root(log_n, &d->omega);
    fp_inv(R, &d->omega_inv, &d->omega);
    fp_t nn;
    fp_from_u64(R, &nn, d->n);
    fp_inv(R, &d->n_inv, &nn);
    domain_root(log_n + 1, &d->shift);
    size_t h = d->n / 2 ? d->n / 2 : 1;
    d->tw = malloc(h * sizeof(fp_t));
    d->tw_inv = malloc(h * sizeof(fp_t));
    d->tw[0] = FR.one;
    d->tw_inv[0] = FR.one;
    for (size_t i = 1; i < h; i++) {
        fp_mul(R, &d->tw[i], &d->tw[i - 1], &d->omega);
        fp_mul(R, &d->tw_inv[i], &d->tw_inv[i - 1], &d->omega_inv);
    }
    /* coset table in bit-reversed order: shift^bitrev(p) / n */
    d->coset = malloc(d->n * sizeof(fp_t));
    fp_t acc = d->n_inv;
    for (size_t i = 0; i < d->n; i++) {
        d->coset[bitrev(i, log_n)] = acc;
        fp_mul(R, &acc, &acc, &d->shift);
    }
    return 0;
}

void domain_free(domain_t *d) {
    free(d->tw);
    free(d->tw_inv);
    free(d->coset);
    memset(d, 0, sizeof *d);
}

void bitrev_permute(fp_t *a, size_t n) {
    int bits = 0;
    while (((size_t)1 << bits) < n) bits++;
    for (size_t i = 0; i < n; i++) {
        size_t j = bitrev(i, bits);
        if (j > i) { fp_t t = a[i]; a[i] = a[j]; a[j] = t; }
    }
}

/* decimation in time: bit-reversed input, natural output */
static void dit(fp_t *a, size_t n, const fp_t *tw) {
    for (size_t half = 1; half < n; half <<= 1) {
        size_t step = n / (2 * half);
        long nblocks = (long)(n / (2 * half));
#pragma omp parallel for schedule(static) if (n >= 4096)
        for (long b = 0; b < nblocks; b++) {
            size_t k = (size_t)b * 2 * half;
            for (size_t j = 0; j < half; j++) {
                fp_t u = a[k + j], v;
                fp_mul(R, &v, &a[k + j + half], &tw[j * step]);
                fp_add(R, &a[k + j], &u, &v);
                fp_sub(R, &a[k + j + half], &u, &v);
            }
        }
    }
}

/* decimation in frequency: natural input, bit-reversed output */
static void dif(fp_t *a, size_t n, const fp_t *tw) {
    for (size_t half = n / 2; half >= 1; half >>= 1) {
        size_t step = n / (2 * half);
        long nblocks = (long)(n / (2 * half));
#pragma omp parallel for schedule(static) if (n >= 4096)
        for (long b = 0; b < nblocks; b++) {
            size_t k = (size_t)b * 2 * half;
            for (size_t j = 0; j < half; j++) {
                fp_t u = a[k + j], v = a[k + j + half], d;
                fp_add(R, &a[k + j], &u, &v);
                fp_sub(R, &d, &u, &v);
                fp_mul(R, &a[k + j + half], &d, &tw[j * step]);
            }
        }
        if (half == 1) break;
    }
}

void ntt_forward(const domain_t *d, fp_t *a) {
    if (d->n <= 1) return;
    bitrev_permute(a, d->n);
    dit(a, d->n, d->tw);
}

void ntt_inverse(const domain_t *d, fp_t *a) {
    if (d->n <= 1) return;
    bitrev_permute(a, d->n);
    dit(a, d->n, d->tw_inv);
#pragma omp parallel for schedule(static) if (d->n >= 4096)
    for (long i = 0; i < (long)d->n; i++) fp_mul(R, &a[i], &a[i], &d->n_inv);
}

void distribute_powers(fp_t *a, size_t n, const fp_t *shift) {
    fp_t acc = FR.one;
    for (size_t i = 0; i < n; i++) {
        fp_mul(R, &a[i], &a[i], &acc);
        fp_mul(R, &acc, &acc, shift);
    }
}

void intt_coset_ntt(const domain_t *d, fp_t *a) {
    size_t n = d->n;
    if (n <= 1) {
        /* size 1: iNTT and NTT are the identity, the coset table entry is 1/n = 1 */
        return;
    }
    dif(a, n, d->tw_inv);
#pragma omp parallel for schedule(static) if (n >= 4096)
    for (long i = 0; i < (long)n; i++) fp_mul(R, &a[i], &a[i], &d->coset[i]);
    dit(a, n, d->tw);
}
