/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Montgomery arithmetic over BN254's Fr and Fq with R = 2^256, restating
 * snarkrs' raw field layer (crates/field/src/raw.rs:59-76 moduli and n0,
 * :186 CIOS; results always fully reduced into [0, p), raw.rs:382-560), and
 * the Fq2/Fq6/Fq12 tower the pairing needs (u^2 = -1, xi = 9 + u,
 * crates/cuda/src/kernels/bn254_curve.cuh:300-378 for Fq2).
 */
#include "bn254.h"
#include <string.h>

typedef unsigned __int128 u128;

field_t FR = {{0x43e1f593f0000001ULL, 0x2833e84879b97091ULL,
               0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0, {{0}}, {{0}}};
field_t FQ = {{0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL,
               0xb85045b68181585dULL, 0x30644e72e131a029ULL}, 0, {{0}}, {{0}}};

static int geq_p(const uint64_t *a, const uint64_t *p) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] > p[i]) return 1;
        if (a[i] < p[i]) return 0;
    }
    return 1;
}

static uint64_t sub4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    uint64_t borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        r[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) ? 1 : 0;
    }
    return borrow;
}

static uint64_t add4(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    uint64_t carry = 0;
    for (int i = 0; i < 4; i++) {
        u128 s = (u128)a[i] + b[i] + carry;
        r[i] = (uint64_t)s;
        carry = (uint64_t)(s >> 64);
    }
    return carry;
}

void fp_add(const field_t *f, fp_t *r, const fp_t *a, const fp_t *b) {
    uint64_t t[4];
    uint64_t c = add4(t, a->v, b->v);
    if (c || geq_p(t, f->p)) sub4(t, t, f->p);
    memcpy(r->v, t, sizeof t);
}

void fp_sub(const field_t *f, fp_t *r, const fp_t *a, const fp_t *b) {
    uint64_t t[4];
    if (sub4(t, a->v, b->v)) add4(t, t, f->p);
    memcpy(r->v, t, sizeof t);
}

void fp_neg(const field_t *f, fp_t *r, const fp_t *a) {
    if (fp_is_zero(a)) { memset(r, 0, sizeof *r); return; }
    sub4(r->v, f->p, a->v);
}

/* CIOS Montgomery product: a*b*R^-1 mod p, inputs and output in [0, p). */
void fp_mul(const field_t *f, fp_t *r, const fp_t *a, const fp_t *b) {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        uint64_t carry = 0;
        for (int j = 0; j < 4; j++) {
            u128 uv = (u128)a->v[j] * b->v[i] + t[j] + carry;
            t[j] = (uint64_t)uv;
            carry = (uint64_t)(uv >> 64);
        }
        u128 s = (u128)t[4] + carry;
        t[4] = (uint64_t)s;
        t[5] = (uint64_t)(s >> 64);
        uint64_t m = t[0] * f->n0;
        u128 uv = (u128)m * f->p[0] + t[0];
        carry = (uint64_t)(uv >> 64);
        for (int j = 1; j < 4; j++) {
            uv = (u128)m * f->p[j] + t[j] + carry;
            t[j - 1] = (uint64_t)uv;
            carry = (uint64_t)(uv >> 64);
        }
        s = (u128)t[4] + carry;
        t[3] = (uint64_t)s;
        t[4] = t[5] + (uint64_t)(s >> 64);
    }
    if (t[4] || geq_p(t, f->p)) sub4(t, t, f->p);
    memcpy(r->v, t, 32);
}

void fp_sqr(const field_t *f, fp_t *r, const fp_t *a) { fp_mul(f, r, a, a); }

int fp_is_zero(const fp_t *a) { return (a->v[0] | a->v[1] | a->v[2] | a->v[3]) == 0; }

int fp_eq(const fp_t *a, const fp_t *b) { return memcmp(a->v, b->v, 32) == 0; }

int fp_lt_modulus(const field_t *f, const fp_t *raw) { return !geq_p(raw->v, f->p); }

void fp_to_mont(const field_t *f, fp_t *r, const fp_t *s) { fp_mul(f, r, s, &f->r2); }

void fp_from_mont(const field_t *f, fp_t *r, const fp_t *m) {
    fp_t one = {{1, 0, 0, 0}};
    fp_mul(f, r, m, &one);
}

void fp_from_u64(const field_t *f, fp_t *r, uint64_t x) {
    fp_t s = {{x, 0, 0, 0}};
    fp_to_mont(f, r, &s);
}

/* left-to-right square and multiply over a little-endian u64 exponent */
void fp_pow(const field_t *f, fp_t *r, const fp_t *a, const uint64_t *e, int nlimbs) {
    fp_t acc = f->one, base = *a;
    for (int i = nlimbs * 64 - 1; i >= 0; i--) {
        fp_sqr(f, &acc, &acc);
        if ((e[i / 64] >> (i % 64)) & 1) fp_mul(f, &acc, &acc, &base);
    }
    *r = acc;
}

void fp_inv(const field_t *f, fp_t *r, const fp_t *a) {
    /* Fermat: a^(p-2) */
    uint64_t e[4];
    uint64_t two[4] = {2, 0, 0, 0};
    sub4(e, f->p, two);
    fp_pow(f, r, a, e, 4);
}

/* q = 3 mod 4: sqrt(a) = a^((q+1)/4); returns 0 when a is a non-residue. */
int fp_sqrt(const field_t *f, fp_t *r, const fp_t *a) {
    uint64_t e[4], one[4] = {1, 0, 0, 0};
    add4(e, f->p, one);
    /* (p+1)/4: shift right by 2 */
    for (int i = 0; i < 4; i++) e[i] = (e[i] >> 2) | (i < 3 ? (e[i + 1] << 62) : 0);
    fp_t s, chk;
    fp_pow(f, &s, a, e, 4);
    fp_sqr(f, &chk, &s);
    if (!fp_eq(&chk, a)) return 0;
    *r = s;
    return 1;
}

static void compute_consts(field_t *f) {
    /* n0 = -p^-1 mod 2^64 by Newton iteration */
    uint64_t inv = 1;
    for (int i = 0; i < 7; i++) inv *= 2 - f->p[0] * inv;
    f->n0 = (uint64_t)0 - inv;
    /* R mod p by 256 modular doublings of 1, R^2 by 256 more */
    fp_t x = {{1, 0, 0, 0}};
    for (int i = 0; i < 512; i++) {
        if (i == 256) f->one = x;
        fp_add(f, &x, &x, &x);
    }
    f->r2 = x;
}

/* ------------------------------- Fq2 ------------------------------------ */
#define Q (&FQ)

void fq2_add(fq2_t *r, const fq2_t *a, const fq2_t *b) {
    fp_add(Q, &r->c0, &a->c0, &b->c0);
    fp_add(Q, &r->c1, &a->c1, &b->c1);
}
void fq2_sub(fq2_t *r, const fq2_t *a, const fq2_t *b) {
    fp_sub(Q, &r->c0, &a->c0, &b->c0);
    fp_sub(Q, &r->c1, &a->c1, &b->c1);
}
void fq2_neg(fq2_t *r, const fq2_t *a) {
    fp_neg(Q, &r->c0, &a->c0);
    fp_neg(Q, &r->c1, &a->c1);
}
void fq2_conj(fq2_t *r, const fq2_t *a) {
    r->c0 = a->c0;
    fp_neg(Q, &r->c1, &a->c1);
}
void fq2_mul(fq2_t *r, const fq2_t *a, const fq2_t *b) {
    fp_t t0, t1, s0, s1, m;
    fp_mul(Q, &t0, &a->c0, &b->c0);
    fp_mul(Q, &t1, &a->c1, &b->c1);
    fp_add(Q, &s0, &a->c0, &a->c1);
    fp_add(Q, &s1, &b->c0, &b->c1);
    fp_mul(Q, &m, &s0, &s1);
    fp_sub(Q, &m, &m, &t0);
    fp_sub(Q, &r->c1, &m, &t1);
    fp_sub(Q, &r->c0, &t0, &t1);
}
void fq2_sqr(fq2_t *r, const fq2_t *a) { fq2_mul(r, a, a); }
void fq2_mul_fq(fq2_t *r, const fq2_t *a, const fp_t *b) {
    fp_mul(Q, &r->c0, &a->c0, b);
    fp_mul(Q, &r->c1, &a->c1, b);
}
void fq2_inv(fq2_t *r, const fq2_t *a) {
    fp_t t0, t1, n;
    fp_sqr(Q, &t0, &a->c0);
    fp_sqr(Q, &t1, &a->c1);
    fp_add(Q, &n, &t0, &t1);
    fp_inv(Q, &n, &n);
    fp_mul(Q, &r->c0, &a->c0, &n);
    fp_mul(Q, &t1, &a->c1, &n);
    fp_neg(Q, &r->c1, &t1);
}
/* (a0 + a1 u)(9 + u) = (9 a0 - a1) + (a0 + 9 a1) u */
void fq2_mul_xi(fq2_t *r, const fq2_t *a) {
    fp_t n0 = a->c0, n1 = a->c1, t;
    fp_t a9_0, a9_1;
    /* 9x = 8x + x */
    fp_add(Q, &t, &n0, &n0); fp_add(Q, &t, &t, &t); fp_add(Q, &t, &t, &t); fp_add(Q, &a9_0, &t, &n0);
    fp_add(Q, &t, &n1, &n1); fp_add(Q, &t, &t, &t); fp_add(Q, &t, &t, &t); fp_add(Q, &a9_1, &t, &n1);
    fp_sub(Q, &r->c0, &a9_0, &n1);
    fp_add(Q, &r->c1, &n0, &a9_1);
}
void fq2_set_one(fq2_t *r) {
    r->c0 = FQ.one;
    memset(&r->c1, 0, sizeof r->c1);
}
int fq2_is_zero(const fq2_t *a) { return fp_is_zero(&a->c0) && fp_is_zero(&a->c1); }
int fq2_eq(const fq2_t *a, const fq2_t *b) { return fp_eq(&a->c0, &b->c0) && fp_eq(&a->c1, &b->c1); }
void fq2_pow(fq2_t *r, const fq2_t *a, const uint64_t *e, int nlimbs) {
    fq2_t acc, base = *a;
    fq2_set_one(&acc);
    for (int i = nlimbs * 64 - 1; i >= 0; i--) {
        fq2_sqr(&acc, &acc);
        if ((e[i / 64] >> (i % 64)) & 1) fq2_mul(&acc, &acc, &base);
    }
    *r = acc;
}

/*
 * Square root in Fq2 for q = 3 mod 4 (Adj and Rodriguez-Henriquez,
 * "Square root computation over even extension fields", Algorithm 9).
 */
int fq2_sqrt(fq2_t *r, const fq2_t *a) {
    if (fq2_is_zero(a)) { memset(r, 0, sizeof *r); return 1; }
    uint64_t e1[4], e2[4];
    uint64_t three[4] = {3, 0, 0, 0}, one[4] = {1, 0, 0, 0};
    /* e1 = (q - 3) / 4 */
    sub4(e1, FQ.p, three);
    for (int i = 0; i < 4; i++) e1[i] = (e1[i] >> 2) | (i < 3 ? (e1[i + 1] << 62) : 0);
    /* e2 = (q - 1) / 2 */
    sub4(e2, FQ.p, one);
    for (int i = 0; i < 4; i++) e2[i] = (e2[i] >> 1) | (i < 3 ? (e2[i + 1] << 63) : 0);
    fq2_t a1, alpha, a0, x0, minus_one, b, chk;
    fq2_pow(&a1, a, e1, 4);
    fq2_mul(&alpha, &a1, a);
    fq2_mul(&alpha, &alpha, &a1);      /* alpha = a^((q-1)/2)... times a1 */
    fq2_conj(&a0, &alpha);
    fq2_mul(&a0, &a0, &alpha);          /* a0 = alpha^(q+1) */
    fq2_set_one(&minus_one);
    fq2_neg(&minus_one, &minus_one);
    if (fq2_eq(&a0, &minus_one)) return 0;
    fq2_mul(&x0, &a1, a);
    if (fq2_eq(&alpha, &minus_one)) {
        /* x = i * x0 */
        fq2_t i_ = {{{0}}, FQ.one};
        fq2_mul(r, &i_, &x0);
    } else {
        fq2_t one2;
        fq2_set_one(&one2);
        fq2_add(&b, &one2, &alpha);
        fq2_pow(&b, &b, e2, 4);
        fq2_mul(r, &b, &x0);
    }
    fq2_sqr(&chk, r);
    return fq2_eq(&chk, a);
}

/* ------------------------------- Fq6 ------------------------------------ */
static void fq6_add(fq6_t *r, const fq6_t *a, const fq6_t *b) {
    fq2_add(&r->c0, &a->c0, &b->c0);
    fq2_add(&r->c1, &a->c1, &b->c1);
    fq2_add(&r->c2, &a->c2, &b->c2);
}
static void fq6_sub(fq6_t *r, const fq6_t *a, const fq6_t *b) {
    fq2_sub(&r->c0, &a->c0, &b->c0);
    fq2_sub(&r->c1, &a->c1, &b->c1);
    fq2_sub(&r->c2, &a->c2, &b->c2);
}
static void fq6_neg(fq6_t *r, const fq6_t *a) {
    fq2_neg(&r->c0, &a->c0);
    fq2_neg(&r->c1, &a->c1);
    fq2_neg(&r->c2, &a->c2);
}
static void fq6_mul(fq6_t *r, const fq6_t *a, const fq6_t *b) {
    fq2_t t0, t1, t2, x, y, c0, c1, c2;
    fq2_mul(&t0, &a->c0, &b->c0);
    fq2_mul(&t1, &a->c1, &b->c1);
    fq2_mul(&t2, &a->c2, &b->c2);
    /* c0 = t0 + xi (a1 b2 + a2 b1) */
    fq2_mul(&x, &a->c1, &b->c2);
    fq2_mul(&y, &a->c2, &b->c1);
    fq2_add(&x, &x, &y);
    fq2_mul_xi(&x, &x);
    fq2_add(&c0, &t0, &x);
    /* c1 = a0 b1 + a1 b0 + xi t2 */
    fq2_mul(&x, &a->c0, &b->c1);
    fq2_mul(&y, &a->c1, &b->c0);
    fq2_add(&x, &x, &y);
    fq2_mul_xi(&y, &t2);
    fq2_add(&c1, &x, &y);
    /* c2 = a0 b2 + t1 + a2 b0 */
    fq2_mul(&x, &a->c0, &b->c2);
    fq2_mul(&y, &a->c2, &b->c0);
    fq2_add(&x, &x, &y);
    fq2_add(&c2, &x, &t1);
    r->c0 = c0; r->c1 = c1; r->c2 = c2;
}
/* times v: (c0, c1, c2) v = (xi c2, c0, c1) */
static void fq6_mul_v(fq6_t *r, const fq6_t *a) {
    fq2_t t;
    fq2_mul_xi(&t, &a->c2);
    r->c2 = a->c1;
    r->c1 = a->c0;
    r->c0 = t;
}
static void fq6_inv(fq6_t *r, const fq6_t *a) {
    fq2_t t0, t1, t2, x, d;
    fq2_sqr(&t0, &a->c0);
    fq2_mul(&x, &a->c1, &a->c2);
    fq2_mul_xi(&x, &x);
    fq2_sub(&t0, &t0, &x);          /* a0^2 - xi a1 a2 */
    fq2_sqr(&t1, &a->c2);
    fq2_mul_xi(&t1, &t1);
    fq2_mul(&x, &a->c0, &a->c1);
    fq2_sub(&t1, &t1, &x);          /* xi a2^2 - a0 a1 */
    fq2_sqr(&t2, &a->c1);
    fq2_mul(&x, &a->c0, &a->c2);
    fq2_sub(&t2, &t2, &x);          /* a1^2 - a0 a2 */
    fq2_mul(&d, &a->c2, &t1);
    fq2_mul(&x, &a->c1, &t2);
    fq2_add(&d, &d, &x);
    fq2_mul_xi(&d, &d);
    fq2_mul(&x, &a->c0, &t0);
    fq2_add(&d, &d, &x);
    fq2_inv(&d, &d);
    fq2_mul(&r->c0, &t0, &d);
    fq2_mul(&r->c1, &t1, &d);
    fq2_mul(&r->c2, &t2, &d);
}

/* ------------------------------- Fq12 ----------------------------------- */
void fq12_set_one(fq12_t *r) {
    memset(r, 0, sizeof *r);
    fq2_set_one(&r->c0.c0);
}
void fq12_mul(fq12_t *r, const fq12_t *a, const fq12_t *b) {
    fq6_t t0, t1, x, y;
    fq6_mul(&t0, &a->c0, &b->c0);
    fq6_mul(&t1, &a->c1, &b->c1);
    fq6_mul(&x, &a->c0, &b->c1);
    fq6_mul(&y, &a->c1, &b->c0);
    fq6_add(&r->c1, &x, &y);
    fq6_mul_v(&t1, &t1);
    fq6_add(&r->c0, &t0, &t1);
}
void fq12_sqr(fq12_t *r, const fq12_t *a) { fq12_mul(r, a, a); }
void fq12_conj(fq12_t *r, const fq12_t *a) {
    r->c0 = a->c0;
    fq6_neg(&r->c1, &a->c1);
}
void fq12_inv(fq12_t *r, const fq12_t *a) {
    fq6_t t0, t1, d;
    fq6_mul(&t0, &a->c0, &a->c0);
    fq6_mul(&t1, &a->c1, &a->c1);
    fq6_mul_v(&t1, &t1);
    fq6_sub(&d, &t0, &t1);
    fq6_inv(&d, &d);
    fq6_mul(&r->c0, &a->c0, &d);
    fq6_mul(&t0, &a->c1, &d);
    fq6_neg(&r->c1, &t0);
}
int fq12_eq(const fq12_t *a, const fq12_t *b) { return memcmp(a, b, sizeof *a) == 0; }
int fq12_is_one(const fq12_t *a) {
    fq12_t one;
    fq12_set_one(&one);
    return fq12_eq(a, &one);
}

/* gamma[j] = xi^(j (q-1)/6): (x w^j)^q = conj(x) w^j gamma[j], since w^6 = xi */
static fq2_t FROB_GAMMA[6];

/* f = sum_k g_k w^(2k) + h_k w^(2k+1) with c0 = (g0,g1,g2), c1 = (h0,h1,h2) */
void fq12_frob(fq12_t *r, const fq12_t *a) {
    fq2_t t;
    fq2_conj(&t, &a->c0.c0); r->c0.c0 = t;
    fq2_conj(&t, &a->c0.c1); fq2_mul(&r->c0.c1, &t, &FROB_GAMMA[2]);
    fq2_conj(&t, &a->c0.c2); fq2_mul(&r->c0.c2, &t, &FROB_GAMMA[4]);
    fq2_conj(&t, &a->c1.c0); fq2_mul(&r->c1.c0, &t, &FROB_GAMMA[1]);
    fq2_conj(&t, &a->c1.c1); fq2_mul(&r->c1.c1, &t, &FROB_GAMMA[3]);
    fq2_conj(&t, &a->c1.c2); fq2_mul(&r->c1.c2, &t, &FROB_GAMMA[5]);
}

const fq2_t *bn254_frob_gamma(int j) { return &FROB_GAMMA[j]; }

void bn254_curve_init(void);
void bn254_pairing_init(void);

void bn254_init(void) {
    static int done = 0;
    if (done) return;
    compute_consts(&FR);
    compute_consts(&FQ);
    /* (q - 1) / 6 */
    uint64_t e[4], one[4] = {1, 0, 0, 0};
    sub4(e, FQ.p, one);
    u128 rem = 0;
    for (int i = 3; i >= 0; i--) {
        u128 cur = (rem << 64) | e[i];
        e[i] = (uint64_t)(cur / 6);
        rem = cur % 6;
    }
    fq2_t xi = {FQ.one, FQ.one};
    fq2_mul_xi(&xi, &(fq2_t){FQ.one, {{0}}});   /* xi = 9 + u */
    fq2_t g1;
    fq2_pow(&g1, &xi, e, 4);
    fq2_set_one(&FROB_GAMMA[0]);
    for (int j = 1; j < 6; j++) fq2_mul(&FROB_GAMMA[j], &FROB_GAMMA[j - 1], &g1);
    done = 1;
    bn254_curve_init();
    bn254_pairing_init();
}
