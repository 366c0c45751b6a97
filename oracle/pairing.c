/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Optimal ate pairing on BN254, written from the published construction
 * (Vercauteren, "Optimal pairings", 2010; Beuchat et al., "High-speed
 * software implementation of the optimal ate pairing over Barreto-Naehrig
 * curves", 2010): a Miller loop over 6u+2 with affine line functions on the
 * twist, the two Frobenius correction lines, then the final exponentiation
 * (q^12-1)/r split into (q^6-1)(q^2+1) and a plain square-and-multiply hard
 * part.  Speed is irrelevant here; this is the checker for the Groth16
 * verification equation the reference runs in crates/groth16/src/verify.rs:112-137.
 */
#include "bn254.h"
#include <string.h>

const fq2_t *bn254_frob_gamma(int j);

/* BN parameter u and the hard exponent (q^4 - q^2 + 1) / r, computed at init */
static const uint64_t BN_U = 0x44e992b44a6909f1ULL;
static uint32_t HARD_EXP[40];
static int HARD_BITS;

/* ---- a tiny unsigned bigint on 32-bit limbs, just enough for init ---- */
#define BL 40
typedef struct { uint32_t w[BL]; } big_t;
static void big_from_fp(big_t *r, const uint64_t *v) {
    memset(r, 0, sizeof *r);
    for (int i = 0; i < 4; i++) { r->w[2 * i] = (uint32_t)v[i]; r->w[2 * i + 1] = (uint32_t)(v[i] >> 32); }
}
static void big_mul(big_t *r, const big_t *a, const big_t *b) {
    uint32_t out[BL] = {0};
    for (int i = 0; i < BL; i++) {
        uint64_t carry = 0;
        for (int j = 0; i + j < BL; j++) {
            uint64_t t = (uint64_t)a->w[i] * b->w[j] + out[i + j] + carry;
            out[i + j] = (uint32_t)t;
            carry = t >> 32;
        }
    }
    memcpy(r->w, out, sizeof out);
}
static int big_cmp(const big_t *a, const big_t *b) {
    for (int i = BL - 1; i >= 0; i--) { if (a->w[i] != b->w[i]) return a->w[i] > b->w[i] ? 1 : -1; }
    return 0;
}
static void big_sub(big_t *r, const big_t *a, const big_t *b) {
    int64_t borrow = 0;
    for (int i = 0; i < BL; i++) {
        int64_t d = (int64_t)a->w[i] - b->w[i] - borrow;
        borrow = d < 0;
        r->w[i] = (uint32_t)(d + (borrow ? ((int64_t)1 << 32) : 0));
    }
}
static void big_add_small(big_t *r, uint32_t x) {
    uint64_t c = x;
    for (int i = 0; i < BL && c; i++) { c += r->w[i]; r->w[i] = (uint32_t)c; c >>= 32; }
}
static int big_bits(const big_t *a) {
    for (int i = BL * 32 - 1; i >= 0; i--) if ((a->w[i / 32] >> (i % 32)) & 1) return i + 1;
    return 0;
}
static void big_shl1(big_t *a) {
    for (int i = BL - 1; i > 0; i--) a->w[i] = (a->w[i] << 1) | (a->w[i - 1] >> 31);
    a->w[0] <<= 1;
}
/* quotient of a / b by shift-and-subtract */
static void big_div(big_t *quo, const big_t *a, const big_t *b) {
    big_t rem;
    memset(&rem, 0, sizeof rem);
    memset(quo, 0, sizeof *quo);
    for (int i = big_bits(a) - 1; i >= 0; i--) {
        big_shl1(&rem);
        rem.w[0] |= (a->w[i / 32] >> (i % 32)) & 1;
        if (big_cmp(&rem, b) >= 0) { big_sub(&rem, &rem, b); quo->w[i / 32] |= 1u << (i % 32); }
    }
}

void bn254_pairing_init(void) {
    big_t q, r, q2, q4, e;
    big_from_fp(&q, FQ.p);
    big_from_fp(&r, FR.p);
    big_mul(&q2, &q, &q);
    big_mul(&q4, &q2, &q2);
    big_sub(&e, &q4, &q2);
    big_add_small(&e, 1);
    big_t quo;
    big_div(&quo, &e, &r);
    memcpy(HARD_EXP, quo.w, sizeof HARD_EXP);
    HARD_BITS = big_bits(&quo);
}

/* exported so the tests can check the exponent against Python big integers */
int oracle_hard_exponent(uint32_t *out40) { memcpy(out40, HARD_EXP, sizeof HARD_EXP); return HARD_BITS; }

/* ---- Miller loop ---- */

/* l(P) for the line of slope lambda through T (twist coordinates):
 *   c0 = (yP, 0, 0),  c1 = (-lambda xP, lambda xT - yT, 0)                 */
static void line_eval(fq12_t *l, const fq2_t *lambda, const fq2_t *xT, const fq2_t *yT, const g1a_t *p) {
    memset(l, 0, sizeof *l);
    l->c0.c0.c0 = p->y;
    fq2_t t;
    fq2_mul_fq(&t, lambda, &p->x);
    fq2_neg(&l->c1.c0, &t);
    fq2_mul(&t, lambda, xT);
    fq2_sub(&l->c1.c1, &t, yT);
}

/* vertical line x = xT: xP - xT w^2 = (xP, -xT, 0) in c0 */
static void vertical_eval(fq12_t *l, const fq2_t *xT, const g1a_t *p) {
    memset(l, 0, sizeof *l);
    l->c0.c0.c0 = p->x;
    fq2_neg(&l->c0.c1, xT);
}

/* T <- 2T, f <- f * l_{T,T}(P) (the caller squares f first) */
static void step_dbl(fq12_t *f, g2a_t *T, const g1a_t *p) {
    fq12_t l;
    if (T->inf) return;
    if (fq2_is_zero(&T->y)) {
        vertical_eval(&l, &T->x, p);
        fq12_mul(f, f, &l);
        T->inf = 1;
        return;
    }
    fq2_t num, den, lambda, x3, y3, t;
    fq2_sqr(&num, &T->x);
    fq2_add(&t, &num, &num);
    fq2_add(&num, &t, &num);          /* 3 x^2 */
    fq2_add(&den, &T->y, &T->y);      /* 2 y */
    fq2_inv(&den, &den);
    fq2_mul(&lambda, &num, &den);
    line_eval(&l, &lambda, &T->x, &T->y, p);
    fq12_mul(f, f, &l);
    fq2_sqr(&x3, &lambda);
    fq2_sub(&x3, &x3, &T->x);
    fq2_sub(&x3, &x3, &T->x);
    fq2_sub(&t, &T->x, &x3);
    fq2_mul(&y3, &lambda, &t);
    fq2_sub(&y3, &y3, &T->y);
    T->x = x3;
    T->y = y3;
}

/* T <- T + Q, f <- f * l_{T,Q}(P) */
static void step_add(fq12_t *f, g2a_t *T, const g2a_t *Qp, const g1a_t *p) {
    fq12_t l;
    if (Qp->inf) return;
    if (T->inf) { *T = *Qp; return; }
    fq2_t dx, dy, lambda, x3, y3, t;
    fq2_sub(&dx, &Qp->x, &T->x);
    fq2_sub(&dy, &Qp->y, &T->y);
    if (fq2_is_zero(&dx)) {
        if (fq2_is_zero(&dy)) { step_dbl(f, T, p); return; }
        vertical_eval(&l, &T->x, p);
        fq12_mul(f, f, &l);
        T->inf = 1;
        return;
    }
    fq2_inv(&t, &dx);
    fq2_mul(&lambda, &dy, &t);
    line_eval(&l, &lambda, &T->x, &T->y, p);
    fq12_mul(f, f, &l);
    fq2_sqr(&x3, &lambda);
    fq2_sub(&x3, &x3, &T->x);
    fq2_sub(&x3, &x3, &Qp->x);
    fq2_sub(&t, &T->x, &x3);
    fq2_mul(&y3, &lambda, &t);
    fq2_sub(&y3, &y3, &T->y);
    T->x = x3;
    T->y = y3;
}

/* the twist Frobenius pi(x, y) = (conj(x) xi^((q-1)/3), conj(y) xi^((q-1)/2)) */
static void twist_frob(g2a_t *r, const g2a_t *a) {
    fq2_t t;
    r->inf = a->inf;
    fq2_conj(&t, &a->x);
    fq2_mul(&r->x, &t, bn254_frob_gamma(2));
    fq2_conj(&t, &a->y);
    fq2_mul(&r->y, &t, bn254_frob_gamma(3));
}

void miller_loop(fq12_t *f, const g1a_t *p, const g2a_t *q) {
    fq12_set_one(f);
    if (p->inf || q->inf) return;
    unsigned __int128 s = (unsigned __int128)BN_U * 6 + 2;
    int top = 127;
    while (!((s >> top) & 1)) top--;
    g2a_t T = *q;
    for (int i = top - 1; i >= 0; i--) {
        fq12_sqr(f, f);
        step_dbl(f, &T, p);
        if ((s >> i) & 1) step_add(f, &T, q, p);
    }
    g2a_t q1, q2;
    twist_frob(&q1, q);
    twist_frob(&q2, &q1);
    fq2_neg(&q2.y, &q2.y);
    step_add(f, &T, &q1, p);
    step_add(f, &T, &q2, p);
}

void final_exponentiation(fq12_t *r, const fq12_t *f) {
    fq12_t a, b, t;
    /* easy part: f^(q^6 - 1) (q^2 + 1) */
    fq12_conj(&a, f);
    fq12_inv(&b, f);
    fq12_mul(&a, &a, &b);
    fq12_frob(&t, &a);
    fq12_frob(&t, &t);
    fq12_mul(&a, &t, &a);
    /* hard part */
    fq12_t acc;
    fq12_set_one(&acc);
    for (int i = HARD_BITS - 1; i >= 0; i--) {
        fq12_sqr(&acc, &acc);
        if ((HARD_EXP[i / 32] >> (i % 32)) & 1) fq12_mul(&acc, &acc, &a);
    }
    *r = acc;
}

int pairing_product_is_one(const g1a_t *p, const g2a_t *q, int n) {
    fq12_t f, m;
    fq12_set_one(&f);
    for (int i = 0; i < n; i++) {
        miller_loop(&m, &p[i], &q[i]);
        fq12_mul(&f, &f, &m);
    }
    fq12_t e;
    final_exponentiation(&e, &f);
    return fq12_is_one(&e);
}
