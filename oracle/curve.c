/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * BN254 G1 (y^2 = x^3 + 3 over Fq) and G2 (the D-type sextic twist
 * y^2 = x^3 + 3/(9+u) over Fq2) in Jacobian coordinates.  Formulas are the
 * Explicit-Formulas Database ones for a = 0 (dbl-2009-l, add-2007-bl,
 * madd-2007-bl).  The reference computes with arkworks' projective points
 * and XYZZ buckets (crates/msm/src/xyzz.rs); every comparison is made on
 * normalised affine points (crates/groth16/src/trace.rs:19-24), where the
 * coordinate system leaves no trace.
 */
#include "bn254.h"
#include <string.h>
#include <stdlib.h>

g1a_t G1_GEN;
g2a_t G2_GEN;
static fp_t B1;     /* 3 */
static fq2_t B2;    /* 3 / (9 + u) */

/* decimal string -> standard-form limbs (no reduction) */
void oracle_parse_dec(fp_t *out, const char *s) {
    memset(out, 0, sizeof *out);
    for (; *s; s++) {
        unsigned __int128 carry = (unsigned)(*s - '0');
        for (int i = 0; i < 4; i++) {
            unsigned __int128 t = (unsigned __int128)out->v[i] * 10 + carry;
            out->v[i] = (uint64_t)t;
            carry = t >> 64;
        }
    }
}

static void fq_dec(fp_t *r, const char *s) {
    fp_t t;
    oracle_parse_dec(&t, s);
    fp_to_mont(&FQ, r, &t);
}

/* ---- per-field helpers so one template body serves G1 and G2 ---- */
#define Q (&FQ)
static inline void f1_add(fp_t *r, const fp_t *a, const fp_t *b) { fp_add(Q, r, a, b); }
static inline void f1_sub(fp_t *r, const fp_t *a, const fp_t *b) { fp_sub(Q, r, a, b); }
static inline void f1_mul(fp_t *r, const fp_t *a, const fp_t *b) { fp_mul(Q, r, a, b); }
static inline void f1_sqr(fp_t *r, const fp_t *a) { fp_mul(Q, r, a, a); }
static inline void f1_neg(fp_t *r, const fp_t *a) { fp_neg(Q, r, a); }
static inline void f1_inv(fp_t *r, const fp_t *a) { fp_inv(Q, r, a); }
static inline int  f1_is_zero(const fp_t *a) { return fp_is_zero(a); }
static inline int  f1_eq(const fp_t *a, const fp_t *b) { return fp_eq(a, b); }
static inline void f1_one(fp_t *r) { *r = FQ.one; }

static inline void f2_one(fq2_t *r) { fq2_set_one(r); }

#define DEFINE_CURVE(G, F, FT, CURVE_B)                                              \
void G##j_set_inf(G##j_t *r) { memset(r, 0, sizeof *r); F##_one(&r->x); F##_one(&r->y); } \
int  G##j_is_inf(const G##j_t *a) { return F##_is_zero(&a->z); }                     \
void G##j_from_affine(G##j_t *r, const G##a_t *a) {                                  \
    if (a->inf) { G##j_set_inf(r); return; }                                         \
    r->x = a->x; r->y = a->y; F##_one(&r->z);                                        \
}                                                                                    \
void G##j_dbl(G##j_t *r, const G##j_t *p) {                                          \
    if (G##j_is_inf(p)) { *r = *p; return; }                                         \
    FT A, B, C, D, E, Fv, t, x3, y3, z3;                                             \
    F##_sqr(&A, &p->x); F##_sqr(&B, &p->y); F##_sqr(&C, &B);                         \
    F##_add(&t, &p->x, &B); F##_sqr(&t, &t); F##_sub(&t, &t, &A); F##_sub(&t, &t, &C);\
    F##_add(&D, &t, &t);                                                             \
    F##_add(&E, &A, &A); F##_add(&E, &E, &A);                                        \
    F##_sqr(&Fv, &E);                                                                \
    F##_add(&t, &D, &D); F##_sub(&x3, &Fv, &t);                                      \
    F##_sub(&t, &D, &x3); F##_mul(&y3, &E, &t);                                      \
    F##_add(&C, &C, &C); F##_add(&C, &C, &C); F##_add(&C, &C, &C);                   \
    F##_sub(&y3, &y3, &C);                                                           \
    F##_mul(&z3, &p->y, &p->z); F##_add(&z3, &z3, &z3);                              \
    r->x = x3; r->y = y3; r->z = z3;                                                 \
}                                                                                    \
void G##j_add(G##j_t *r, const G##j_t *p, const G##j_t *q) {                         \
    if (G##j_is_inf(p)) { *r = *q; return; }                                         \
    if (G##j_is_inf(q)) { *r = *p; return; }                                         \
    FT z1z1, z2z2, u1, u2, s1, s2, h, i, j, rr, v, t, x3, y3, z3;                    \
    F##_sqr(&z1z1, &p->z); F##_sqr(&z2z2, &q->z);                                    \
    F##_mul(&u1, &p->x, &z2z2); F##_mul(&u2, &q->x, &z1z1);                          \
    F##_mul(&s1, &p->y, &q->z); F##_mul(&s1, &s1, &z2z2);                            \
    F##_mul(&s2, &q->y, &p->z); F##_mul(&s2, &s2, &z1z1);                            \
    F##_sub(&h, &u2, &u1); F##_sub(&rr, &s2, &s1);                                   \
    if (F##_is_zero(&h)) {                                                           \
        if (F##_is_zero(&rr)) { G##j_dbl(r, p); return; }                            \
        G##j_set_inf(r); return;                                                     \
    }                                                                                \
    F##_add(&i, &h, &h); F##_sqr(&i, &i);                                            \
    F##_mul(&j, &h, &i);                                                             \
    F##_add(&rr, &rr, &rr);                                                          \
    F##_mul(&v, &u1, &i);                                                            \
    F##_sqr(&x3, &rr); F##_sub(&x3, &x3, &j); F##_sub(&x3, &x3, &v); F##_sub(&x3, &x3, &v); \
    F##_sub(&t, &v, &x3); F##_mul(&y3, &rr, &t);                                     \
    F##_mul(&t, &s1, &j); F##_add(&t, &t, &t); F##_sub(&y3, &y3, &t);                \
    F##_add(&t, &p->z, &q->z); F##_sqr(&t, &t); F##_sub(&t, &t, &z1z1);              \
    F##_sub(&t, &t, &z2z2); F##_mul(&z3, &t, &h);                                    \
    r->x = x3; r->y = y3; r->z = z3;                                                 \
}                                                                                    \
void G##j_add_affine(G##j_t *r, const G##j_t *p, const G##a_t *q) {                  \
    if (q->inf) { *r = *p; return; }                                                 \
    if (G##j_is_inf(p)) { G##j_from_affine(r, q); return; }                          \
    FT z1z1, u2, s2, h, hh, i, j, rr, v, t, x3, y3, z3;                              \
    F##_sqr(&z1z1, &p->z);                                                           \
    F##_mul(&u2, &q->x, &z1z1);                                                      \
    F##_mul(&s2, &q->y, &p->z); F##_mul(&s2, &s2, &z1z1);                            \
    F##_sub(&h, &u2, &p->x); F##_sub(&rr, &s2, &p->y);                               \
    if (F##_is_zero(&h)) {                                                           \
        if (F##_is_zero(&rr)) { G##j_dbl(r, p); return; }                            \
        G##j_set_inf(r); return;                                                     \
    }                                                                                \
    F##_sqr(&hh, &h);                                                                \
    F##_add(&i, &hh, &hh); F##_add(&i, &i, &i);                                      \
    F##_mul(&j, &h, &i);                                                             \
    F##_add(&rr, &rr, &rr);                                                          \
    F##_mul(&v, &p->x, &i);                                                          \
    F##_sqr(&x3, &rr); F##_sub(&x3, &x3, &j); F##_sub(&x3, &x3, &v); F##_sub(&x3, &x3, &v); \
    F##_sub(&t, &v, &x3); F##_mul(&y3, &rr, &t);                                     \
    F##_mul(&t, &p->y, &j); F##_add(&t, &t, &t); F##_sub(&y3, &y3, &t);              \
    F##_add(&t, &p->z, &h); F##_sqr(&t, &t); F##_sub(&t, &t, &z1z1); F##_sub(&z3, &t, &hh); \
    r->x = x3; r->y = y3; r->z = z3;                                                 \
}                                                                                    \
void G##j_neg(G##j_t *r, const G##j_t *p) { *r = *p; F##_neg(&r->y, &p->y); }        \
void G##j_to_affine(G##a_t *r, const G##j_t *p) {                                    \
    if (G##j_is_inf(p)) { memset(r, 0, sizeof *r); r->inf = 1; return; }             \
    FT zi, zi2, zi3;                                                                 \
    F##_inv(&zi, &p->z); F##_sqr(&zi2, &zi); F##_mul(&zi3, &zi2, &zi);               \
    F##_mul(&r->x, &p->x, &zi2); F##_mul(&r->y, &p->y, &zi3); r->inf = 0;            \
}                                                                                    \
void G##j_mul(G##j_t *r, const G##j_t *p, const fp_t *k) {                           \
    G##j_t acc; G##j_set_inf(&acc);                                                  \
    for (int i = 255; i >= 0; i--) {                                                 \
        G##j_dbl(&acc, &acc);                                                        \
        if ((k->v[i / 64] >> (i % 64)) & 1) G##j_add(&acc, &acc, p);                 \
    }                                                                                \
    *r = acc;                                                                        \
}                                                                                    \
int G##a_on_curve(const G##a_t *a) {                                                 \
    if (a->inf) return 1;                                                            \
    FT l, rr;                                                                        \
    F##_sqr(&l, &a->y);                                                              \
    F##_sqr(&rr, &a->x); F##_mul(&rr, &rr, &a->x); F##_add(&rr, &rr, &CURVE_B);      \
    return F##_eq(&l, &rr);                                                          \
}                                                                                    \
int G##a_eq(const G##a_t *a, const G##a_t *b) {                                      \
    if (a->inf || b->inf) return a->inf == b->inf;                                   \
    return F##_eq(&a->x, &b->x) && F##_eq(&a->y, &b->y);                             \
}

static inline void f2_add(fq2_t *r, const fq2_t *a, const fq2_t *b) { fq2_add(r, a, b); }
static inline void f2_sub(fq2_t *r, const fq2_t *a, const fq2_t *b) { fq2_sub(r, a, b); }
static inline void f2_mul(fq2_t *r, const fq2_t *a, const fq2_t *b) { fq2_mul(r, a, b); }
static inline void f2_sqr(fq2_t *r, const fq2_t *a) { fq2_mul(r, a, a); }
static inline void f2_neg(fq2_t *r, const fq2_t *a) { fq2_neg(r, a); }
static inline void f2_inv(fq2_t *r, const fq2_t *a) { fq2_inv(r, a); }
static inline int  f2_is_zero(const fq2_t *a) { return fq2_is_zero(a); }
static inline int  f2_eq(const fq2_t *a, const fq2_t *b) { return fq2_eq(a, b); }

DEFINE_CURVE(g1, f1, fp_t, B1)
DEFINE_CURVE(g2, f2, fq2_t, B2)

/* r * Q == 0 for the group order r */
int g2a_in_subgroup(const g2a_t *a) {
    if (a->inf) return 1;
    g2j_t p, t;
    g2j_from_affine(&p, a);
    fp_t order = {{FR.p[0], FR.p[1], FR.p[2], FR.p[3]}};
    g2j_mul(&t, &p, &order);
    return g2j_is_inf(&t);
}

void bn254_curve_init(void) {
    fp_from_u64(&FQ, &B1, 3);
    fq2_t xi = {{{0}}, {{0}}}, three = {{{0}}, {{0}}};
    fp_from_u64(&FQ, &xi.c0, 9);
    xi.c1 = FQ.one;
    three.c0 = B1;
    fq2_t xi_inv;
    fq2_inv(&xi_inv, &xi);
    fq2_mul(&B2, &three, &xi_inv);

    fp_from_u64(&FQ, &G1_GEN.x, 1);
    fp_from_u64(&FQ, &G1_GEN.y, 2);
    G1_GEN.inf = 0;
    /* The standard BN254 G2 generator (as in EIP-197). */
    fq_dec(&G2_GEN.x.c0, "10857046999023057135944570762232829481370756359578518086990519993285655852781");
    fq_dec(&G2_GEN.x.c1, "11559732032986387107991004021392285783925812861821192530917403151452391805634");
    fq_dec(&G2_GEN.y.c0, "8495653923123431417604973247489272438418190587263600148770280649306958101930");
    fq_dec(&G2_GEN.y.c1, "4082367875863433681332203403145435568316851327593401208105741076214120093531");
    G2_GEN.inf = 0;
}
