/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * XYZZ point arithmetic for the timed CPU baseline (port_msm.c) and the
 * oracle's key generator (synth.c), the formulas of crates/msm/src/xyzz.rs:
 * madd-2008-s, add-2008-s, dbl-2008-s-1 and mdbl-2008-s-1 for a = 0, with the
 * identity as ZZ = 0 and the exceptional cases (identity operand, P + P,
 * P + (-P)) handled explicitly.  PORT_DEFINE_CURVE instantiates them for one
 * group: G1 over Fq (prefix pq) or G2 over Fq2 (prefix pq2).
 */
#ifndef G16_ORACLE_PORT_CURVE_H
#define G16_ORACLE_PORT_CURVE_H
#include "port_field.h"

#define pq_is_zero pf_is_zero
#define pq_eq pf_eq

static const fp_t PF_ZERO = {{0, 0, 0, 0}};
/* R mod q: the Montgomery form of 1 */
static const fp_t PF_QONE = {{0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL,
                              0x0e0a77c19a07df2fULL}};
static const fq2_t PF2_ZERO = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
static const fq2_t PF2_ONE = {{{0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL,
                                0x0e0a77c19a07df2fULL}},
                              {{0, 0, 0, 0}}};

#define PORT_DEFINE_CURVE(G, F, JAC, P, ZERO_F, ONE_F)                                               \
typedef struct { F x, y, zz, zzz; } G##_xyzz;                                                         \
                                                                                                      \
static inline void G##_set_id(G##_xyzz *r) { r->zz = ZERO_F; r->zzz = ZERO_F; r->x = ONE_F; r->y = ONE_F; } \
static inline int G##_is_id(const G##_xyzz *r) { return P##_is_zero(&r->zz); }                        \
                                                                                                      \
/* 2 (x, y), mdbl-2008-s-1 */                                                                        \
static void G##_dbl_affine(G##_xyzz *r, const F *x, const F *y) {                                     \
    F u, v, w, s, xx, m, t;                                                                           \
    P##_dbl(&u, y);                                                                                   \
    P##_sqr(&v, &u);                                                                                  \
    P##_mul(&w, &u, &v);                                                                              \
    P##_mul(&s, x, &v);                                                                               \
    P##_sqr(&xx, x);                                                                                  \
    P##_dbl(&m, &xx);                                                                                 \
    P##_add(&m, &m, &xx);                                                                             \
    P##_sqr(&r->x, &m);                                                                               \
    P##_sub(&r->x, &r->x, &s);                                                                        \
    P##_sub(&r->x, &r->x, &s);                                                                        \
    P##_sub(&t, &s, &r->x);                                                                           \
    P##_mul(&t, &m, &t);                                                                              \
    P##_mul(&u, &w, y);                                                                               \
    P##_sub(&r->y, &t, &u);                                                                           \
    r->zz = v;                                                                                        \
    r->zzz = w;                                                                                       \
}                                                                                                     \
                                                                                                      \
/* 2 p, dbl-2008-s-1 */                                                                              \
static void G##_dbl(G##_xyzz *r, const G##_xyzz *p) {                                                 \
    if (G##_is_id(p)) { *r = *p; return; }                                                            \
    F u, v, w, s, xx, m, t, y1 = p->y, zz1 = p->zz, zzz1 = p->zzz;                                    \
    P##_dbl(&u, &p->y);                                                                               \
    P##_sqr(&v, &u);                                                                                  \
    P##_mul(&w, &u, &v);                                                                              \
    P##_mul(&s, &p->x, &v);                                                                           \
    P##_sqr(&xx, &p->x);                                                                              \
    P##_dbl(&m, &xx);                                                                                 \
    P##_add(&m, &m, &xx);                                                                             \
    P##_sqr(&r->x, &m);                                                                               \
    P##_sub(&r->x, &r->x, &s);                                                                        \
    P##_sub(&r->x, &r->x, &s);                                                                        \
    P##_sub(&t, &s, &r->x);                                                                           \
    P##_mul(&t, &m, &t);                                                                              \
    P##_mul(&u, &w, &y1);                                                                             \
    P##_sub(&r->y, &t, &u);                                                                           \
    P##_mul(&r->zz, &v, &zz1);                                                                        \
    P##_mul(&r->zzz, &w, &zzz1);                                                                      \
}                                                                                                     \
                                                                                                      \
/* p += (x2, y2), madd-2008-s */                                                                     \
static void G##_madd(G##_xyzz *p, const F *x2, const F *y2) {                                         \
    if (G##_is_id(p)) { p->x = *x2; p->y = *y2; p->zz = ONE_F; p->zzz = ONE_F; return; }              \
    F u2, s2, pp_, rr, pp, ppp, q, t;                                                                 \
    P##_mul(&u2, x2, &p->zz);                                                                         \
    P##_mul(&s2, y2, &p->zzz);                                                                        \
    P##_sub(&pp_, &u2, &p->x);                                                                        \
    P##_sub(&rr, &s2, &p->y);                                                                         \
    if (P##_is_zero(&pp_)) {                                                                          \
        if (P##_is_zero(&rr)) G##_dbl_affine(p, x2, y2);                                              \
        else G##_set_id(p);                                                                           \
        return;                                                                                       \
    }                                                                                                 \
    P##_sqr(&pp, &pp_);                                                                               \
    P##_mul(&ppp, &pp_, &pp);                                                                         \
    P##_mul(&q, &p->x, &pp);                                                                          \
    P##_sqr(&p->x, &rr);                                                                              \
    P##_sub(&p->x, &p->x, &ppp);                                                                      \
    P##_sub(&p->x, &p->x, &q);                                                                        \
    P##_sub(&p->x, &p->x, &q);                                                                        \
    P##_sub(&t, &q, &p->x);                                                                           \
    P##_mul(&t, &rr, &t);                                                                             \
    P##_mul(&q, &p->y, &ppp);                                                                         \
    P##_sub(&p->y, &t, &q);                                                                           \
    P##_mul(&p->zz, &p->zz, &pp);                                                                     \
    P##_mul(&p->zzz, &p->zzz, &ppp);                                                                  \
}                                                                                                     \
                                                                                                      \
/* p += q, add-2008-s */                                                                             \
static void G##_add(G##_xyzz *p, const G##_xyzz *q) {                                                 \
    if (G##_is_id(q)) return;                                                                         \
    if (G##_is_id(p)) { *p = *q; return; }                                                            \
    F u1, u2, s1, s2, pp_, rr, pp, ppp, qq, t;                                                        \
    P##_mul(&u1, &p->x, &q->zz);                                                                      \
    P##_mul(&u2, &q->x, &p->zz);                                                                      \
    P##_mul(&s1, &p->y, &q->zzz);                                                                     \
    P##_mul(&s2, &q->y, &p->zzz);                                                                     \
    P##_sub(&pp_, &u2, &u1);                                                                          \
    P##_sub(&rr, &s2, &s1);                                                                           \
    if (P##_is_zero(&pp_)) {                                                                          \
        if (P##_is_zero(&rr)) { G##_xyzz d; G##_dbl(&d, p); *p = d; }                                 \
        else G##_set_id(p);                                                                           \
        return;                                                                                       \
    }                                                                                                 \
    P##_sqr(&pp, &pp_);                                                                               \
    P##_mul(&ppp, &pp_, &pp);                                                                         \
    P##_mul(&qq, &u1, &pp);                                                                           \
    P##_sqr(&p->x, &rr);                                                                              \
    P##_sub(&p->x, &p->x, &ppp);                                                                      \
    P##_sub(&p->x, &p->x, &qq);                                                                       \
    P##_sub(&p->x, &p->x, &qq);                                                                       \
    P##_sub(&t, &qq, &p->x);                                                                          \
    P##_mul(&t, &rr, &t);                                                                             \
    P##_mul(&qq, &s1, &ppp);                                                                          \
    P##_sub(&p->y, &t, &qq);                                                                          \
    P##_mul(&p->zz, &p->zz, &q->zz);                                                                  \
    P##_mul(&p->zz, &p->zz, &pp);                                                                     \
    P##_mul(&p->zzz, &p->zzz, &q->zzz);                                                               \
    P##_mul(&p->zzz, &p->zzz, &ppp);                                                                  \
}                                                                                                     \
                                                                                                      \
/* XYZZ -> the oracle's Jacobian without an inversion: Z = ZZ ZZZ, X' = X ZZ ZZZ^2, Y' = Y ZZ^3 ZZZ^2 */ \
static void G##_to_jac(JAC *r, const G##_xyzz *p) {                                                   \
    if (G##_is_id(p)) { r->x = ONE_F; r->y = ONE_F; r->z = ZERO_F; return; }                          \
    F z3, zz2;                                                                                        \
    P##_sqr(&z3, &p->zzz);                                                                            \
    P##_mul(&r->z, &p->zz, &p->zzz);                                                                  \
    P##_mul(&r->x, &p->x, &p->zz);                                                                    \
    P##_mul(&r->x, &r->x, &z3);                                                                       \
    P##_sqr(&zz2, &p->zz);                                                                            \
    P##_mul(&zz2, &zz2, &p->zz);                                                                      \
    P##_mul(&r->y, &p->y, &zz2);                                                                      \
    P##_mul(&r->y, &r->y, &z3);                                                                       \
}                                                                                                     \

PORT_DEFINE_CURVE(pg1, fp_t, g1j_t, pq, PF_ZERO, PF_QONE)
PORT_DEFINE_CURVE(pg2, fq2_t, g2j_t, pq2, PF2_ZERO, PF2_ONE)

#endif
