/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Field and curve arithmetic for the timed CPU baseline (port_*.c): the same
 * values as field.c / curve.c, written for speed the way the reference's raw
 * field layer is (crates/field/src/raw.rs:186 CIOS on 4 x 64-bit limbs,
 * always fully reduced; crates/msm/src/xyzz.rs XYZZ formulas).  The moduli are
 * compile-time constants and the Montgomery product is the fully unrolled
 * CIOS whose last carry needs no extra word because both BN254 moduli leave
 * the top bit of the top limb clear.
 */
#ifndef G16_ORACLE_PORT_FIELD_H
#define G16_ORACLE_PORT_FIELD_H
#include <stdint.h>
#include <string.h>
#include "bn254.h"

typedef unsigned __int128 pu128;

#define PF_Q0 0x3c208c16d87cfd47ULL
#define PF_Q1 0x97816a916871ca8dULL
#define PF_Q2 0xb85045b68181585dULL
#define PF_Q3 0x30644e72e131a029ULL
#define PF_QN0 0x87d20782e4866389ULL
#define PF_R0 0x43e1f593f0000001ULL
#define PF_R1 0x2833e84879b97091ULL
#define PF_R2 0xb85045b68181585dULL
#define PF_R3 0x30644e72e131a029ULL
#define PF_RN0 0xc2e1f593efffffffULL

/* a * b / 2^256 mod p for p < 2^255, inputs below p */
#define PF_DEFINE_MUL(NAME, P0, P1, P2, P3, N0)                                                       \
    static inline void NAME(fp_t *r, const fp_t *x, const fp_t *y) {                                  \
        const uint64_t a0 = x->v[0], a1 = x->v[1], a2 = x->v[2], a3 = x->v[3];                       \
        uint64_t t0 = 0, t1 = 0, t2 = 0, t3 = 0;                                                      \
        _Pragma("GCC unroll 4")                                                                       \
        for (int i = 0; i < 4; i++) {                                                                 \
            const uint64_t b = y->v[i];                                                               \
            pu128 s;                                                                                  \
            uint64_t c, m, t4;                                                                        \
            s = (pu128)a0 * b + t0; t0 = (uint64_t)s; c = (uint64_t)(s >> 64);                        \
            s = (pu128)a1 * b + t1 + c; t1 = (uint64_t)s; c = (uint64_t)(s >> 64);                    \
            s = (pu128)a2 * b + t2 + c; t2 = (uint64_t)s; c = (uint64_t)(s >> 64);                    \
            s = (pu128)a3 * b + t3 + c; t3 = (uint64_t)s; t4 = (uint64_t)(s >> 64);                   \
            m = t0 * (N0);                                                                            \
            s = (pu128)m * (P0) + t0; c = (uint64_t)(s >> 64);                                        \
            s = (pu128)m * (P1) + t1 + c; t0 = (uint64_t)s; c = (uint64_t)(s >> 64);                  \
            s = (pu128)m * (P2) + t2 + c; t1 = (uint64_t)s; c = (uint64_t)(s >> 64);                  \
            s = (pu128)m * (P3) + t3 + c; t2 = (uint64_t)s; c = (uint64_t)(s >> 64);                  \
            t3 = t4 + c;                                                                              \
        }                                                                                             \
        /* result < 2p: one conditional subtraction */                                               \
        pu128 d;                                                                                      \
        uint64_t u0, u1, u2, u3, bw;                                                                  \
        d = (pu128)t0 - (P0); u0 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                          \
        d = (pu128)t1 - (P1) - bw; u1 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                     \
        d = (pu128)t2 - (P2) - bw; u2 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                     \
        d = (pu128)t3 - (P3) - bw; u3 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                     \
        const uint64_t keep = (uint64_t)0 - bw; /* all ones: t < p, keep t (branch-free) */           \
        r->v[0] = (t0 & keep) | (u0 & ~keep);                                                         \
        r->v[1] = (t1 & keep) | (u1 & ~keep);                                                         \
        r->v[2] = (t2 & keep) | (u2 & ~keep);                                                         \
        r->v[3] = (t3 & keep) | (u3 & ~keep);                                                         \
    }

#define PF_DEFINE_ADDSUB(PREFIX, P0, P1, P2, P3)                                                      \
    static inline void PREFIX##_add(fp_t *r, const fp_t *a, const fp_t *b) {                          \
        pu128 s;                                                                                      \
        uint64_t t0, t1, t2, t3, c;                                                                   \
        s = (pu128)a->v[0] + b->v[0]; t0 = (uint64_t)s; c = (uint64_t)(s >> 64);                      \
        s = (pu128)a->v[1] + b->v[1] + c; t1 = (uint64_t)s; c = (uint64_t)(s >> 64);                  \
        s = (pu128)a->v[2] + b->v[2] + c; t2 = (uint64_t)s; c = (uint64_t)(s >> 64);                  \
        s = (pu128)a->v[3] + b->v[3] + c; t3 = (uint64_t)s;                                           \
        pu128 d;                                                                                      \
        uint64_t u0, u1, u2, u3, bw;                                                                  \
        d = (pu128)t0 - (P0); u0 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                          \
        d = (pu128)t1 - (P1) - bw; u1 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                     \
        d = (pu128)t2 - (P2) - bw; u2 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                     \
        d = (pu128)t3 - (P3) - bw; u3 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                     \
        const uint64_t keep = (uint64_t)0 - bw;                                                       \
        r->v[0] = (t0 & keep) | (u0 & ~keep);                                                         \
        r->v[1] = (t1 & keep) | (u1 & ~keep);                                                         \
        r->v[2] = (t2 & keep) | (u2 & ~keep);                                                         \
        r->v[3] = (t3 & keep) | (u3 & ~keep);                                                         \
    }                                                                                                 \
    static inline void PREFIX##_sub(fp_t *r, const fp_t *a, const fp_t *b) {                          \
        pu128 d;                                                                                      \
        uint64_t t0, t1, t2, t3, bw;                                                                  \
        d = (pu128)a->v[0] - b->v[0]; t0 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;                  \
        d = (pu128)a->v[1] - b->v[1] - bw; t1 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;             \
        d = (pu128)a->v[2] - b->v[2] - bw; t2 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;             \
        d = (pu128)a->v[3] - b->v[3] - bw; t3 = (uint64_t)d; bw = (uint64_t)(d >> 64) & 1;             \
        const uint64_t m_ = (uint64_t)0 - bw; /* add p back on a borrow (branch-free) */              \
        pu128 s;                                                                                      \
        uint64_t c;                                                                                   \
        s = (pu128)t0 + ((P0) & m_); t0 = (uint64_t)s; c = (uint64_t)(s >> 64);                       \
        s = (pu128)t1 + ((P1) & m_) + c; t1 = (uint64_t)s; c = (uint64_t)(s >> 64);                   \
        s = (pu128)t2 + ((P2) & m_) + c; t2 = (uint64_t)s; c = (uint64_t)(s >> 64);                   \
        t3 = t3 + ((P3) & m_) + c;                                                                    \
        r->v[0] = t0; r->v[1] = t1; r->v[2] = t2; r->v[3] = t3;                                       \
    }

PF_DEFINE_MUL(pq_mul, PF_Q0, PF_Q1, PF_Q2, PF_Q3, PF_QN0)
PF_DEFINE_MUL(pr_mul, PF_R0, PF_R1, PF_R2, PF_R3, PF_RN0)
PF_DEFINE_ADDSUB(pq, PF_Q0, PF_Q1, PF_Q2, PF_Q3)
PF_DEFINE_ADDSUB(pr, PF_R0, PF_R1, PF_R2, PF_R3)

static inline int pf_is_zero(const fp_t *a) { return (a->v[0] | a->v[1] | a->v[2] | a->v[3]) == 0; }
static inline int pf_eq(const fp_t *a, const fp_t *b) {
    return ((a->v[0] ^ b->v[0]) | (a->v[1] ^ b->v[1]) | (a->v[2] ^ b->v[2]) | (a->v[3] ^ b->v[3])) == 0;
}
static inline void pq_sqr(fp_t *r, const fp_t *a) { pq_mul(r, a, a); }
static inline void pq_dbl(fp_t *r, const fp_t *a) { pq_add(r, a, a); }
static inline void pq_neg(fp_t *r, const fp_t *a) {
    static const fp_t zero = {{0, 0, 0, 0}};
    pq_sub(r, &zero, a);
}

/* ---- Fq2 = Fq[u]/(u^2 + 1), Karatsuba product ---- */
static inline void pq2_add(fq2_t *r, const fq2_t *a, const fq2_t *b) {
    pq_add(&r->c0, &a->c0, &b->c0);
    pq_add(&r->c1, &a->c1, &b->c1);
}
static inline void pq2_sub(fq2_t *r, const fq2_t *a, const fq2_t *b) {
    pq_sub(&r->c0, &a->c0, &b->c0);
    pq_sub(&r->c1, &a->c1, &b->c1);
}
static inline void pq2_dbl(fq2_t *r, const fq2_t *a) { pq2_add(r, a, a); }
static inline void pq2_neg(fq2_t *r, const fq2_t *a) {
    pq_neg(&r->c0, &a->c0);
    pq_neg(&r->c1, &a->c1);
}
static inline void pq2_mul(fq2_t *r, const fq2_t *a, const fq2_t *b) {
    fp_t t0, t1, s0, s1, m;
    pq_mul(&t0, &a->c0, &b->c0);
    pq_mul(&t1, &a->c1, &b->c1);
    pq_add(&s0, &a->c0, &a->c1);
    pq_add(&s1, &b->c0, &b->c1);
    pq_mul(&m, &s0, &s1);
    pq_sub(&m, &m, &t0);
    pq_sub(&r->c1, &m, &t1);
    pq_sub(&r->c0, &t0, &t1);
}
static inline void pq2_sqr(fq2_t *r, const fq2_t *a) {
    /* (a0 + a1)(a0 - a1) + 2 a0 a1 u */
    fp_t s, d, p;
    pq_add(&s, &a->c0, &a->c1);
    pq_sub(&d, &a->c0, &a->c1);
    pq_mul(&p, &a->c0, &a->c1);
    pq_mul(&r->c0, &s, &d);
    pq_add(&r->c1, &p, &p);
}
static inline int pq2_is_zero(const fq2_t *a) { return pf_is_zero(&a->c0) && pf_is_zero(&a->c1); }
static inline int pq2_eq(const fq2_t *a, const fq2_t *b) { return pf_eq(&a->c0, &b->c0) && pf_eq(&a->c1, &b->c1); }

/* Tasks per parallel loop: a few per thread of the enclosing team, so that
 * loops balance without drowning in task overhead (thousands of small
 * OpenMP tasks measured several times slower than this). */
#ifdef _OPENMP
#include <omp.h>
static inline int port_tasks(void) { return 4 * omp_get_num_threads(); }
#else
static inline int port_tasks(void) { return 1; }
#endif

/* inverses by Fermat's little theorem over the fast product */
void pq_inv(fp_t *r, const fp_t *a);
void pq2_inv(fq2_t *r, const fq2_t *a);

#endif
