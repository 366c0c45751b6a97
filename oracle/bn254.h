/*
 * CPU ORACLE -- test infrastructure only.
 *
 * A plain-C restatement of the reference CPU prover (zemse/snarkrs) for the
 * Groth16 / BN254 hot path: field and curve arithmetic, the radix-2 NTT and
 * the prover's iNTT -> coset -> NTT chain, signed-digit Pippenger MSMs, the
 * stage-0 CSR gather, stage-11 assembly and the optimal-ate pairing check.
 *
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg may
 * load this code.  It is the checker the CUDA product is compared against,
 * never part of the product path.
 *
 * Representation (matches snarkrs' PackedFr / ark-ff in-memory Fp,
 * crates/gpu-layout/src/lib.rs:30-46): 4 x u64 little-endian limbs,
 * Montgomery form with R = 2^256, always fully reduced into [0, p).
 */
#ifndef G16_ORACLE_BN254_H
#define G16_ORACLE_BN254_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { uint64_t v[4]; } fp_t;

/* A prime field: modulus, -p^-1 mod 2^64, R mod p, R^2 mod p. */
typedef struct {
    uint64_t p[4];
    uint64_t n0;
    fp_t one;   /* R mod p: the Montgomery form of 1 */
    fp_t r2;    /* R^2 mod p */
} field_t;

extern field_t FR;   /* BN254 scalar field r */
extern field_t FQ;   /* BN254 base field q */

void bn254_init(void);   /* idempotent; computes derived constants */

/* ---- generic prime-field arithmetic (Montgomery, fully reduced) ---- */
void fp_add(const field_t *f, fp_t *r, const fp_t *a, const fp_t *b);
void fp_sub(const field_t *f, fp_t *r, const fp_t *a, const fp_t *b);
void fp_neg(const field_t *f, fp_t *r, const fp_t *a);
void fp_mul(const field_t *f, fp_t *r, const fp_t *a, const fp_t *b);
void fp_sqr(const field_t *f, fp_t *r, const fp_t *a);
void fp_pow(const field_t *f, fp_t *r, const fp_t *a, const uint64_t *e, int nlimbs);
void fp_inv(const field_t *f, fp_t *r, const fp_t *a);      /* 0 -> 0 */
void fp_to_mont(const field_t *f, fp_t *r, const fp_t *std_form);
void fp_from_mont(const field_t *f, fp_t *r, const fp_t *mont);
void fp_from_u64(const field_t *f, fp_t *r, uint64_t x);
int  fp_is_zero(const fp_t *a);
int  fp_eq(const fp_t *a, const fp_t *b);
int  fp_lt_modulus(const field_t *f, const fp_t *raw);          /* raw < p */
int  fp_sqrt(const field_t *f, fp_t *r, const fp_t *a);          /* q = 3 mod 4 only */

/* ---- Fq2 = Fq[u]/(u^2 + 1) ---- */
typedef struct { fp_t c0, c1; } fq2_t;
void fq2_add(fq2_t *r, const fq2_t *a, const fq2_t *b);
void fq2_sub(fq2_t *r, const fq2_t *a, const fq2_t *b);
void fq2_neg(fq2_t *r, const fq2_t *a);
void fq2_mul(fq2_t *r, const fq2_t *a, const fq2_t *b);
void fq2_sqr(fq2_t *r, const fq2_t *a);
void fq2_inv(fq2_t *r, const fq2_t *a);
void fq2_conj(fq2_t *r, const fq2_t *a);
void fq2_mul_fq(fq2_t *r, const fq2_t *a, const fp_t *b);
void fq2_mul_xi(fq2_t *r, const fq2_t *a);   /* times xi = 9 + u */
void fq2_pow(fq2_t *r, const fq2_t *a, const uint64_t *e, int nlimbs);
int  fq2_is_zero(const fq2_t *a);
int  fq2_eq(const fq2_t *a, const fq2_t *b);
int  fq2_sqrt(fq2_t *r, const fq2_t *a);
void fq2_set_one(fq2_t *r);

/* ---- Fq6 = Fq2[v]/(v^3 - xi), Fq12 = Fq6[w]/(w^2 - v) ---- */
typedef struct { fq2_t c0, c1, c2; } fq6_t;
typedef struct { fq6_t c0, c1; } fq12_t;
void fq12_set_one(fq12_t *r);
void fq12_mul(fq12_t *r, const fq12_t *a, const fq12_t *b);
void fq12_sqr(fq12_t *r, const fq12_t *a);
void fq12_inv(fq12_t *r, const fq12_t *a);
void fq12_conj(fq12_t *r, const fq12_t *a);
void fq12_frob(fq12_t *r, const fq12_t *a);           /* a^q */
int  fq12_is_one(const fq12_t *a);
int  fq12_eq(const fq12_t *a, const fq12_t *b);

/* ---- G1 over Fq (y^2 = x^3 + 3), G2 over Fq2 (y^2 = x^3 + 3/(9+u)) ---- */
typedef struct { fp_t x, y; int inf; } g1a_t;           /* affine */
typedef struct { fp_t x, y, z; } g1j_t;                 /* Jacobian, z = 0 is infinity */
typedef struct { fq2_t x, y; int inf; } g2a_t;
typedef struct { fq2_t x, y, z; } g2j_t;

extern g1a_t G1_GEN;
extern g2a_t G2_GEN;

void g1j_set_inf(g1j_t *r);
int  g1j_is_inf(const g1j_t *a);
void g1j_from_affine(g1j_t *r, const g1a_t *a);
void g1j_dbl(g1j_t *r, const g1j_t *a);
void g1j_add(g1j_t *r, const g1j_t *a, const g1j_t *b);
void g1j_add_affine(g1j_t *r, const g1j_t *a, const g1a_t *b);
void g1j_neg(g1j_t *r, const g1j_t *a);
void g1j_to_affine(g1a_t *r, const g1j_t *a);
void g1j_mul(g1j_t *r, const g1j_t *a, const fp_t *scalar_std);   /* scalar in standard form */
int  g1a_on_curve(const g1a_t *a);
int  g1a_eq(const g1a_t *a, const g1a_t *b);

void g2j_set_inf(g2j_t *r);
int  g2j_is_inf(const g2j_t *a);
void g2j_from_affine(g2j_t *r, const g2a_t *a);
void g2j_dbl(g2j_t *r, const g2j_t *a);
void g2j_add(g2j_t *r, const g2j_t *a, const g2j_t *b);
void g2j_add_affine(g2j_t *r, const g2j_t *a, const g2a_t *b);
void g2j_neg(g2j_t *r, const g2j_t *a);
void g2j_to_affine(g2a_t *r, const g2j_t *a);
void g2j_mul(g2j_t *r, const g2j_t *a, const fp_t *scalar_std);
int  g2a_on_curve(const g2a_t *a);
int  g2a_in_subgroup(const g2a_t *a);
int  g2a_eq(const g2a_t *a, const g2a_t *b);

/* ---- pairing ---- */
void miller_loop(fq12_t *f, const g1a_t *p, const g2a_t *q);
void final_exponentiation(fq12_t *r, const fq12_t *f);
/* prod_i e(p[i], q[i]) == 1 ?  pairs with an infinity point contribute 1. */
int  pairing_product_is_one(const g1a_t *p, const g2a_t *q, int n);

#ifdef __cplusplus
}
#endif
#endif
